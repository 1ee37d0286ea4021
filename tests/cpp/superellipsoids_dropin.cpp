// Drop-in check for superellipsoids: a scene of superellipsoids on a plane with friction,
// built with the reference's 3D constructors (include/scopi/objects/types/superellipsoid.hpp:59-70,
// plane.hpp, property.hpp) and stepped through ScopiSolver<3, Friction, ..., vap_fpd>.
// The scene comes from a text file (one body per line) so that the Python side can hand
// it the same bodies it gives the oracle; the final state is printed as JSON.
#include <cstdio>
#include <fstream>
#include <iostream>

#include <scopi/container.hpp>
#include <scopi/objects/types/plane.hpp>
#include <scopi/objects/types/superellipsoid.hpp>
#include <scopi/property.hpp>
#include <scopi/solver.hpp>
#include <scopi/solvers/OptimGradient.hpp>
#include <scopi/solvers/apgd.hpp>
#include <scopi/vap/vap_fpd.hpp>

int main(int argc, char** argv) {
    constexpr std::size_t dim = 3;
    if (argc < 2) return 2;
    std::ifstream in(argv[1]);
    std::size_t n = 0, steps = 0;
    double dt, mu, dmax, kd, tol;
    std::size_t max_ite;
    in >> n >> steps >> dt >> mu >> dmax >> kd >> tol >> max_ite;
    scopi::scopi_container<dim> particles;
    for (std::size_t b = 0; b < n; ++b) {
        int shape, active;
        std::array<double, 3> c, r, j, f, v;
        std::array<double, 4> q;
        std::array<double, 2> sq;
        double m;
        in >> shape >> active;
        for (auto& x : c) in >> x;
        for (auto& x : q) in >> x;
        for (auto& x : r) in >> x;
        for (auto& x : sq) in >> x;
        in >> m;
        for (auto& x : j) in >> x;
        for (auto& x : f) in >> x;
        for (auto& x : v) in >> x;
        auto prop = scopi::property<dim>().mass(m).moment_inertia(j).force(f).velocity(v);
        if (!active) prop.deactivate();
        if (shape == SCOPI_GPU_PLANE) {
            scopi::plane<dim> p({c}, {q});
            particles.push_back(p, prop);
        } else {
            scopi::superellipsoid<dim> s({c}, {q}, {r}, {sq});
            particles.push_back(s, prop);
        }
    }
    if (!in) return 3;
    using optim_solver = scopi::OptimGradient<scopi::apgd>;
    scopi::ScopiSolver<dim, scopi::Friction, optim_solver, scopi::contact_kdtree, scopi::vap_fpd> solver(particles);
    auto params = solver.get_params();
    params.optim_params.tolerance = tol;
    params.optim_params.max_ite = max_ite;
    params.default_contact_property.mu = mu;
    params.contact_method_params.dmax = dmax;
    params.contact_method_params.kd_tree_radius = kd;
    solver.run(dt, steps);
    std::printf("{\"positions\": [");
    for (std::size_t i = 0; i < particles.size(); ++i) {
        auto p = particles.pos()(i);
        std::printf("%s[%.17g, %.17g, %.17g]", i ? ", " : "", p(0), p(1), p(2));
    }
    const auto& cc = solver.current_contacts();
    std::printf("], \"contacts\": [");
    for (std::size_t k = 0; k < cc.size(); ++k) std::printf("%s[%zu, %zu]", k ? ", " : "", cc[k].i, cc[k].j);
    std::printf("]}\n");
    return 0;
}
