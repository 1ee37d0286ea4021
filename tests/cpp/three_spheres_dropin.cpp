// Drop-in check: the "3 Spheres NoFriction / Viscous / Viscous Friction" scenes of the
// reference's solver tests (test/test_gradient.cpp:377-503, 574-642) written against the scopi:: API exactly as a
// reference user writes them; only the headers differ (B200 engine through the C ABI).
// Prints the final state as JSON for the Python side to compare with the golden files; with
// an output directory as second argument the solver also writes its snapshot files there,
// the last one after the final step (output_frequency = total_it).
#include <cstdio>
#include <cstring>
#include <type_traits>

#include <scopi/container.hpp>
#include <scopi/objects/types/sphere.hpp>
#include <scopi/property.hpp>
#include <scopi/solver.hpp>
#include <scopi/solvers/OptimGradient.hpp>
#include <scopi/solvers/apgd.hpp>
#include <scopi/vap/vap_fpd.hpp>

template <class problem_t>
int run(double Tf, const char* outdir, const char* name) {
    constexpr std::size_t dim = 2;
    scopi::scopi_container<dim> particles;
    scopi::sphere<dim> s1({{-1.7, 1.3}}, 0.5);
    scopi::sphere<dim> s2({{0.5, 1.7}}, 0.5);
    scopi::sphere<dim> s3({{4.5, 1.3}}, 0.5);
    particles.push_back(s1, scopi::property<dim>().mass(1).moment_inertia(1).force({{1.7, -1.3}}));
    particles.push_back(s2, scopi::property<dim>().mass(1).moment_inertia(1).force({{-0.5, -1.7}}));
    particles.push_back(s3, scopi::property<dim>().mass(1).moment_inertia(1).force({{-4.5, -1.3}}));
    double dt = 0.1;
    using optim_solver = scopi::OptimGradient<scopi::apgd>;
    scopi::ScopiSolver<dim, problem_t, optim_solver, scopi::contact_kdtree, scopi::vap_fpd> solver(particles);
    auto params = solver.get_params();
    params.optim_params.tolerance = 1e-7;
    params.optim_params.max_ite = 10000;
    params.optim_params.alpha = 0.1;
    params.optim_params.dynamic_descent = true;
    if constexpr (std::is_same_v<problem_t, scopi::ViscousFriction>) {
        params.default_contact_property.mu = 0.5;
        params.default_contact_property.fixed_point_tol = 1e-3;
        params.default_contact_property.fixed_point_max_iter = 1000;
        params.default_contact_property.gamma = 0;
        params.default_contact_property.gamma_min = -1.4;
        params.default_contact_property.gamma_tol = 1e-6;
    }
    std::size_t total_it = Tf / dt;
    if (outdir) {
        params.solver_params.output_frequency = total_it;
        params.solver_params.path = outdir;
        params.solver_params.filename = name;
    }
    solver.run(dt, total_it);
    std::printf("{\"objects\": [");
    for (std::size_t i = 0; i < particles.size(); ++i) {
        auto p = particles.pos()(i);
        auto v = particles.v()(i);
        auto q = particles.q()(i);
        std::printf("%s{\"position\": [%.17g, %.17g], \"velocity\": [%.17g, %.17g], \"omega\": [%.17g], "
                    "\"quaternion\": [%.17g, %.17g, %.17g, %.17g]}",
                    i ? ", " : "", p(0), p(1), v(0), v(1), particles.omega()(i), q(0), q(1), q(2), q(3));
    }
    std::printf("], \"contacts\": %zu}\n", solver.current_contacts().size());
    return 0;
}

int main(int argc, char** argv) {
    const char* outdir = argc > 2 ? argv[2] : nullptr;
    if (argc > 1 && std::strcmp(argv[1], "viscous") == 0) return run<scopi::Viscous>(7.0, outdir, "3spheres_viscous");
    if (argc > 1 && std::strcmp(argv[1], "viscous_friction") == 0)
        return run<scopi::ViscousFriction>(7.0, outdir, "3spheres_viscous_friction");
    return run<scopi::NoFriction>(6.0, outdir, "3spheres_nofriction");
}
