// Restart check: the reference's "3 Spheres NoFriction" scene (test/test_gradient.cpp:377-439)
// run for 60 steps at once ("continuous"), or run for 30 steps with a snapshot file, then
// rebuilt from that file with from_json (restart.hpp:20-67) and run by a new solver for the
// 30 steps left ("restart <dir>").  Prints the final state as JSON.
#include <cstdio>
#include <cstring>

#include <scopi/container.hpp>
#include <scopi/objects/types/sphere.hpp>
#include <scopi/property.hpp>
#include <scopi/restart.hpp>
#include <scopi/solver.hpp>
#include <scopi/solvers/OptimGradient.hpp>
#include <scopi/solvers/apgd.hpp>
#include <scopi/vap/vap_fpd.hpp>

constexpr std::size_t dim = 2;
using solver_t = scopi::ScopiSolver<dim, scopi::NoFriction, scopi::OptimGradient<scopi::apgd>, scopi::contact_kdtree,
                                    scopi::vap_fpd>;

void configure(solver_t& solver) {
    auto params = solver.get_params();
    params.optim_params.tolerance = 1e-7;
    params.optim_params.max_ite = 10000;
    params.optim_params.alpha = 0.1;
    params.optim_params.dynamic_descent = true;
}

void print(scopi::scopi_container<dim>& particles) {
    std::printf("{\"objects\": [");
    for (std::size_t i = 0; i < particles.size(); ++i) {
        auto p = particles.pos()(i);
        auto v = particles.v()(i);
        auto q = particles.q()(i);
        std::printf("%s{\"position\": [%.17g, %.17g], \"velocity\": [%.17g, %.17g], \"omega\": %.17g, "
                    "\"quaternion\": [%.17g, %.17g, %.17g, %.17g]}",
                    i ? ", " : "", p(0), p(1), v(0), v(1), particles.omega()(i), q(0), q(1), q(2), q(3));
    }
    std::printf("]}\n");
}

int main(int argc, char** argv) {
    const double dt = 0.1;
    scopi::scopi_container<dim> particles;
    scopi::sphere<dim> s1({{-1.7, 1.3}}, 0.5);
    scopi::sphere<dim> s2({{0.5, 1.7}}, 0.5);
    scopi::sphere<dim> s3({{4.5, 1.3}}, 0.5);
    particles.push_back(s1, scopi::property<dim>().mass(1).moment_inertia(1).force({{1.7, -1.3}}));
    particles.push_back(s2, scopi::property<dim>().mass(1).moment_inertia(1).force({{-0.5, -1.7}}));
    particles.push_back(s3, scopi::property<dim>().mass(1).moment_inertia(1).force({{-4.5, -1.3}}));
    if (argc > 2 && std::strcmp(argv[1], "restart") == 0) {
        {
            solver_t solver(particles);
            configure(solver);
            auto params = solver.get_params();
            params.solver_params.output_frequency = 30;
            params.solver_params.path = argv[2];
            params.solver_params.filename = "restart";
            solver.run(dt, 30);
        }
        auto restarted = scopi::from_json<dim>(std::filesystem::path(argv[2]) / "restart_0030.json");
        solver_t solver(restarted);
        configure(solver);
        solver.run(dt, 60, 30);
        print(restarted);
        return 0;
    }
    solver_t solver(particles);
    configure(solver);
    solver.run(dt, 60);
    print(particles);
    return 0;
}
