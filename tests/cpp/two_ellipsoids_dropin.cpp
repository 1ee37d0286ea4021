// Drop-in check for 2D superellipsoids: the "two ellipsoids" scenes of the reference's
// superellipsoid tests (test/test_superellipsoid.cpp:451-628) written against the scopi::
// API as the reference writes them (superellipsoid<2>(pos, {q}, {{rx, ry}}, e), default
// ScopiSolver<2>).  Argument: symmetrical | asymmetrical.  Prints the state after
// total_it - 1 steps, then runs one more step and prints its contacts (detected on that
// state), as JSON.
#include <cmath>
#include <cstdio>
#include <cstring>

#include <scopi/container.hpp>
#include <scopi/objects/types/superellipsoid.hpp>
#include <scopi/property.hpp>
#include <scopi/solver.hpp>

int main(int argc, char** argv) {
    constexpr std::size_t dim = 2;
    const bool asym = argc > 1 && std::strcmp(argv[1], "asymmetrical") == 0;
    const double PI = 4 * std::atan(1.0);
    const double dy = asym ? 0.05 : 0.0;
    const std::size_t total_it = asym ? 1000 : 200;
    double dt = .005;
    scopi::superellipsoid<dim> s1({{-0.2, -dy}}, {scopi::quaternion(PI / 4)}, {{.1, .05}}, 1);
    scopi::superellipsoid<dim> s2({{0.2, dy}}, {scopi::quaternion(-PI / 4)}, {{.1, .05}}, 1);
    auto p = scopi::property<dim>().desired_velocity({{0.25, 0}}).mass(1.).moment_inertia(0.1);
    scopi::scopi_container<dim> particles;
    particles.push_back(s1, p);
    particles.push_back(s2, p.desired_velocity({{-0.25, 0}}));
    scopi::ScopiSolver<dim> solver(particles);
    solver.run(dt, total_it - 1);
    std::printf("{\"objects\": [");
    for (std::size_t i = 0; i < particles.size(); ++i) {
        auto x = particles.pos()(i);
        auto q = particles.q()(i);
        std::printf("%s{\"position\": [%.17g, %.17g], \"quaternion\": [%.17g, %.17g, %.17g, %.17g]}", i ? ", " : "",
                    x(0), x(1), q(0), q(1), q(2), q(3));
    }
    solver.run(dt, 1);
    const auto& cc = solver.current_contacts();
    std::printf("], \"contacts\": [");
    for (std::size_t k = 0; k < cc.size(); ++k)
        std::printf("%s{\"nij\": [%.17g, %.17g], \"pi\": [%.17g, %.17g], \"pj\": [%.17g, %.17g]}", k ? ", " : "",
                    cc[k].nij[0], cc[k].nij[1], cc[k].pi[0], cc[k].pi[1], cc[k].pj[0], cc[k].pj[1]);
    std::printf("]}\n");
    return 0;
}
