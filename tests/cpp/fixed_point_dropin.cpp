// Drop-in check for FrictionFixedPoint: the reference's "sphere - plane friction fixed point"
// test (test/test_gradient.cpp:215-283) written against the scopi:: API as the reference
// writes it.  Prints the sphere's final state as JSON for the Python side to compare with
// the analytic rolling solution.
#include <cmath>
#include <cstdio>

#include <scopi/container.hpp>
#include <scopi/objects/types/plane.hpp>
#include <scopi/objects/types/sphere.hpp>
#include <scopi/property.hpp>
#include <scopi/solver.hpp>
#include <scopi/solvers/OptimGradient.hpp>
#include <scopi/solvers/apgd.hpp>
#include <scopi/vap/vap_fpd.hpp>

int main() {
    constexpr std::size_t dim = 2;
    const double PI = 4 * std::atan(1.0);
    scopi::scopi_container<dim> particles;
    double radius = 1.;
    double g = 1.;
    double dt = 0.01;
    std::size_t total_it = 500;
    double h = 2. * radius;
    double alpha = PI / 4;
    scopi::plane<dim> plane({{0., 0.}}, PI / 2);
    scopi::sphere<dim> sphere({{0, h}}, radius);
    particles.push_back(plane, scopi::property<dim>().deactivate());
    particles.push_back(sphere, scopi::property<dim>()
                                    .mass(1)
                                    .moment_inertia(1. * radius * radius / 2.)
                                    .force({{g * std::sin(alpha), -g * std::cos(alpha)}}));
    using problem_t = scopi::FrictionFixedPoint;
    using optim_solver = scopi::OptimGradient<scopi::apgd>;
    scopi::ScopiSolver<dim, problem_t, optim_solver, scopi::contact_kdtree, scopi::vap_fpd> solver(particles);
    auto params = solver.get_params();
    params.optim_params.tolerance = 1e-7;
    params.optim_params.max_ite = 10000;
    params.optim_params.alpha = 0.01;
    params.optim_params.dynamic_descent = true;
    params.default_contact_property.mu = 0.5;
    params.default_contact_property.fixed_point_tol = 1e-6;
    params.default_contact_property.fixed_point_max_iter = 1000;
    solver.run(dt, total_it);
    auto p = particles.pos()(1);
    auto v = particles.v()(1);
    auto q = particles.q()(1);
    std::printf("{\"position\": [%.17g, %.17g], \"velocity\": [%.17g, %.17g], \"omega\": %.17g, "
                "\"quaternion\": [%.17g, %.17g, %.17g, %.17g]}\n",
                p(0), p(1), v(0), v(1), particles.omega()(1), q(0), q(1), q(2), q(3));
    return 0;
}
