// Drop-in check: a periodic BoxDomain (box.hpp) through the scopi:: API, ScopiSolver(box,
// particles) as in the reference (solver.hpp:117): two disks meet across the bound x = 0 of
// the box [0, 4] (periodic along x).  Prints the final positions as JSON.
#include <cstdio>

#include <scopi/box.hpp>
#include <scopi/container.hpp>
#include <scopi/objects/types/sphere.hpp>
#include <scopi/property.hpp>
#include <scopi/solver.hpp>
#include <scopi/solvers/OptimGradient.hpp>
#include <scopi/solvers/apgd.hpp>
#include <scopi/vap/vap_fixed.hpp>

int main() {
    constexpr std::size_t dim = 2;
    scopi::scopi_container<dim> particles;
    particles.push_back(scopi::sphere<dim>({{0.3, 0.}}, 0.25),
                        scopi::property<dim>().mass(1.).moment_inertia(0.1).desired_velocity({{-0.5, 0.}}));
    particles.push_back(scopi::sphere<dim>({{3.7, 0.}}, 0.25),
                        scopi::property<dim>().mass(1.).moment_inertia(0.1).desired_velocity({{0.5, 0.}}));
    scopi::BoxDomain<dim> box({0., 0.}, {4., 0.});
    box.with_periodicity(0);
    scopi::ScopiSolver<dim, scopi::NoFriction, scopi::OptimGradient<scopi::apgd>, scopi::contact_kdtree,
                       scopi::vap_fixed>
        solver(box, particles);
    auto params = solver.get_params();
    params.optim_params.tolerance = 1e-10;
    params.optim_params.max_ite = 20000;
    params.optim_params.alpha = 0.1;
    params.contact_method_params.dmax = 0.5;
    solver.run(0.01, 40);
    std::printf("{\"positions\": [[%.17g, %.17g], [%.17g, %.17g]], \"contacts\": %zu}\n", particles.pos()(0)(0),
                particles.pos()(0)(1), particles.pos()(1)(0), particles.pos()(1)(1), solver.current_contacts().size());
    return 0;
}
