// Drop-in check: the reference's "two worms" solver test (test/test_worm.cpp:480-530) written
// against the scopi:: API as a reference user writes it; only the headers differ (B200 engine
// through the C ABI).  argv[1] = "kdtree" or "brute_force", argv[2] = output directory: the
// solver writes its snapshot files there (output_frequency = total_it), the last one after
// the final step, for the golden-file comparison of test/utils.cpp:14-75.
#include <cstring>
#include <string>

#include <scopi/container.hpp>
#include <scopi/objects/types/worm.hpp>
#include <scopi/property.hpp>
#include <scopi/solver.hpp>
#include <scopi/solvers/OptimGradient.hpp>
#include <scopi/solvers/apgd.hpp>
#include <scopi/vap/vap_fixed.hpp>

template <template <class> class contact_t>
int run(const char* outdir) {
    constexpr std::size_t dim = 2;
    double dt = .005;
    std::size_t total_it = 1000;
    scopi::scopi_container<dim> particles;
    auto prop = scopi::property<dim>().mass(1.).moment_inertia(0.1);
    scopi::worm<dim> w1({{1., 0.7}, {3., 0.7}, {5., 0.7}, {7., 0.7}, {9., 0.7}, {11., 0.7}},
                        {{scopi::quaternion(0.)}, {scopi::quaternion(0.)}, {scopi::quaternion(0.)},
                         {scopi::quaternion(0.)}, {scopi::quaternion(0.)}, {scopi::quaternion(0.)}},
                        1., 6);
    scopi::worm<dim> w2({{-1., -0.7}, {-3., -0.7}, {-5., -0.7}, {-7., -0.7}, {-9., -0.7}, {-11., -0.7}},
                        {{scopi::quaternion(0.)}, {scopi::quaternion(0.)}, {scopi::quaternion(0.)},
                         {scopi::quaternion(0.)}, {scopi::quaternion(0.)}, {scopi::quaternion(0.)}},
                        1., 6);
    particles.push_back(w1, prop.desired_velocity({{-1., 0.}}));
    particles.push_back(w2, prop.desired_velocity({{1., 0.}}));

    scopi::ScopiSolver<dim, scopi::NoFriction, scopi::OptimGradient<scopi::apgd>, contact_t, scopi::vap_fixed> solver(
        particles);
    auto params = solver.get_params();
    params.contact_method_params.dmax = 1.;
    params.solver_params.output_frequency = total_it;
    params.solver_params.filename = "two_worms";
    params.solver_params.path = outdir;
    solver.run(dt, total_it);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    if (std::strcmp(argv[1], "brute_force") == 0) return run<scopi::contact_brute_force>(argv[2]);
    return run<scopi::contact_kdtree>(argv[2]);
}
