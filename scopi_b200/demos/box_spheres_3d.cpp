// Spheres falling into a box (the setting of the reference's demos/box_spheres_3d.cpp),
// written against the scopi:: API with the B200 policy types:
//   ScopiSolver<3, NoFriction, gpu::OptimGradient<gpu::apgd<gpu::mixed>>, gpu::contact_kdtree, gpu::vap_fpd>
// Build (from the repository root):
//   g++ -O2 -std=c++17 -I scopi_b200/include -I include scopi_b200/demos/box_spheres_3d.cpp
//       -L scopi_b200 -lscopi_gpu -Wl,-rpath,$PWD/scopi_b200 -o box_spheres_3d
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include <scopi/container.hpp>
#include <scopi/objects/types/plane.hpp>
#include <scopi/objects/types/sphere.hpp>
#include <scopi/solver.hpp>

int main(int argc, char** argv) {
    constexpr std::size_t dim = 3;
    const std::size_t n = argc > 1 ? std::strtoul(argv[1], nullptr, 10) : 20;  // n^3 spheres
    const std::size_t steps = argc > 2 ? std::strtoul(argv[2], nullptr, 10) : 50;
    const double PI = std::acos(-1.0);
    const double r0 = 0.5 / n / 2.0, g = 9.81, dt = 1e-3;
    scopi::scopi_container<dim> particles;
    const std::array<double, 3> ay{0., 1., 0.}, az{0., 0., 1.};
    // six planes bounding the unit box; the obstacles come first
    particles.push_back(scopi::plane<dim>({{0., 0., 0.}}, {scopi::quaternion(0., az)}), scopi::property<dim>().deactivate());
    particles.push_back(scopi::plane<dim>({{1., 0., 0.}}, {scopi::quaternion(0., az)}), scopi::property<dim>().deactivate());
    particles.push_back(scopi::plane<dim>({{0., 0., 0.}}, {scopi::quaternion(PI / 2, az)}), scopi::property<dim>().deactivate());
    particles.push_back(scopi::plane<dim>({{0., 1., 0.}}, {scopi::quaternion(PI / 2, az)}), scopi::property<dim>().deactivate());
    particles.push_back(scopi::plane<dim>({{0., 0., 0.}}, {scopi::quaternion(PI / 2, ay)}), scopi::property<dim>().deactivate());
    particles.push_back(scopi::plane<dim>({{0., 0., 1.}}, {scopi::quaternion(PI / 2, ay)}), scopi::property<dim>().deactivate());
    for (std::size_t i = 0; i < n; ++i)
        for (std::size_t j = 0; j < n; ++j)
            for (std::size_t k = 0; k < n; ++k) {
                const double x = 0.25 + (i + 0.5) * 2.2 * r0, y = 0.25 + (j + 0.5) * 2.2 * r0, z = 0.05 + (k + 0.5) * 2.2 * r0;
                const double m = 1.0, J = 0.4 * m * r0 * r0;
                particles.push_back(scopi::sphere<dim>({{x, y, z}}, r0),
                                    scopi::property<dim>().mass(m).moment_inertia({J, J, J}).force({{0., 0., -g * m}}));
            }
    using optim = scopi::gpu::OptimGradient<scopi::gpu::apgd<scopi::gpu::mixed>>;
    scopi::ScopiSolver<dim, scopi::NoFriction, optim, scopi::gpu::contact_kdtree, scopi::gpu::vap_fpd> solver(particles);
    auto params = solver.get_params();
    params.contact_method_params.dmax = 0.9 * r0;
    params.contact_method_params.kd_tree_radius = std::pow(2.2 * r0 + 0.9 * r0, 2);
    params.optim_params.tolerance = 1e-6;
    params.optim_params.max_ite = 40000;
    for (std::size_t s = 0; s < steps; s += 10) {
        solver.run(dt, 10);
        auto st = solver.stats();
        std::printf("step %zu: %lld contacts, %lld APGD iterations, violation %.2e, %.2f ms/step\n", s + 10,
                    (long long)st.contacts, (long long)st.iterations, st.violation, st.ms_step);
    }
    return 0;
}
