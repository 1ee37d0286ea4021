// The reference's worm construction tests (test/test_worm.cpp:26-478: "Worm 2D", "Worm 2D
// const", "Worm 3D", "Worm 3D const") against the drop-in's worm<dim> and scopi_container,
// without a GPU: the positions and quaternions of the spheres read through the worm and
// through the container's object access, the radius and the size.  Exits non-zero on a
// mismatch.
#include <cmath>
#include <cstdio>

#include <scopi/container.hpp>
#include <scopi/objects/types/worm.hpp>
#include <scopi/property.hpp>

static int failures = 0;
static void check(bool ok, const char* what, int line) {
    if (!ok) {
        std::fprintf(stderr, "line %d: %s\n", line, what);
        ++failures;
    }
}
#define CHECK_NEAR(a, b) check(std::abs((a) - (b)) <= 1e-12 * (1 + std::abs(b)), #a " == " #b, __LINE__)

template <std::size_t dim, class W, class C>
void check_worm(const W& w, C& particles, double z) {
    for (std::size_t i = 0; i < 6; ++i) {
        const double x = 2. + 2. * (double)i;
        CHECK_NEAR(w.pos(i)(0), x);
        CHECK_NEAR(w.pos(i)(1), 0.7);
        CHECK_NEAR(particles[0]->pos(i)(0), x);
        CHECK_NEAR(particles[0]->pos(i)(1), 0.7);
        if constexpr (dim == 3) {
            CHECK_NEAR(w.pos(i)(2), z);
            CHECK_NEAR(particles[0]->pos(i)(2), z);
        }
        for (std::size_t d = 0; d < 4; ++d) {
            CHECK_NEAR(w.q(i)(d), d == 0 ? 1. : 0.);
            CHECK_NEAR(particles[0]->q(i)(d), d == 0 ? 1. : 0.);
        }
    }
    CHECK_NEAR(w.radius(), 1.);
    check(w.size() == 6, "size", __LINE__);
    check(particles.nb_objects() == 1 && particles.size() == 6, "container: one object of six bodies", __LINE__);
}

int main() {
    using scopi::quaternion;
    {
        constexpr std::size_t dim = 2;
        scopi::worm<dim> w({{2., 0.7}, {4., 0.7}, {6., 0.7}, {8., 0.7}, {10., 0.7}, {12., 0.7}},
                           {{quaternion(0.)}, {quaternion(0.)}, {quaternion(0.)}, {quaternion(0.)}, {quaternion(0.)},
                            {quaternion(0.)}},
                           1., 6);
        scopi::property<dim> p(scopi::property<dim>().desired_velocity({{0.25, 0}}));
        scopi::scopi_container<dim> particles;
        particles.push_back(w, p);
        check_worm<dim>(w, particles, 0.);
        const scopi::worm<dim> wc = w;
        const scopi::property<dim> pc = p;
        scopi::scopi_container<dim> particles_c;
        particles_c.push_back(wc, pc);
        check_worm<dim>(wc, particles_c, 0.);
    }
    {
        constexpr std::size_t dim = 3;
        scopi::worm<dim> w({{2., 0.7, 0.2}, {4., 0.7, 0.2}, {6., 0.7, 0.2}, {8., 0.7, 0.2}, {10., 0.7, 0.2},
                            {12., 0.7, 0.2}},
                           {{quaternion(0.)}, {quaternion(0.)}, {quaternion(0.)}, {quaternion(0.)}, {quaternion(0.)},
                            {quaternion(0.)}},
                           1., 6);
        scopi::property<dim> p(scopi::property<dim>().desired_velocity({{0.25, 0, 0}}));
        scopi::scopi_container<dim> particles;
        particles.push_back(w, p);
        check_worm<dim>(w, particles, 0.2);
        const scopi::worm<dim> wc = w;
        scopi::scopi_container<dim> particles_c;
        particles_c.push_back(wc, p);
        check_worm<dim>(wc, particles_c, 0.2);
    }
    std::printf("%d failures\n", failures);
    return failures == 0 ? 0 : 1;
}
