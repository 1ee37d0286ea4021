// The reference's callable contact methods and contact-Jacobian classes through the drop-in:
// contact_kdtree / contact_brute_force constructed from their ContactsParams and run on a
// container (test/test_contacts_kdtree.cpp:14-73, test/test_contacts_brute_force.cpp:12-71),
// and AMatrix / ATMatrix built on the returned contacts (test/test_matrices.cpp:17-79): the
// same scenes and checks, with std::vector in place of xtensor and a small relative-tolerance
// check in place of doctest::Approx (same default epsilon).  Runs on the GPU; exits non-zero
// on a mismatch and prints the checked values as JSON.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include <scopi/contact/contact_brute_force.hpp>
#include <scopi/contact/contact_kdtree.hpp>
#include <scopi/container.hpp>
#include <scopi/matrix/velocities.hpp>
#include <scopi/objects/types/plane.hpp>
#include <scopi/objects/types/sphere.hpp>

static int failures = 0;
static bool approx(double a, double b) {
    const double eps = 1.1920928955078125e-07 * 100;  // doctest::Approx's default epsilon
    return std::fabs(a - b) < eps * (1.0 + std::max(std::fabs(a), std::fabs(b)));
}
#define CHECK(c)                                                 \
    do {                                                         \
        if (!(c)) {                                              \
            std::fprintf(stderr, "line %d: %s\n", __LINE__, #c); \
            ++failures;                                          \
        }                                                        \
    } while (0)

namespace scopi {

static constexpr double PI = 3.14159265358979323846;  // the reference tests' own constant (test/utils.hpp)

// three disks, one pair within reach: the pair (0, 1) and its geometry
template <class Contacts>
static void check_three_disks(const Contacts& contacts) {
    CHECK(contacts.size() == 1);
    if (contacts.empty()) return;
    CHECK(contacts[0].i == 0 && contacts[0].j == 1);
    CHECK(approx(contacts[0].dij, std::sqrt(2.) - 0.1 - 0.2));
    CHECK(approx(contacts[0].nij(0), -1. / std::sqrt(2.)) && approx(contacts[0].nij(1), -1. / std::sqrt(2.)));
    CHECK(approx(contacts[0].pi(0), 0.1 * std::sqrt(2.) / 2.) && approx(contacts[0].pi(1), 0.1 * std::sqrt(2.) / 2.));
    CHECK(approx(contacts[0].pj(0), 1. - 0.2 * std::sqrt(2.) / 2.) &&
          approx(contacts[0].pj(1), 1. - 0.2 * std::sqrt(2.) / 2.));
}

static void three_disks(scopi_container<2>& particles) {
    sphere<2> s1({{0., 0.}}, 0.1);
    sphere<2> s2({{1., 1.}}, 0.2);
    sphere<2> s3({{5., 10.}}, 0.1);
    particles.push_back(s1);
    particles.push_back(s2);
    particles.push_back(s3);
}

static void contacts_kdtree() {
    scopi_container<2> particles;
    three_disks(particles);
    ContactsParams<contact_kdtree<NoFriction>> params;
    params.kd_tree_radius = 100.;
    contact_kdtree cont(params);
    auto contacts = cont.run(particles);
    check_three_disks(contacts);
}

static void contacts_brute_force() {
    scopi_container<2> particles;
    three_disks(particles);
    ContactsParams<contact_brute_force<NoFriction>> params;
    contact_brute_force cont(params);
    auto contacts = cont.run(particles);
    check_three_disks(contacts);
}

// A and its adjoint: dot(A u, f) == dot(u, A^T f) for random u, f
static double matrix_adjoint() {
    scopi_container<3> particles;
    sphere<3> s1({{0., 0., 0.}}, 0.1);
    sphere<3> s2({{1., 1., 0.}}, 0.2);
    particles.push_back(s1);
    particles.push_back(s2);
    ContactsParams<contact_brute_force<NoFriction>> params;
    contact_brute_force cont(params);
    auto contacts = cont.run(particles);
    AMatrix a(contacts, particles);
    ATMatrix at(contacts, particles);
    std::mt19937 gen(7);
    std::uniform_real_distribution<double> uni(0., 1.);
    std::vector<double> u(6 * particles.nb_active()), f(3 * contacts.size());
    for (auto& x : u) x = uni(gen);
    for (auto& x : f) x = uni(gen);
    const auto& au = a.mat_mult(u);
    double lhs = 0.0;
    for (std::size_t k = 0; k < f.size(); ++k) lhs += au[k] * f[k];
    const auto& atf = at.mat_mult(f);
    double rhs = 0.0;
    for (std::size_t k = 0; k < u.size(); ++k) rhs += u[k] * atf[k];
    CHECK(contacts.size() == 1);
    CHECK(approx(lhs, rhs));
    return lhs - rhs;
}

// a disk on an inclined plane: known values of A u
static void matrix_case2(double* out) {
    scopi_container<2> particles;
    sphere<2> s({{2., 1.}}, 0.5);
    plane<2> p({{0., 0.}}, PI / 2 - PI / 4);
    particles.push_back(p, property<2>().deactivate());
    particles.push_back(s, property<2>().mass(1).moment_inertia(0.1));
    ContactsParams<contact_brute_force<NoFriction>> params;
    contact_brute_force<NoFriction> cont(params);
    auto contacts = cont.run(particles);
    AMatrix a(contacts, particles);
    std::vector<double> u{0.187562190766376, -1.184390935327111, 0., 0., 0., -0.00453709103433};
    const auto& sol = a.mat_mult(u);
    CHECK(sol.size() == 3);
    CHECK(approx(sol[0], -0.18595809) && approx(sol[1], 1.18278683));
    out[0] = sol[0];
    out[1] = sol[1];
}

}  // namespace scopi

int main() {
    scopi::contacts_kdtree();
    scopi::contacts_brute_force();
    const double adj = scopi::matrix_adjoint();
    double case2[2] = {0., 0.};
    scopi::matrix_case2(case2);
    std::printf("{\"failures\": %d, \"adjoint_difference\": %.17g, \"case2\": [%.17g, %.17g]}\n", failures, adj,
                case2[0], case2[1]);
    return failures == 0 ? 0 : 1;
}
