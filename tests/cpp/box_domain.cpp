// BoxDomain<dim> (box.hpp) of the drop-in, without a GPU: default box, corners, the three
// with_periodicity forms and the accessors.  Exits non-zero on a mismatch.
#include <cstdio>

#include <scopi/box.hpp>

static int failures = 0;
#define CHECK(c)                                                      \
    do {                                                              \
        if (!(c)) {                                                   \
            std::fprintf(stderr, "line %d: %s\n", __LINE__, #c);      \
            ++failures;                                               \
        }                                                             \
    } while (0)

int main() {
    scopi::BoxDomain<2> none;
    CHECK(!none.is_periodic(0) && !none.is_periodic(1));
    CHECK(none.lower_bound(0) == 0. && none.upper_bound(1) == 0.);
    scopi::BoxDomain<2> box({0., -1.}, {4., 2.});
    CHECK(!box.is_periodic(0) && !box.is_periodic(1));
    box.with_periodicity(0);
    CHECK(box.is_periodic(0) && !box.is_periodic(1));
    CHECK(box.lower_bound(0) == 0. && box.upper_bound(0) == 4. && box.lower_bound(1) == -1. && box.upper_bound(1) == 2.);
    CHECK(box.min_corner()[1] == -1. && box.max_corner()[0] == 4.);
    scopi::BoxDomain<3> b3({0., 0., 0.}, {1., 2., 3.});
    b3.with_periodicity({0, 2});
    CHECK(b3.is_periodic(0) && !b3.is_periodic(1) && b3.is_periodic(2));
    scopi::BoxDomain<3> all({0., 0., 0.}, {1., 1., 1.});
    all.with_periodicity();
    CHECK(all.is_periodic()[0] && all.is_periodic()[1] && all.is_periodic()[2]);
    std::printf("%d failures\n", failures);
    return failures == 0 ? 0 : 1;
}
