// The snapshot writer of the C++ drop-in (write_output_files, solver.hpp:368-438) and its
// reader (from_json, restart.hpp:20-67) on containers of every shape, without a GPU: writes
// the "objects" document of a 2D and a 3D container as JSON and as BSON into the directory
// given as argument, each read back and written again (*_rt.json); with a snapshot file as
// second argument, that file read and written again as snapfile_rt.json.
#include <cmath>
#include <fstream>

#include <scopi/container.hpp>
#include <scopi/objects/types/plane.hpp>
#include <scopi/objects/types/segment.hpp>
#include <scopi/objects/types/sphere.hpp>
#include <scopi/objects/types/superellipsoid.hpp>
#include <scopi/property.hpp>
#include <scopi/restart.hpp>
#include <scopi/solver.hpp>

template <std::size_t dim>
void write(const scopi::scopi_container<dim>& c, const std::string& base) {
    scopi::io::Value doc = scopi::io::Value::object();
    doc.set("objects", c.snapshot_objects());
    doc.set("contacts", scopi::io::Value());
    std::ofstream j(base + ".json");
    scopi::io::write_json(j, doc);
    const auto b = scopi::io::to_bson(doc);
    std::ofstream f(base + ".bson", std::ios::binary);
    f.write(reinterpret_cast<const char*>(b.data()), (std::streamsize)b.size());
}
template <std::size_t dim>
void round_trip(const std::string& in, const std::string& out) {
    const scopi::scopi_container<dim> c = scopi::from_json<dim>(std::filesystem::path(in));
    scopi::io::Value doc = scopi::io::Value::object();
    doc.set("objects", c.snapshot_objects());
    doc.set("contacts", scopi::io::Value());
    std::ofstream j(out);
    scopi::io::write_json(j, doc);
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    const double PI = 4 * std::atan(1.0);
    {
        scopi::scopi_container<2> p;
        p.push_back(scopi::plane<2>({{0., 0.}}, PI / 3), scopi::property<2>().deactivate());
        p.push_back(scopi::segment<2>({{-1., 0.5}}, {{2., 1.5}}), scopi::property<2>().deactivate());
        p.push_back(scopi::sphere<2>({{0.3, 1.2}}, 0.25),
                    scopi::property<2>().mass(2.).moment_inertia(0.3).velocity({{1., -2.}}).force({{0., -9.81}}));
        p.push_back(scopi::superellipsoid<2>({{1.5, 2.}}, {scopi::quaternion(PI / 5)}, {{0.2, 0.1}}, 1.2),
                    scopi::property<2>().desired_velocity({{0.25, 0.}}).omega(0.5));
        write(p, dir + "/snap2d");
    }
    {
        scopi::scopi_container<3> p;
        p.push_back(scopi::sphere<3>({{1., 2., 3.}}, 0.5),
                    scopi::property<3>().mass(3.).moment_inertia({{0.1, 0.2, 0.3}}).omega({{1., 2., 3.}}));
        p.push_back(scopi::superellipsoid<3>({{0., 0., 1.}}, {scopi::quaternion(PI / 7, {{0., 1., 0.}})},
                                             {{0.3, 0.2, 0.1}}, {{0.8, 1.3}}),
                    scopi::property<3>().velocity({{0., 0., -1.}}));
        write(p, dir + "/snap3d");
    }
    round_trip<2>(dir + "/snap2d.json", dir + "/snap2d_rt.json");
    round_trip<3>(dir + "/snap3d.json", dir + "/snap3d_rt.json");
    if (argc > 2) round_trip<2>(argv[2], dir + "/snapfile_rt.json");
    if (argc > 3) round_trip<2>(argv[3], dir + "/wormfile_rt.json");
    return 0;
}
