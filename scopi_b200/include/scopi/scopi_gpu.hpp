// scopi_gpu.hpp -- header-only C++ mirror of the SCoPI API (hpc-maths/scopi v0.1.0) whose
// time step runs on a B200 through the C ABI of libscopi_gpu.so (include/scopi_gpu.h).
//
// Same names, argument meaning and defaults as the reference for the hot path:
//   scopi_container<dim>::push_back           include/scopi/container.hpp:339-384
//   property<dim> builder                     include/scopi/property.hpp:16-200
//   sphere / plane / segment                  include/scopi/objects/types/{sphere,plane,segment}.hpp
//   quaternion(), mult_quaternion, normalize  src/quaternion.cpp:6-120
//   NoFriction / Friction / Viscous           include/scopi/contact/property.hpp:14-36
//   contact_property<...>                     include/scopi/contact/property.hpp:41-128
//   ContactsParams<contact_kdtree/brute>      include/scopi/contact/contact_kdtree.hpp:27-61,
//                                             include/scopi/contact/contact_brute_force.hpp:25-50
//   contact_kdtree / contact_brute_force      include/scopi/contact/base.hpp:20-90 (run)
//   neighbor<dim, problem_t>                  include/scopi/contact/neighbor.hpp:24-55
//   AMatrix / ATMatrix                        include/scopi/matrix/velocities.hpp:53-254
//   apgd_params / OptimGradient<apgd>         include/scopi/solvers/apgd.hpp:105-124,
//                                             include/scopi/solvers/OptimGradient.hpp:56-349
//   vap_fixed / vap_fpd                       include/scopi/vap/vap_fixed.hpp, vap_fpd.hpp
//   ScopiSolver<dim, problem, optim, contact, vap>::run / get_params / current_contacts
//                                             include/scopi/solver.hpp:91-327
//   Params<solver> (optim_params, default_contact_property, contact_method_params,
//                   vap_params, solver_params) include/scopi/params.hpp:144-197
//
// The policy types are the GPU ones (namespace scopi::gpu); the reference's policy names
// are aliases of them, so a reference demo compiles against these headers unchanged and a
// demo written for the reference only swaps its policy types to scopi::gpu::... .
// Precision of the APGD iterations is a policy: gpu::apgd<gpu::fp64> (the reference's
// arithmetic) or gpu::apgd<gpu::mixed> (FP32 iterations + FP64 outer correction).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <memory>
#include <utility>
#include <initializer_list>
#include <iostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../../include/scopi_gpu.h"

namespace scopi {

namespace type {
template <std::size_t dim>
using position_t = std::array<double, dim>;
using quaternion_t = std::array<double, 4>;
}  // namespace type

// ------------------------------------------------------------------ quaternions
inline void normalize(type::quaternion_t& q) {
    const double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (auto& c : q) c /= n;
}
inline type::quaternion_t quaternion(double angle, const std::array<double, 3>& axes) {
    type::quaternion_t out = {std::cos(angle / 2), std::sin(angle / 2) * axes[0], std::sin(angle / 2) * axes[1],
                              std::sin(angle / 2) * axes[2]};
    normalize(out);
    return out;
}
inline type::quaternion_t quaternion(double angle, const std::array<double, 2>& axes) {
    return quaternion(angle, std::array<double, 3>{axes[0], axes[1], 1.0});
}
inline type::quaternion_t quaternion(double angle = 0.0) { return quaternion(angle, std::array<double, 3>{0., 0., 1.}); }
inline type::quaternion_t mult_quaternion(const type::quaternion_t& a, const type::quaternion_t& b) {
    type::quaternion_t r;
    r[0] = a[0] * b[0];
    for (std::size_t d = 0; d < 3; ++d) {
        r[0] -= a[d + 1] * b[d + 1];
        r[d + 1] = a[0] * b[d + 1] + b[0] * a[d + 1];
    }
    r[1] += (a[2] * b[3] - a[3] * b[2]);
    r[2] += (a[3] * b[1] - a[1] * b[3]);
    r[3] += (a[1] * b[2] - a[2] * b[1]);
    return r;
}

// ------------------------------------------------------------------ contact models
class NoFriction {};
class Friction {};
class Viscous {};
class FrictionFixedPoint {};  // property.hpp:26
class ViscousFriction {};     // property.hpp:34

template <class problem_t>
struct contact_property;
template <>
struct contact_property<NoFriction> {};
template <>
struct contact_property<Friction> {
    double mu = 0.1;
};
template <>
struct contact_property<Viscous> {
    double gamma = 0;
    double gamma_min = -2.;
    double gamma_tol = 1e-6;
};
template <>
struct contact_property<FrictionFixedPoint> : contact_property<Friction> {  // property.hpp:84-96,131-147
    double fixed_point_tol = 1e-6;
    double fixed_point_max_iter = 1000;
};
template <>
struct contact_property<ViscousFriction> : contact_property<Viscous>,  // property.hpp:149-172
                                           contact_property<Friction> {
    double fixed_point_tol = 1e-6;
    double fixed_point_max_iter = 1000;
};

template <class problem_t>
constexpr int32_t problem_code() {
    if constexpr (std::is_same_v<problem_t, Friction>) return SCOPI_GPU_FRICTION;
    if constexpr (std::is_same_v<problem_t, Viscous>) return SCOPI_GPU_VISCOUS;
    if constexpr (std::is_same_v<problem_t, FrictionFixedPoint>) return SCOPI_GPU_FRICTION_FIXED_POINT;
    if constexpr (std::is_same_v<problem_t, ViscousFriction>) return SCOPI_GPU_VISCOUS_FRICTION;
    return SCOPI_GPU_NOFRICTION;
}

// ------------------------------------------------------------------ objects
template <std::size_t dim>
struct object_base {
    type::position_t<dim> position{};
    type::quaternion_t q = quaternion(0.0);
    int32_t shape = SCOPI_GPU_SPHERE;
    double radius_ = 0.0;
    double length_ = 0.0;
    std::array<double, 3> axes_{0.0, 0.0, 0.0};  // superellipsoid semi-axes
    std::array<double, 2> sq_{1.0, 1.0};         // superellipsoid squareness (e, n)
};

template <std::size_t dim, bool owner = true>
class sphere : public object_base<dim> {
  public:
    sphere(std::initializer_list<type::position_t<dim>> pos, double radius) {
        this->position = *pos.begin();
        this->radius_ = radius;
        this->shape = SCOPI_GPU_SPHERE;
    }
    sphere(std::initializer_list<type::position_t<dim>> pos, type::quaternion_t q, double radius)
        : sphere(pos, radius) {
        this->q = q;
    }
    double radius() const { return this->radius_; }
};

template <std::size_t dim, bool owner = true>
class plane : public object_base<dim> {
  public:
    plane(std::initializer_list<type::position_t<dim>> pos, double angle = 0) {
        this->position = *pos.begin();
        this->q = quaternion(angle);
        this->shape = SCOPI_GPU_PLANE;
    }
    plane(std::initializer_list<type::position_t<dim>> pos, std::initializer_list<type::quaternion_t> q) {
        this->position = *pos.begin();
        this->q = *q.begin();
        this->shape = SCOPI_GPU_PLANE;
    }
};

template <std::size_t dim, bool owner = true>
class segment : public object_base<dim> {
    static_assert(dim == 2, "segments are 2D objects");

  public:
    segment(const type::position_t<dim>& p1, const type::position_t<dim>& p2) {
        for (std::size_t d = 0; d < dim; ++d) this->position[d] = 0.5 * (p1[d] + p2[d]);
        this->q = quaternion(std::atan2(p1[0] - p2[0], p2[1] - p1[1]));
        const double dx = p2[0] - p1[0], dy = p2[1] - p1[1];
        this->length_ = std::sqrt(dx * dx + dy * dy);
        this->shape = SCOPI_GPU_SEGMENT;
    }
};

// superellipsoid<dim>(pos, q, radius, squareness), superellipsoid.hpp:59-70
template <std::size_t dim, bool owner = true>
class superellipsoid : public object_base<dim> {
  public:
    using radius_type = std::array<double, dim>;          // (rx, ry) / (rx, ry, rz)
    using squareness_type = std::array<double, dim - 1>;  // e / (e, n)
    superellipsoid(std::initializer_list<type::position_t<dim>> pos, std::initializer_list<type::quaternion_t> q,
                   std::initializer_list<radius_type> radius, std::initializer_list<squareness_type> sq) {
        set(*pos.begin(), *q.begin(), *radius.begin(), *sq.begin());
    }
    // the reference's 2D demos and tests pass the squareness e as a number
    superellipsoid(std::initializer_list<type::position_t<dim>> pos, std::initializer_list<type::quaternion_t> q,
                   std::initializer_list<radius_type> radius, double e) {
        squareness_type sq{};
        sq.fill(e);
        set(*pos.begin(), *q.begin(), *radius.begin(), sq);
    }
    superellipsoid(std::initializer_list<type::position_t<dim>> pos, std::initializer_list<radius_type> radius,
                   std::initializer_list<squareness_type> sq)
        : superellipsoid(pos, {quaternion(0.0)}, radius, sq) {}
    std::array<double, dim> radius() const {
        std::array<double, dim> r;
        for (std::size_t d = 0; d < dim; ++d) r[d] = this->axes_[d];
        return r;
    }
    std::array<double, dim - 1> squareness() const {
        std::array<double, dim - 1> e;
        for (std::size_t d = 0; d + 1 < dim; ++d) e[d] = this->sq_[d];
        return e;
    }

  private:
    void set(const type::position_t<dim>& pos, const type::quaternion_t& q, const radius_type& r,
             const squareness_type& sq) {
        this->position = pos;
        this->q = q;
        double b = 0.0;
        for (std::size_t d = 0; d < dim; ++d) {
            this->axes_[d] = r[d];
            b += r[d] * r[d];
        }
        for (std::size_t d = 0; d + 1 < dim; ++d) this->sq_[d] = sq[d];
        this->radius_ = std::sqrt(b);  // bounding radius
        this->shape = SCOPI_GPU_SUPERELLIPSOID;
    }
};

// worm<dim>(pos, q, radius, size), objects/types/worm.hpp:118-131: a chain of `size` spheres
// of one radius; each sphere is a body of its own and the solver keeps consecutive spheres
// in contact (add_contact.hpp:11-28)
// read-only view of n contiguous doubles with the reference's element access ((d) and [d])
template <std::size_t n>
class const_view {
  public:
    explicit const_view(const double* p) : m_p(p) {}
    double operator()(std::size_t d) const { return m_p[d]; }
    double operator[](std::size_t d) const { return m_p[d]; }
    operator std::array<double, n>() const {
        std::array<double, n> o;
        for (std::size_t d = 0; d < n; ++d) o[d] = m_p[d];
        return o;
    }

  private:
    const double* m_p;
};

template <std::size_t dim, bool owner = true>
class worm {
  public:
    worm(std::vector<type::position_t<dim>> pos, std::vector<type::quaternion_t> q, double radius, std::size_t size)
        : m_pos(std::move(pos)), m_q(std::move(q)), m_radius(radius), m_size(size) {
        if (m_pos.size() != m_size || m_q.size() != m_size)
            throw std::runtime_error("worm: one position and one quaternion per sphere");
    }
    worm(std::vector<type::position_t<dim>> pos, double radius, std::size_t size)
        : worm(pos, std::vector<type::quaternion_t>(pos.size(), quaternion(0.0)), radius, size) {}
    const_view<dim> pos(std::size_t i) const { return const_view<dim>(m_pos[i].data()); }
    const_view<4> q(std::size_t i) const { return const_view<4>(m_q[i].data()); }
    double radius() const { return m_radius; }
    std::size_t size() const { return m_size; }

  private:
    std::vector<type::position_t<dim>> m_pos;
    std::vector<type::quaternion_t> m_q;
    double m_radius;
    std::size_t m_size;
};

// ------------------------------------------------------------------ box
// BoxDomain<dim> (box.hpp): corners and periodic axes; ScopiSolver(box, particles) runs the
// contact search with the copies across the periodic bounds and wraps the bodies after the move
template <std::size_t dim>
class BoxDomain {
  public:
    BoxDomain() {
        m_min.fill(0.0);
        m_max.fill(0.0);
        m_periodic.fill(false);
    }
    BoxDomain(const std::array<double, dim>& min_corner, const std::array<double, dim>& max_corner)
        : m_min(min_corner), m_max(max_corner) {
        m_periodic.fill(false);
    }
    BoxDomain& with_periodicity() {
        m_periodic.fill(true);
        return *this;
    }
    BoxDomain& with_periodicity(std::size_t axis) {
        m_periodic[axis] = true;
        return *this;
    }
    BoxDomain& with_periodicity(const std::initializer_list<std::size_t>& axis) {
        for (auto a : axis) m_periodic[a] = true;
        return *this;
    }
    const std::array<bool, dim>& is_periodic() const { return m_periodic; }
    bool is_periodic(std::size_t axis) const { return m_periodic[axis]; }
    const std::array<double, dim>& min_corner() const { return m_min; }
    const std::array<double, dim>& max_corner() const { return m_max; }
    double lower_bound(std::size_t axis) const { return m_min[axis]; }
    double upper_bound(std::size_t axis) const { return m_max[axis]; }

  private:
    std::array<double, dim> m_min, m_max;
    std::array<bool, dim> m_periodic;
};

// ------------------------------------------------------------------ property
template <std::size_t dim>
class property {
  public:
    using vec = type::position_t<dim>;
    using rot = std::conditional_t<dim == 2, double, std::array<double, 3>>;
    property& velocity(const vec& v) { m_v = v; return *this; }
    property& velocity(std::initializer_list<vec> v) { m_v = *v.begin(); return *this; }
    property& desired_velocity(const vec& v) { m_dv = v; return *this; }
    property& desired_velocity(std::initializer_list<vec> v) { m_dv = *v.begin(); return *this; }
    property& omega(const rot& w) { m_w = w; return *this; }
    property& desired_omega(const rot& w) { m_dw = w; return *this; }
    property& force(const vec& f) { m_f = f; return *this; }
    property& force(std::initializer_list<vec> f) { m_f = *f.begin(); return *this; }
    property& mass(double m) { m_m = m; return *this; }
    property& moment_inertia(const rot& j) { m_j = j; return *this; }
    property& activate() { m_active = true; return *this; }
    property& deactivate() { m_active = false; return *this; }
    const vec& velocity() const { return m_v; }
    const vec& desired_velocity() const { return m_dv; }
    const rot& omega() const { return m_w; }
    const rot& desired_omega() const { return m_dw; }
    const vec& force() const { return m_f; }
    double mass() const { return m_m; }
    const rot& moment_inertia() const { return m_j; }
    bool is_active() const { return m_active; }

  private:
    vec m_v{}, m_dv{}, m_f{};
    rot m_w{}, m_dw{}, m_j{};
    double m_m = 1.0;
    bool m_active = true;
};

// ------------------------------------------------------------------ snapshot documents
// A small document tree for the snapshot files of ScopiSolver::write_output_files
// (solver.hpp:368-438): objects keep their keys sorted (the order the reference's JSON
// library writes), written as indented JSON or as BSON.
namespace io {
struct Value {
    enum Kind { Null, Bool, Int, Double, String, Array, Object } kind = Null;
    bool b = false;
    int64_t i = 0;
    double d = 0.0;
    std::string s;
    std::vector<Value> items;                             // Array
    std::vector<std::pair<std::string, Value>> fields;    // Object, sorted by key

    static Value boolean(bool v) { Value x; x.kind = Bool; x.b = v; return x; }
    static Value integer(int64_t v) { Value x; x.kind = Int; x.i = v; return x; }
    static Value number(double v) { Value x; x.kind = Double; x.d = v; return x; }
    static Value string(std::string v) { Value x; x.kind = String; x.s = std::move(v); return x; }
    static Value array() { Value x; x.kind = Array; return x; }
    static Value object() { Value x; x.kind = Object; return x; }
    static Value numbers(const double* v, std::size_t n) {
        Value x = array();
        for (std::size_t k = 0; k < n; ++k) x.items.push_back(number(v[k]));
        return x;
    }
    Value& set(const std::string& key, Value v) {
        auto it = std::lower_bound(fields.begin(), fields.end(), key,
                                   [](const std::pair<std::string, Value>& f, const std::string& k) { return f.first < k; });
        if (it != fields.end() && it->first == key)
            it->second = std::move(v);
        else
            fields.insert(it, {key, std::move(v)});
        return *this;
    }
};

// shortest decimal that reads back to the same double; integral values keep a ".0"
inline std::string format_double(double v) {
    if (!std::isfinite(v)) return "null";
    char buf[40];
    for (int prec = 15; prec <= 17; ++prec) {
        std::snprintf(buf, sizeof(buf), "%.*g", prec, v);
        if (std::strtod(buf, nullptr) == v) break;
    }
    std::string out(buf);
    if (out.find_first_of(".eE") == std::string::npos) out += ".0";
    return out;
}
inline void write_json(std::ostream& o, const Value& v, int indent = 0) {
    const std::string pad(indent + 4, ' '), end(indent, ' ');
    switch (v.kind) {
        case Value::Null: o << "null"; break;
        case Value::Bool: o << (v.b ? "true" : "false"); break;
        case Value::Int: o << v.i; break;
        case Value::Double: o << format_double(v.d); break;
        case Value::String: o << '"' << v.s << '"'; break;
        case Value::Array:
            if (v.items.empty()) {
                o << "[]";
                break;
            }
            o << "[\n";
            for (std::size_t k = 0; k < v.items.size(); ++k) {
                o << pad;
                write_json(o, v.items[k], indent + 4);
                o << (k + 1 < v.items.size() ? ",\n" : "\n");
            }
            o << end << ']';
            break;
        case Value::Object:
            if (v.fields.empty()) {
                o << "{}";
                break;
            }
            o << "{\n";
            for (std::size_t k = 0; k < v.fields.size(); ++k) {
                o << pad << '"' << v.fields[k].first << "\": ";
                write_json(o, v.fields[k].second, indent + 4);
                o << (k + 1 < v.fields.size() ? ",\n" : "\n");
            }
            o << end << '}';
            break;
    }
}
// BSON (bsonspec.org): int32/int64 by range, double, UTF-8 string, embedded documents;
// arrays are documents keyed "0", "1", ...
inline void bson_put(std::vector<uint8_t>& b, const void* p, std::size_t n) {
    const uint8_t* c = static_cast<const uint8_t*>(p);
    b.insert(b.end(), c, c + n);  // little-endian hosts (x86-64, aarch64)
}
inline void bson_document(std::vector<uint8_t>& b, const Value& v);
inline void bson_element(std::vector<uint8_t>& b, const std::string& key, const Value& v) {
    uint8_t type = 0x0A;
    switch (v.kind) {
        case Value::Null: type = 0x0A; break;
        case Value::Bool: type = 0x08; break;
        case Value::Int: type = (v.i >= INT32_MIN && v.i <= INT32_MAX) ? 0x10 : 0x12; break;
        case Value::Double: type = 0x01; break;
        case Value::String: type = 0x02; break;
        case Value::Array: type = 0x04; break;
        case Value::Object: type = 0x03; break;
    }
    b.push_back(type);
    bson_put(b, key.c_str(), key.size() + 1);
    switch (v.kind) {
        case Value::Null: break;
        case Value::Bool: b.push_back(v.b ? 1 : 0); break;
        case Value::Int:
            if (type == 0x10) {
                const int32_t x = (int32_t)v.i;
                bson_put(b, &x, 4);
            } else {
                bson_put(b, &v.i, 8);
            }
            break;
        case Value::Double: bson_put(b, &v.d, 8); break;
        case Value::String: {
            const int32_t n = (int32_t)v.s.size() + 1;
            bson_put(b, &n, 4);
            bson_put(b, v.s.c_str(), v.s.size() + 1);
            break;
        }
        case Value::Array:
        case Value::Object: bson_document(b, v); break;
    }
}
inline void bson_document(std::vector<uint8_t>& b, const Value& v) {
    const std::size_t start = b.size();
    b.resize(start + 4);
    if (v.kind == Value::Array)
        for (std::size_t k = 0; k < v.items.size(); ++k) bson_element(b, std::to_string(k), v.items[k]);
    else
        for (const auto& f : v.fields) bson_element(b, f.first, f.second);
    b.push_back(0);
    const int32_t n = (int32_t)(b.size() - start);
    std::copy(reinterpret_cast<const uint8_t*>(&n), reinterpret_cast<const uint8_t*>(&n) + 4, b.begin() + start);
}
inline std::vector<uint8_t> to_bson(const Value& v) {
    std::vector<uint8_t> b;
    bson_document(b, v);
    return b;
}

// Reader for snapshot files (the JSON subset they use: objects, arrays, numbers, strings
// with plain escapes, true/false/null).  Integers without '.', 'e' or 'E' become Int.
class JsonReader {
  public:
    explicit JsonReader(const std::string& text) : s_(text) {}
    Value parse() {
        Value v = value();
        ws();
        if (k_ != s_.size()) fail("trailing characters");
        return v;
    }

  private:
    [[noreturn]] void fail(const char* what) const {
        throw std::runtime_error(std::string("snapshot JSON: ") + what + " at offset " + std::to_string(k_));
    }
    void ws() {
        while (k_ < s_.size() && (s_[k_] == ' ' || s_[k_] == '\n' || s_[k_] == '\t' || s_[k_] == '\r')) ++k_;
    }
    bool eat(char c) {
        ws();
        if (k_ < s_.size() && s_[k_] == c) {
            ++k_;
            return true;
        }
        return false;
    }
    void expect(char c) {
        if (!eat(c)) fail("unexpected character");
    }
    std::string str() {
        expect('"');
        std::string out;
        while (k_ < s_.size() && s_[k_] != '"') {
            char c = s_[k_++];
            if (c == '\\') {
                if (k_ >= s_.size()) fail("bad escape");
                const char e = s_[k_++];
                c = e == 'n' ? '\n' : e == 't' ? '\t' : e == 'r' ? '\r' : e == 'b' ? '\b' : e == 'f' ? '\f' : e;
                if (e == 'u') fail("unicode escapes are not used by snapshot files");
            }
            out += c;
        }
        expect('"');
        return out;
    }
    Value value() {
        ws();
        if (k_ >= s_.size()) fail("unexpected end");
        const char c = s_[k_];
        if (c == '{') {
            ++k_;
            Value o = Value::object();
            if (eat('}')) return o;
            do {
                const std::string key = str();
                expect(':');
                o.set(key, value());
            } while (eat(','));
            expect('}');
            return o;
        }
        if (c == '[') {
            ++k_;
            Value a = Value::array();
            if (eat(']')) return a;
            do {
                a.items.push_back(value());
            } while (eat(','));
            expect(']');
            return a;
        }
        if (c == '"') return Value::string(str());
        if (s_.compare(k_, 4, "true") == 0) { k_ += 4; return Value::boolean(true); }
        if (s_.compare(k_, 5, "false") == 0) { k_ += 5; return Value::boolean(false); }
        if (s_.compare(k_, 4, "null") == 0) { k_ += 4; return Value(); }
        const std::size_t start = k_;
        while (k_ < s_.size() && std::string("+-0123456789.eE").find(s_[k_]) != std::string::npos) ++k_;
        if (k_ == start) fail("unexpected character");
        const std::string num = s_.substr(start, k_ - start);
        if (num.find_first_of(".eE") == std::string::npos) return Value::integer(std::strtoll(num.c_str(), nullptr, 10));
        return Value::number(std::strtod(num.c_str(), nullptr));
    }
    const std::string& s_;
    std::size_t k_ = 0;
};
inline Value read_json_file(const std::filesystem::path& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path.string());
    const std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    return JsonReader(text).parse();
}
inline const Value& field(const Value& o, const std::string& key) {
    for (const auto& f : o.fields)
        if (f.first == key) return f.second;
    throw std::runtime_error("snapshot JSON: missing \"" + key + "\"");
}
inline double as_number(const Value& v) {
    if (v.kind == Value::Double) return v.d;
    if (v.kind == Value::Int) return (double)v.i;
    throw std::runtime_error("snapshot JSON: number expected");
}
template <std::size_t n>
inline std::array<double, n> as_array(const Value& v) {
    if (v.kind != Value::Array || v.items.size() != n) throw std::runtime_error("snapshot JSON: array size");
    std::array<double, n> out{};
    for (std::size_t k = 0; k < n; ++k) out[k] = as_number(v.items[k]);
    return out;
}

// rotation_matrix<dim>(q), quaternion.hpp:66-124 (q = (w, x, y, z)), row-major
template <std::size_t dim>
inline std::array<double, dim * dim> rotation(const type::quaternion_t& q) {
    const double x = q[0], y = q[1], z = q[2], w = q[3];
    if constexpr (dim == 2) {
        return {1 - 2 * w * w, -2 * x * w, 2 * x * w, 1 - 2 * w * w};
    } else {
        return {1 - 2 * z * z - 2 * w * w, 2 * y * z - 2 * x * w,     2 * y * w + 2 * x * z,
                2 * y * z + 2 * x * w,     1 - 2 * y * y - 2 * w * w, 2 * z * w - 2 * x * y,
                2 * y * w - 2 * x * z,     2 * z * w + 2 * x * y,     1 - 2 * y * y - 2 * z * z};
    }
}
}  // namespace io

// ------------------------------------------------------------------ container
template <std::size_t dim>
class vec_ref {
  public:
    explicit vec_ref(double* p) : m_p(p) {}
    double& operator()(std::size_t d) const { return m_p[d]; }
    double& operator[](std::size_t d) const { return m_p[d]; }
    vec_ref& operator=(const type::position_t<dim>& v) {
        for (std::size_t d = 0; d < dim; ++d) m_p[d] = v[d];
        return *this;
    }
    vec_ref& operator=(std::initializer_list<double> v) {
        std::size_t d = 0;
        for (double x : v) m_p[d++] = x;
        return *this;
    }
    operator type::position_t<dim>() const {
        type::position_t<dim> o;
        for (std::size_t d = 0; d < dim; ++d) o[d] = m_p[d];
        return o;
    }

  private:
    double* m_p;
};

template <std::size_t dim>
class scopi_container {
  public:
    static constexpr std::size_t dim_ = dim;
    using rot_ref = std::conditional_t<dim == 2, double&, vec_ref<3>>;

    template <class Obj>
    void push_back(const Obj& s, const property<dim>& p = property<dim>()) {
        push_body(s, p, -1);
        m_objects.push_back({size() - 1, 1, false});
    }
    // a worm's spheres, one body each with the worm's property (container.hpp:338-384)
    void push_back(const worm<dim>& w, const property<dim>& p = property<dim>()) {
        if (!p.is_active()) throw std::runtime_error("worms are active objects");
        const std::size_t first = size();
        for (std::size_t i = 0; i < w.size(); ++i) {
            sphere<dim> s({w.pos(i)}, w.q(i), w.radius());
            push_body(s, p, (int32_t)m_n_worms);
        }
        ++m_n_worms;
        m_objects.push_back({first, w.size(), true});
    }

    // bodies (the reference's size() counts objects: the two differ only with worms)
    std::size_t size() const { return m_shape.size(); }
    std::size_t nb_objects() const { return m_objects.size(); }

    // object io as the reference's operator[] gives it (container.hpp:325-336): pos(i) and
    // q(i) of its i-th body
    class object_view {
      public:
        object_view(double* pos, double* q, std::size_t count) : m_pos(pos), m_q(q), m_count(count) {}
        vec_ref<dim> pos(std::size_t i) const { return vec_ref<dim>(m_pos + 3 * i); }
        vec_ref<4> q(std::size_t i) const { return vec_ref<4>(m_q + 4 * i); }
        std::size_t size() const { return m_count; }

      private:
        double *m_pos, *m_q;
        std::size_t m_count;
    };
    std::unique_ptr<object_view> operator[](std::size_t io) {
        const auto& ob = m_objects.at(io);
        return std::make_unique<object_view>(&m_pos[3 * ob.first], &m_q[4 * ob.first], ob.count);
    }

  private:
    template <class Obj>
    void push_body(const Obj& s, const property<dim>& p, int32_t worm_index) {
        if (!p.is_active()) {
            if (m_nb_inactive != size())
                throw std::runtime_error("All the obstacles must be pushed before the active particles.");
            ++m_nb_inactive;
        }
        m_worm.push_back(worm_index);
        m_shape.push_back(s.shape);
        append3(m_pos, s.position);
        for (double c : s.q) m_q.push_back(c);
        append3(m_v, p.velocity());
        append3(m_vd, p.desired_velocity());
        append3(m_f, p.force());
        appendrot(m_w, p.omega());
        appendrot(m_dw, p.desired_omega());
        appendrot(m_j, p.moment_inertia());
        m_m.push_back(p.mass());
        m_radius.push_back(s.radius_);
        m_length.push_back(s.length_);
        for (double c : s.axes_) m_axes.push_back(c);
        for (double c : s.sq_) m_sq.push_back(c);
    }

  public:
    std::size_t nb_inactive() const { return m_nb_inactive; }
    std::size_t nb_active() const { return size() - m_nb_inactive; }

    struct vec_field {
        std::vector<double>* v;
        vec_ref<dim> operator()(std::size_t i) const { return vec_ref<dim>(v->data() + 3 * i); }
        vec_ref<dim> operator[](std::size_t i) const { return (*this)(i); }
    };
    struct rot_field {
        std::vector<double>* v;
        rot_ref operator()(std::size_t i) const {
            if constexpr (dim == 2)
                return (*v)[3 * i + 2];
            else
                return vec_ref<3>(v->data() + 3 * i);
        }
        rot_ref operator[](std::size_t i) const { return (*this)(i); }
    };
    struct quat_field {
        std::vector<double>* v;
        vec_ref<4> operator()(std::size_t i) const { return vec_ref<4>(v->data() + 4 * i); }
        vec_ref<4> operator[](std::size_t i) const { return (*this)(i); }
    };
    vec_field pos() { return {&m_pos}; }
    vec_field v() { return {&m_v}; }
    vec_field vd() { return {&m_vd}; }
    vec_field f() { return {&m_f}; }
    rot_field omega() { return {&m_w}; }
    rot_field desired_omega() { return {&m_dw}; }
    rot_field j() { return {&m_j}; }
    quat_field q() { return {&m_q}; }
    std::vector<double>& m() { return m_m; }

    // C ABI view (host arrays owned by the container)
    scopi_gpu_particles abi() {
        scopi_gpu_particles p{};
        p.n = (int64_t)size();
        p.nb_inactive = (int64_t)m_nb_inactive;
        p.shape = m_shape.data();
        p.pos = m_pos.data();
        p.q = m_q.data();
        p.v = m_v.data();
        p.omega = m_w.data();
        p.vd = m_vd.data();
        p.omega_d = m_dw.data();
        p.f = m_f.data();
        p.m = m_m.data();
        p.j = m_j.data();
        p.radius = m_radius.data();
        p.length = m_length.data();
        p.axes = m_axes.data();
        p.squareness = m_sq.data();
        p.worm = m_n_worms > 0 ? m_worm.data() : nullptr;
        return p;
    }

    // The "objects" array of a snapshot: write_objects.hpp (per shape) and the properties
    // written by write_output_files (solver.hpp:383-400).
    io::Value snapshot_objects() const {
        using io::Value;
        Value out = Value::array();
        for (const auto& ob : m_objects) {
            const std::size_t i = ob.first;
            const double* x = &m_pos[3 * i];
            type::quaternion_t q = {m_q[4 * i], m_q[4 * i + 1], m_q[4 * i + 2], m_q[4 * i + 3]};
            const auto R = io::rotation<dim>(q);
            Value o = Value::object();
            double col0[dim];
            for (std::size_t d = 0; d < dim; ++d) col0[d] = R[d * dim];
            if (ob.worm) {
                // write_objects(worm), write_objects.hpp:183-198: one entry per sphere
                o.set("type", Value::string("worm"));
                Value spheres = Value::array();
                for (std::size_t k = 0; k < ob.count; ++k) {
                    const std::size_t b = i + k;
                    Value e = Value::object();
                    e.set("id", Value::integer((int64_t)b));
                    e.set("position", Value::numbers(&m_pos[3 * b], dim));
                    e.set("quaternion", Value::numbers(&m_q[4 * b], 4));
                    e.set("radius", Value::number(m_radius[b]));
                    spheres.items.push_back(std::move(e));
                }
                o.set("worm", std::move(spheres));
            } else {
            o.set("id", Value::integer((int64_t)i));
            o.set("quaternion", Value::numbers(q.data(), 4));
            switch (m_shape[i]) {
                case SCOPI_GPU_PLANE:
                    o.set("type", Value::string("plane"));
                    o.set("position", Value::numbers(x, dim));
                    o.set("normal", Value::numbers(col0, dim));
                    o.set("rotation", Value::numbers(R.data(), dim * dim));
                    break;
                case SCOPI_GPU_SEGMENT: {
                    o.set("type", Value::string("segment"));
                    const double t[2] = {-col0[1], col0[0]};
                    const double h = 0.5 * m_length[i];
                    // extrema: R (0, -+L/2) + centre (segment.hpp:168-177)
                    const double p1[2] = {R[1] * -h + x[0], R[3] * -h + x[1]};
                    const double p2[2] = {R[1] * h + x[0], R[3] * h + x[1]};
                    o.set("p1", Value::numbers(p1, 2));
                    o.set("p2", Value::numbers(p2, 2));
                    o.set("normal", Value::numbers(col0, 2));
                    o.set("tangent", Value::numbers(t, 2));
                    break;
                }
                case SCOPI_GPU_SUPERELLIPSOID:
                    o.set("type", Value::string("superellipsoid"));
                    o.set("position", Value::numbers(x, dim));
                    o.set("radius", Value::numbers(&m_axes[3 * i], dim));
                    o.set("squareness", Value::numbers(&m_sq[2 * i], dim - 1));
                    o.set("rotation", Value::numbers(R.data(), dim * dim));
                    break;
                default:
                    o.set("type", Value::string("sphere"));
                    o.set("position", Value::numbers(x, dim));
                    o.set("radius", Value::number(m_radius[i]));
                    o.set("rotation", Value::numbers(R.data(), dim * dim));
                    break;
            }
            }
            auto rot = [&](const std::vector<double>& a) {
                return dim == 2 ? Value::number(a[3 * i + 2]) : Value::numbers(&a[3 * i], 3);
            };
            Value pr = Value::object();
            pr.set("velocity", Value::numbers(&m_v[3 * i], dim));
            pr.set("desired_velocity", Value::numbers(&m_vd[3 * i], dim));
            pr.set("omega", rot(m_w));
            pr.set("desired_omega", rot(m_dw));
            pr.set("force", Value::numbers(&m_f[3 * i], dim));
            pr.set("mass", Value::number(m_m[i]));
            pr.set("moment_inertia", rot(m_j));
            pr.set("active", Value::boolean(i >= m_nb_inactive));
            o.set("properties", std::move(pr));
            out.items.push_back(std::move(o));
        }
        return out;
    }

  private:
    template <class V>
    static void append3(std::vector<double>& dst, const V& v) {
        for (std::size_t d = 0; d < 3; ++d) dst.push_back(d < dim ? v[d] : 0.0);
    }
    template <class R>
    static void appendrot(std::vector<double>& dst, const R& r) {
        if constexpr (dim == 2) {
            dst.push_back(0.0);
            dst.push_back(0.0);
            dst.push_back(r);
        } else {
            for (std::size_t d = 0; d < 3; ++d) dst.push_back(r[d]);
        }
    }
    struct object_range {
        std::size_t first, count;
        bool worm;
    };
    std::vector<int32_t> m_shape, m_worm;
    std::vector<double> m_pos, m_q, m_v, m_w, m_vd, m_dw, m_f, m_m, m_j, m_radius, m_length, m_axes, m_sq;
    std::vector<object_range> m_objects;  // the objects as pushed: first body, bodies, worm or not
    std::size_t m_nb_inactive = 0, m_n_worms = 0;
};

// ------------------------------------------------------------------ restart
// from_json<dim> (restart.hpp:20-67, properties as json.hpp:26-44 reads them): a container
// rebuilt from the "objects" of a snapshot document (spheres, superellipsoids, segments,
// planes, worms), obstacles first as the snapshot lists them.
template <std::size_t dim>
scopi_container<dim> from_json(const io::Value& j) {
    using io::as_array;
    using io::as_number;
    using io::field;
    scopi_container<dim> container;
    for (const auto& o : field(j, "objects").items) {
        const auto& pr = field(o, "properties");
        property<dim> p;
        p.velocity(as_array<dim>(field(pr, "velocity")))
            .desired_velocity(as_array<dim>(field(pr, "desired_velocity")))
            .force(as_array<dim>(field(pr, "force")))
            .mass(as_number(field(pr, "mass")));
        if constexpr (dim == 2) {
            p.omega(as_number(field(pr, "omega")))
                .desired_omega(as_number(field(pr, "desired_omega")))
                .moment_inertia(as_number(field(pr, "moment_inertia")));
        } else {
            p.omega(as_array<3>(field(pr, "omega")))
                .desired_omega(as_array<3>(field(pr, "desired_omega")))
                .moment_inertia(as_array<3>(field(pr, "moment_inertia")));
        }
        if (field(pr, "active").b)
            p.activate();
        else
            p.deactivate();
        const std::string type = field(o, "type").s;
        if (type == "sphere") {
            container.push_back(sphere<dim>({as_array<dim>(field(o, "position"))}, as_array<4>(field(o, "quaternion")),
                                            as_number(field(o, "radius"))),
                                p);
        } else if (type == "superellipsoid") {
            container.push_back(superellipsoid<dim>({as_array<dim>(field(o, "position"))},
                                                    {as_array<4>(field(o, "quaternion"))},
                                                    {as_array<dim>(field(o, "radius"))},
                                                    {as_array<dim - 1>(field(o, "squareness"))}),
                                p);
        } else if (type == "segment") {
            if constexpr (dim == 2)
                container.push_back(segment<dim>(as_array<2>(field(o, "p1")), as_array<2>(field(o, "p2"))), p);
        } else if (type == "plane") {
            container.push_back(
                plane<dim>({as_array<dim>(field(o, "position"))}, {as_array<4>(field(o, "quaternion"))}), p);
        } else if (type == "worm") {  // restart.hpp:53-64
            std::vector<type::position_t<dim>> pos;
            std::vector<type::quaternion_t> q;
            const auto& spheres = field(o, "worm").items;
            for (const auto& e : spheres) {
                pos.push_back(as_array<dim>(field(e, "position")));
                q.push_back(as_array<4>(field(e, "quaternion")));
            }
            if (spheres.empty()) throw std::runtime_error("from_json: empty worm");
            container.push_back(worm<dim>(pos, q, as_number(field(spheres[0], "radius")), pos.size()), p);
        } else {
            throw std::runtime_error("from_json: object type \"" + type + "\" is not supported");
        }
    }
    return container;
}
template <std::size_t dim>
scopi_container<dim> from_json(const std::filesystem::path& path) {
    return from_json<dim>(io::read_json_file(path));
}

// ------------------------------------------------------------------ contacts record
namespace type {
// a contact vector read as v[k] or v(k), as the reference's fixed-size tensors allow
template <std::size_t dim>
struct contact_vec : std::array<double, dim> {
    double& operator()(std::size_t k) { return (*this)[k]; }
    double operator()(std::size_t k) const { return (*this)[k]; }
};
}  // namespace type

// neighbor<dim, problem_t> (contact/neighbor.hpp:24-55)
template <std::size_t dim, class problem_t>
struct neighbor {
    std::size_t i, j;
    double dij;
    type::contact_vec<dim> nij, pi, pj;
    contact_property<problem_t> property;
};

// ------------------------------------------------------------------ contact methods
template <class D>
struct ContactsParams;
template <class problem_t>
class contact_kdtree;
template <class problem_t>
class contact_brute_force;

template <class problem_t>
struct ContactsParams<contact_kdtree<problem_t>> {  // contact_kdtree.hpp:27-61
    void init_options() {}
    double dmax{2.};
    double kd_tree_radius{17.};
};
template <class problem_t>
struct ContactsParams<contact_brute_force<problem_t>> {  // contact_brute_force.hpp:25-50
    void init_options() {}
    double dmax{2.};
};

namespace detail {
// contact_base::run (contact/base.hpp:71-84) through the C ABI: a handle with the method's
// parameters detects the container's contacts (periodic copies of `box` included) and
// returns them sorted by (i, j)
template <std::size_t dim, class problem_t>
std::vector<neighbor<dim, problem_t>> detect_contacts(int32_t method, double dmax, double kd_radius,
                                                      const BoxDomain<dim>& box, scopi_container<dim>& particles);
}  // namespace detail

// contact_kdtree<problem_t> / contact_brute_force<problem_t> (contact_kdtree.hpp:70-268,
// contact_brute_force.hpp:59-136): callable as in the reference,
//     ContactsParams<contact_kdtree<NoFriction>> params; contact_kdtree cont(params);
//     auto contacts = cont.run(particles);
// the search is the GPU cell list of this library (same contact set as the kd-tree and the
// brute force: every pair with dij < dmax, kd-tree candidates within the kd radius).
template <class problem_t>
class contact_kdtree {
  public:
    static constexpr int32_t code = SCOPI_GPU_KDTREE;
    using params_t = ContactsParams<contact_kdtree<problem_t>>;
    contact_kdtree() = default;
    explicit contact_kdtree(const params_t& params) : m_params(params) {}
    void init_options() { m_params.init_options(); }
    params_t& get_params() { return m_params; }
    contact_property<problem_t>& default_contact_property() { return m_property; }
    template <std::size_t dim>
    std::vector<neighbor<dim, problem_t>> run(const BoxDomain<dim>& box, scopi_container<dim>& particles) {
        return detail::detect_contacts<dim, problem_t>(code, m_params.dmax, m_params.kd_tree_radius, box, particles);
    }
    template <std::size_t dim>
    std::vector<neighbor<dim, problem_t>> run(scopi_container<dim>& particles) {
        return run(BoxDomain<dim>(), particles);
    }

  private:
    params_t m_params;
    contact_property<problem_t> m_property;
};

template <class problem_t>
class contact_brute_force {
  public:
    static constexpr int32_t code = SCOPI_GPU_BRUTE_FORCE;
    using params_t = ContactsParams<contact_brute_force<problem_t>>;
    contact_brute_force() = default;
    explicit contact_brute_force(const params_t& params) : m_params(params) {}
    void init_options() { m_params.init_options(); }
    params_t& get_params() { return m_params; }
    contact_property<problem_t>& default_contact_property() { return m_property; }
    template <std::size_t dim>
    std::vector<neighbor<dim, problem_t>> run(const BoxDomain<dim>& box, scopi_container<dim>& particles) {
        return detail::detect_contacts<dim, problem_t>(code, m_params.dmax, 0.0, box, particles);
    }
    template <std::size_t dim>
    std::vector<neighbor<dim, problem_t>> run(scopi_container<dim>& particles) {
        return run(BoxDomain<dim>(), particles);
    }

  private:
    params_t m_params;
    contact_property<problem_t> m_property;
};

namespace detail {
inline void check_abi(int32_t rc, scopi_gpu_handle* h, const char* what);

// a handle holding the container (and, for the matrices, a given contact list)
template <std::size_t dim>
scopi_gpu_handle* open_handle(int32_t problem, int32_t method, double dmax, double kd_radius,
                              const BoxDomain<dim>& box, scopi_container<dim>& particles) {
    scopi_gpu_params p;
    scopi_gpu_default_params(&p, (int32_t)dim);
    p.problem = problem;
    p.contact_method = method;
    p.dmax = dmax;
    if (method == SCOPI_GPU_KDTREE) p.kd_tree_radius = kd_radius;
    for (std::size_t d = 0; d < dim; ++d) {
        p.box_lower[d] = box.lower_bound(d);
        p.box_upper[d] = box.upper_bound(d);
        p.periodic[d] = box.is_periodic(d) ? 1 : 0;
    }
    scopi_gpu_handle* h = nullptr;
    check_abi(scopi_gpu_create(&p, &h), nullptr, "create");
    scopi_gpu_particles abi = particles.abi();
    const int32_t rc = scopi_gpu_set_particles(h, &abi);
    if (rc < 0) {
        const std::string msg = scopi_gpu_last_error(h);
        scopi_gpu_destroy(h);
        throw std::runtime_error("scopi_gpu_set_particles: " + msg);
    }
    return h;
}

struct handle_guard {
    scopi_gpu_handle* h;
    ~handle_guard() {
        if (h) scopi_gpu_destroy(h);
    }
};
}  // namespace detail

// ------------------------------------------------------------------ GPU policies
namespace gpu {
struct fp64 {
    static constexpr int32_t code = SCOPI_GPU_FP64;
};
struct mixed {
    static constexpr int32_t code = SCOPI_GPU_MIXED;
};

struct apgd_params {  // apgd.hpp:105-124 (+ the mixed form's correction target)
    double alpha = 0.05;
    std::size_t max_ite = 10000;
    double tolerance = 1e-7;
    bool dynamic_descent = true;
    double mixed_violation_tol = 1e-6;
    int mixed_max_corrections = 3;
    int initial_step = SCOPI_GPU_STEP_AUTO;  // first step: reference alpha or curvature estimate
};

template <class precision = fp64>
struct apgd {
    using params_t = apgd_params;
    using precision_t = precision;
};

template <class Method>
struct OptimGradient {
    using method_t = Method;
    using params_t = typename Method::params_t;
    params_t m_params;
    params_t& get_params() { return m_params; }
};

// the contact methods above, under the GPU policy names
template <class D>
using ContactsParams = scopi::ContactsParams<D>;
template <class problem_t>
using contact_kdtree = scopi::contact_kdtree<problem_t>;
template <class problem_t>
using contact_brute_force = scopi::contact_brute_force<problem_t>;

struct VapParams {};
struct vap_fixed {
    static constexpr int32_t code = SCOPI_GPU_VAP_FIXED;
    using params_t = VapParams;
};
struct vap_fpd {
    static constexpr int32_t code = SCOPI_GPU_VAP_FPD;
    using params_t = VapParams;
};
}  // namespace gpu

// reference policy names
using apgd_params = gpu::apgd_params;
using apgd = gpu::apgd<gpu::fp64>;
template <class Method>
using OptimGradient = gpu::OptimGradient<Method>;
using vap_fixed = gpu::vap_fixed;
using vap_fpd = gpu::vap_fpd;

struct ScopiParams {  // params.hpp:89-134 (snapshot files: ScopiSolver::write_output_files)
    std::size_t output_frequency = std::size_t(-1);
    std::filesystem::path path = "Results";
    std::string filename = "scopi_objects";
    bool write_velocity = false;
    bool write_lagrange_multiplier = false;
    bool binary_output = false;
};

template <class solver_t>
struct Params {  // params.hpp:144-197
    typename solver_t::optim_solver_t::params_t& optim_params;
    contact_property<typename solver_t::problem_t>& default_contact_property;
    typename solver_t::contact_params_t& contact_method_params;
    typename solver_t::vap_t::params_t& vap_params;
    ScopiParams& solver_params;
};

class gpu_error : public std::runtime_error {
  public:
    using std::runtime_error::runtime_error;
};

// ------------------------------------------------------------------ ScopiSolver
template <std::size_t dim, class problem_type = NoFriction, class optim_solver_type = OptimGradient<apgd>,
          template <class> class contact_method_type = contact_kdtree, class vap_type = vap_fixed>
class ScopiSolver {
  public:
    using problem_t = problem_type;
    using optim_solver_t = optim_solver_type;
    using contact_method_t = contact_method_type<problem_t>;
    using contact_params_t = gpu::ContactsParams<contact_method_t>;
    using vap_t = vap_type;
    using params_t = Params<ScopiSolver>;

    explicit ScopiSolver(scopi_container<dim>& particles) : m_particles(particles) {}
    ScopiSolver(const BoxDomain<dim>& box, scopi_container<dim>& particles) : m_particles(particles), m_box(box) {}
    ~ScopiSolver() {
        if (m_h) scopi_gpu_destroy(m_h);
    }
    ScopiSolver(const ScopiSolver&) = delete;
    ScopiSolver& operator=(const ScopiSolver&) = delete;

    params_t get_params() {
        return params_t{m_optim.get_params(), m_default_property, m_contact_params, m_vap_params, m_params};
    }

    // ScopiSolver::run (solver.hpp:267-303): the container is uploaded, the steps run on
    // the GPU, and positions, quaternions and velocities are copied back.  Snapshot files as
    // the reference writes them: one at the start (index initial_iter, with the contacts of
    // the previous step), then after every step nite with (nite + 1) % output_frequency == 0
    // (index nite + 1); the steps between two snapshots run on the GPU in one call.
    void run(double dt, std::size_t total_it, std::size_t initial_iter = 0) {
        ensure();
        scopi_gpu_particles p = m_particles.abi();
        check(scopi_gpu_set_particles(m_h, &p), "set_particles");
        write_output_files(initial_iter);
        const std::size_t freq = m_params.output_frequency;
        std::size_t nite = initial_iter;
        bool noconv = false;
        while (nite < total_it) {
            std::size_t end = total_it;
            if (freq != std::size_t(-1) && freq > 0) end = std::min(total_it, (nite / freq + 1) * freq);
            const int32_t rc = scopi_gpu_run(m_h, dt, (int64_t)end, (int64_t)nite);
            if (rc < 0) check(rc, "run");
            noconv = noconv || rc == SCOPI_GPU_ENOCONV;
            nite = end;
            if (freq != std::size_t(-1) && freq > 0 && nite % freq == 0) {
                check(scopi_gpu_get_particles(m_h, &p), "get_particles");
                write_output_files(nite);
            }
        }
        if (noconv) std::cerr << "APGD didn't converge." << std::endl;
        check(scopi_gpu_get_particles(m_h, &p), "get_particles");
    }

    // write_output_files (solver.hpp:368-438): {path}/{filename}_{nite:04d}.json (or .bson
    // with binary_output) holding the objects of the container and the contacts of the last
    // step (null when there are none), each with the multiplier of the same index when
    // write_lagrange_multiplier is set (as the reference indexes it).
    void write_output_files(std::size_t nite) {
        using io::Value;
        std::filesystem::create_directories(m_params.path);
        Value doc = Value::object();
        doc.set("objects", m_particles.snapshot_objects());
        const auto& cc = current_contacts();
        std::vector<double> lam;
        if (m_params.write_lagrange_multiplier && !cc.empty()) lam = lagrange_multiplier();
        Value contacts;  // null without contacts
        if (!cc.empty()) {
            contacts = Value::array();
            for (std::size_t k = 0; k < cc.size(); ++k) {
                const auto& c = cc[k];
                Value o = Value::object();
                o.set("i", Value::integer((int64_t)c.i));
                o.set("j", Value::integer((int64_t)c.j));
                o.set("pi", Value::numbers(c.pi.data(), dim));
                o.set("pj", Value::numbers(c.pj.data(), dim));
                o.set("normal", Value::numbers(c.nij.data(), dim));
                o.set("distance", Value::number(c.dij));
                o.set("property", property_json(c));
                if (m_params.write_lagrange_multiplier && k < lam.size())
                    o.set("lagrange multiplier", Value::number(lam[k]));
                contacts.items.push_back(std::move(o));
            }
        }
        doc.set("contacts", std::move(contacts));
        char idx[32];
        std::snprintf(idx, sizeof(idx), "_%04zu", nite);
        const std::string base = (m_params.path / m_params.filename).string() + idx;
        if (m_params.binary_output) {
            const std::vector<uint8_t> b = io::to_bson(doc);
            std::ofstream f(base + ".bson", std::ios::out | std::ios::binary);
            f.write(reinterpret_cast<const char*>(b.data()), (std::streamsize)b.size());
        } else {
            std::ofstream f(base + ".json");
            io::write_json(f, doc);
        }
    }

    // current_contacts (solver.hpp:314-317)
    const std::vector<neighbor<dim, problem_t>>& current_contacts() {
        ensure();
        int64_t n = 0;
        check(scopi_gpu_get_contacts(m_h, 0, &n, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr),
              "get_contacts");
        std::vector<int64_t> ci(n), cj(n);
        std::vector<double> d(n), nij(3 * n), pi(3 * n), pj(3 * n), g(n);
        check(scopi_gpu_get_contacts(m_h, n, &n, ci.data(), cj.data(), d.data(), nij.data(), pi.data(), pj.data(),
                                     g.data()),
              "get_contacts");
        m_contacts.resize(n);
        for (int64_t k = 0; k < n; ++k) {
            auto& c = m_contacts[k];
            c.i = (std::size_t)ci[k];
            c.j = (std::size_t)cj[k];
            c.dij = d[k];
            for (std::size_t x = 0; x < dim; ++x) {
                c.nij[x] = nij[3 * k + x];
                c.pi[x] = pi[3 * k + x];
                c.pj[x] = pj[3 * k + x];
            }
            if constexpr (std::is_same_v<problem_t, Viscous> || std::is_same_v<problem_t, ViscousFriction>)
                c.property.gamma = g[k];
        }
        return m_contacts;
    }

    std::vector<double> lagrange_multiplier() {
        ensure();
        int64_t n = 0;
        check(scopi_gpu_get_lambda(m_h, 0, &n, nullptr), "get_lambda");
        std::vector<double> out(n);
        check(scopi_gpu_get_lambda(m_h, n, &n, out.data()), "get_lambda");
        return out;
    }

    scopi_gpu_stats stats() {
        scopi_gpu_stats s{};
        if (m_h) scopi_gpu_get_stats(m_h, &s);
        return s;
    }

  private:
    // contact_property<problem_t>::to_json (property.hpp): the contact's own gamma for Viscous
    io::Value property_json(const neighbor<dim, problem_t>& c) const {
        using io::Value;
        Value o = Value::object();
        if constexpr (std::is_same_v<problem_t, Friction>) {
            o.set("type", Value::string("friction"));
            o.set("mu", Value::number(m_default_property.mu));
        } else if constexpr (std::is_same_v<problem_t, FrictionFixedPoint>) {
            o.set("type", Value::string("friction fixed point"));
            o.set("mu", Value::number(m_default_property.mu));
            o.set("fixed_point_tol", Value::number(m_default_property.fixed_point_tol));
            o.set("fixed_point_max_iter", Value::number(m_default_property.fixed_point_max_iter));
        } else if constexpr (std::is_same_v<problem_t, Viscous>) {
            o.set("type", Value::string("viscous"));
            o.set("gamma", Value::number(c.property.gamma));
            o.set("gamma_min", Value::number(m_default_property.gamma_min));
            o.set("gamma_tol", Value::number(m_default_property.gamma_tol));
        } else if constexpr (std::is_same_v<problem_t, ViscousFriction>) {
            o.set("type", Value::string("viscous friction"));
            o.set("gamma", Value::number(c.property.gamma));
            o.set("gamma_min", Value::number(m_default_property.gamma_min));
            o.set("gamma_tol", Value::number(m_default_property.gamma_tol));
            o.set("mu", Value::number(m_default_property.mu));
            o.set("fixed_point_tol", Value::number(m_default_property.fixed_point_tol));
            o.set("fixed_point_max_iter", Value::number(m_default_property.fixed_point_max_iter));
        } else {
            (void)c;
            o.set("type", Value::string("no friction"));
        }
        return o;
    }

    void check(int32_t rc, const char* what) {
        if (rc < 0) throw gpu_error(std::string("scopi_gpu_") + what + ": " + scopi_gpu_last_error(m_h));
    }
    void ensure() {
        if (m_h) return;
        scopi_gpu_params p;
        scopi_gpu_default_params(&p, (int32_t)dim);
        p.problem = problem_code<problem_t>();
        p.vap = vap_t::code;
        p.contact_method = contact_method_t::code;
        p.precision = optim_solver_t::method_t::precision_t::code;
        const auto& op = m_optim.get_params();
        p.alpha = op.alpha;
        p.max_ite = (int64_t)op.max_ite;
        p.tolerance = op.tolerance;
        p.dynamic_descent = op.dynamic_descent ? 1 : 0;
        p.mixed_violation_tol = op.mixed_violation_tol;
        p.mixed_max_corrections = op.mixed_max_corrections;
        p.initial_step = op.initial_step;
        p.dmax = m_contact_params.dmax;
        if constexpr (std::is_same_v<contact_method_t, gpu::contact_kdtree<problem_t>>)
            p.kd_tree_radius = m_contact_params.kd_tree_radius;
        if constexpr (std::is_same_v<problem_t, Friction>) p.mu = m_default_property.mu;
        if constexpr (std::is_same_v<problem_t, FrictionFixedPoint>) {
            p.mu = m_default_property.mu;
            p.fixed_point_tol = m_default_property.fixed_point_tol;
            p.fixed_point_max_iter = (int64_t)m_default_property.fixed_point_max_iter;
        }
        if constexpr (std::is_same_v<problem_t, Viscous> || std::is_same_v<problem_t, ViscousFriction>) {
            p.gamma = m_default_property.gamma;
            p.gamma_min = m_default_property.gamma_min;
            p.gamma_tol = m_default_property.gamma_tol;
        }
        if constexpr (std::is_same_v<problem_t, ViscousFriction>) {
            p.mu = m_default_property.mu;
            p.fixed_point_tol = m_default_property.fixed_point_tol;
            p.fixed_point_max_iter = (int64_t)m_default_property.fixed_point_max_iter;
        }
        for (std::size_t d = 0; d < dim; ++d) {
            p.box_lower[d] = m_box.lower_bound(d);
            p.box_upper[d] = m_box.upper_bound(d);
            p.periodic[d] = m_box.is_periodic(d) ? 1 : 0;
        }
        const int32_t rc = scopi_gpu_create(&p, &m_h);
        if (rc < 0) throw gpu_error(std::string("scopi_gpu_create: ") + scopi_gpu_last_error(nullptr));
    }

    scopi_container<dim>& m_particles;
    BoxDomain<dim> m_box;
    optim_solver_t m_optim;
    contact_property<problem_t> m_default_property;
    contact_params_t m_contact_params;
    typename vap_t::params_t m_vap_params;
    ScopiParams m_params;
    std::vector<neighbor<dim, problem_t>> m_contacts;
    scopi_gpu_handle* m_h = nullptr;
};

// ------------------------------------------------------------------ contact methods, matrices
namespace detail {
inline void check_abi(int32_t rc, scopi_gpu_handle* h, const char* what) {
    if (rc < 0) throw gpu_error(std::string("scopi_gpu_") + what + ": " + scopi_gpu_last_error(h));
}

template <std::size_t dim, class problem_t>
std::vector<neighbor<dim, problem_t>> detect_contacts(int32_t method, double dmax, double kd_radius,
                                                      const BoxDomain<dim>& box, scopi_container<dim>& particles) {
    handle_guard g{open_handle<dim>(problem_code<problem_t>(), method, dmax, kd_radius, box, particles)};
    int64_t n = 0;
    check_abi(scopi_gpu_detect(g.h, &n), g.h, "detect");
    std::vector<int64_t> ci(n), cj(n);
    std::vector<double> d(n), nij(3 * n), pi(3 * n), pj(3 * n);
    check_abi(scopi_gpu_get_contacts(g.h, n, &n, ci.data(), cj.data(), d.data(), nij.data(), pi.data(), pj.data(),
                                     nullptr),
              g.h, "get_contacts");
    std::vector<neighbor<dim, problem_t>> out((std::size_t)n);
    for (int64_t k = 0; k < n; ++k) {
        auto& c = out[(std::size_t)k];
        c.i = (std::size_t)ci[k];
        c.j = (std::size_t)cj[k];
        c.dij = d[k];
        for (std::size_t x = 0; x < dim; ++x) {
            c.nij[x] = nij[3 * k + x];
            c.pi[x] = pi[3 * k + x];
            c.pj[x] = pj[3 * k + x];
        }
    }
    return out;
}

// a handle on the container with `contacts` as its contact list
template <class Contacts_t, std::size_t dim>
scopi_gpu_handle* jacobian_handle(const Contacts_t& contacts, const scopi_container<dim>& particles) {
    auto& parts = const_cast<scopi_container<dim>&>(particles);  // read only: uploaded, not written
    scopi_gpu_handle* h = open_handle<dim>(SCOPI_GPU_NOFRICTION, SCOPI_GPU_BRUTE_FORCE, 2.0, 0.0, BoxDomain<dim>(), parts);
    const std::size_t n = contacts.size();
    std::vector<int64_t> ci(n), cj(n);
    std::vector<double> d(n), nij(3 * n, 0.0), pi(3 * n, 0.0), pj(3 * n, 0.0);
    for (std::size_t k = 0; k < n; ++k) {
        const auto& c = contacts[k];
        ci[k] = (int64_t)c.i;
        cj[k] = (int64_t)c.j;
        d[k] = c.dij;
        for (std::size_t x = 0; x < dim; ++x) {
            nij[3 * k + x] = c.nij[x];
            pi[3 * k + x] = c.pi[x];
            pj[3 * k + x] = c.pj[x];
        }
    }
    const int32_t rc = scopi_gpu_set_contacts(h, (int64_t)n, ci.data(), cj.data(), d.data(), nij.data(), pi.data(),
                                              pj.data());
    if (rc < 0) {
        const std::string msg = scopi_gpu_last_error(h);
        scopi_gpu_destroy(h);
        throw gpu_error("scopi_gpu_set_contacts: " + msg);
    }
    return h;
}
}  // namespace detail

// AMatrix (matrix/velocities.hpp:53-144): per contact (v_i - (p_i - x_i) x R_i w_i) -
// (v_j - (p_j - x_j) x R_j w_j) on the active bodies; u holds 6 values per active body
// (velocity, then rotation), the result 3 per contact.  Applied on the GPU.
template <class Contacts_t, class Particles_t>
class AMatrix {
  public:
    static constexpr std::size_t dim = Particles_t::dim_;
    AMatrix(const Contacts_t& contacts, const Particles_t& particles) : m_contacts(contacts), m_particles(particles) {}
    template <class Vec>
    const std::vector<double>& mat_mult(const Vec& u) const {
        if (std::size(u) != 6 * m_particles.nb_active()) throw gpu_error("AMatrix::mat_mult: u must hold 6 values per active body");
        detail::handle_guard g{detail::jacobian_handle(m_contacts, m_particles)};
        m_work.assign(3 * m_contacts.size(), 0.0);
        if (!m_contacts.empty()) detail::check_abi(scopi_gpu_amat(g.h, std::data(u), m_work.data()), g.h, "amat");
        return m_work;
    }

  private:
    const Contacts_t& m_contacts;
    const Particles_t& m_particles;
    mutable std::vector<double> m_work;
};

// ATMatrix (matrix/velocities.hpp:153-254): the adjoint, forces (3 per contact) to 6 values
// per active body.  Applied on the GPU.
template <class Contacts_t, class Particles_t>
class ATMatrix {
  public:
    static constexpr std::size_t dim = Particles_t::dim_;
    ATMatrix(const Contacts_t& contacts, const Particles_t& particles) : m_contacts(contacts), m_particles(particles) {}
    template <class Vec>
    const std::vector<double>& mat_mult(const Vec& f) const {
        if (std::size(f) != 3 * m_contacts.size()) throw gpu_error("ATMatrix::mat_mult: f must hold 3 values per contact");
        detail::handle_guard g{detail::jacobian_handle(m_contacts, m_particles)};
        m_work.assign(6 * m_particles.nb_active(), 0.0);
        if (!m_contacts.empty()) detail::check_abi(scopi_gpu_atmat(g.h, std::data(f), m_work.data()), g.h, "atmat");
        return m_work;
    }

  private:
    const Contacts_t& m_contacts;
    const Particles_t& m_particles;
    mutable std::vector<double> m_work;
};

}  // namespace scopi
