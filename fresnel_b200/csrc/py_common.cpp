// py_common.cpp -- the `_common` extension module: value types shared by every backend.
//
// Mirrors fresnel's `_common` module (fresnel/common/module-common.cc:37-115) class for class:
// RGBf, Material, vec3f, UserCamera, CameraModel, CameraBasis, Lights, plus gpu_built(),
// cpu_built() and find_polyhedron_faces().  This build ships only the GPU backend.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <algorithm>
#include <cmath>
#include <sstream>
#include <stdexcept>
#include <vector>

#include "host_types.hpp"

namespace py = pybind11;
using namespace frh;

namespace {

struct D3 {
    double x, y, z;
};
inline D3 sub(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double dotd(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 crossd(D3 a, D3 b)
{
    return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Number of corners of the convex polygon formed by coplanar points (monotone chain in the
// plane's 2-D frame; points on edges or inside are not corners).
size_t polygon_corners(const std::vector<D3>& pts, D3 n, std::vector<D3>& corners)
{
    D3 a = std::fabs(n.x) < 0.9 ? D3{1, 0, 0} : D3{0, 1, 0};
    D3 e1 = crossd(n, a);
    double l1 = std::sqrt(dotd(e1, e1));
    e1 = D3{e1.x / l1, e1.y / l1, e1.z / l1};
    D3 e2 = crossd(n, e1);
    struct P {
        double u, v;
        size_t i;
    };
    std::vector<P> p;
    for (size_t i = 0; i < pts.size(); ++i)
        p.push_back(P{dotd(pts[i], e1), dotd(pts[i], e2), i});
    std::sort(p.begin(), p.end(), [](const P& x, const P& y) {
        return x.u < y.u || (x.u == y.u && x.v < y.v);
    });
    double scale = 0;
    for (auto& q : p)
        scale = std::max(scale, std::max(std::fabs(q.u), std::fabs(q.v)));
    const double eps = 1e-9 * (scale * scale + 1e-300);
    auto turn = [](const P& o, const P& a_, const P& b) {
        return (a_.u - o.u) * (b.v - o.v) - (a_.v - o.v) * (b.u - o.u);
    };
    std::vector<P> h(2 * p.size() + 1);
    size_t k = 0;
    for (size_t i = 0; i < p.size(); ++i) {
        while (k >= 2 && turn(h[k - 2], h[k - 1], p[i]) <= eps)
            k--;
        h[k++] = p[i];
    }
    for (size_t i = p.size() - 1, t = k + 1; i-- > 0;) {
        while (k >= t && turn(h[k - 2], h[k - 1], p[i]) <= eps)
            k--;
        h[k++] = p[i];
    }
    size_t nc = k > 1 ? k - 1 : k;
    corners.clear();
    for (size_t i = 0; i < nc; ++i)
        corners.push_back(pts[h[i].i]);
    return nc;
}

// find_polyhedron_faces (fresnel/common/ConvexPolyhedronBuilder.cc:25-83).  The reference
// computes the hull with qhull (absent here); this version enumerates supporting planes
// through vertex triples, merges coplanar ones, and reports per face the centroid of its corner
// vertices, the outward unit normal, colour (0.9, 0.9, 0.9) and corner count.  It is O(N^4)
// and meant for the small vertex sets of particle shapes.
py::dict find_polyhedron_faces(py::array_t<double, py::array::c_style | py::array::forcecast> verts)
{
    py::buffer_info info = verts.request();
    if (info.ndim != 2)
        throw std::runtime_error("verts must be a 2-dimensional array");
    if (info.shape[1] != 3)
        throw std::runtime_error("verts must be an N by 3 array");
    size_t N = size_t(info.shape[0]);
    const double* c = static_cast<const double*>(info.ptr);
    std::vector<D3> v(N);
    double scale = 0;
    for (size_t i = 0; i < N; ++i) {
        v[i] = D3{c[3 * i], c[3 * i + 1], c[3 * i + 2]};
        scale = std::max(scale, std::sqrt(dotd(v[i], v[i])));
    }
    if (N < 4)
        throw std::runtime_error("a convex polyhedron needs at least 4 vertices");
    const double tol = 1e-9 * std::max(scale, 1e-300) * 1e3;
    struct Plane {
        D3 n;
        double d;
    };
    std::vector<Plane> planes;
    for (size_t i = 0; i < N; ++i)
        for (size_t j = i + 1; j < N; ++j)
            for (size_t k = j + 1; k < N; ++k) {
                D3 n = crossd(sub(v[j], v[i]), sub(v[k], v[i]));
                double ln = std::sqrt(dotd(n, n));
                if (ln <= 1e-12 * scale * scale)
                    continue;
                n = D3{n.x / ln, n.y / ln, n.z / ln};
                double d = dotd(n, v[i]);
                bool pos = false, neg = false;
                for (size_t m = 0; m < N && !(pos && neg); ++m) {
                    double s = dotd(n, v[m]) - d;
                    if (s > tol)
                        pos = true;
                    else if (s < -tol)
                        neg = true;
                }
                if (pos && neg)
                    continue;
                if (!pos && !neg)
                    throw std::runtime_error("vertices are coplanar");
                if (pos) {
                    n = D3{-n.x, -n.y, -n.z};
                    d = -d;
                }
                bool dup = false;
                for (auto& p : planes)
                    if (dotd(p.n, n) > 1.0 - 1e-10 && std::fabs(p.d - d) <= tol) {
                        dup = true;
                        break;
                    }
                if (!dup)
                    planes.push_back(Plane{n, d});
            }
    std::vector<float> origin, normal, color;
    std::vector<unsigned int> sides;
    for (auto& p : planes) {
        std::vector<D3> on;
        for (size_t m = 0; m < N; ++m)
            if (std::fabs(dotd(p.n, v[m]) - p.d) <= tol)
                on.push_back(v[m]);
        std::vector<D3> corners;
        size_t nc = polygon_corners(on, p.n, corners);
        D3 o{0, 0, 0};
        for (auto& q : corners) {
            o.x += q.x;
            o.y += q.y;
            o.z += q.z;
        }
        double inv = nc ? 1.0 / double(nc) : 0.0;
        origin.insert(origin.end(), {float(o.x * inv), float(o.y * inv), float(o.z * inv)});
        normal.insert(normal.end(), {float(p.n.x), float(p.n.y), float(p.n.z)});
        color.insert(color.end(), {0.9f, 0.9f, 0.9f});
        sides.push_back(unsigned(nc));
    }
    double radius = 0;
    for (size_t i = 0; i < N; ++i)
        radius = std::max(radius, std::sqrt(dotd(v[i], v[i])));
    size_t F = planes.size();
    py::dict r;
    r["face_origin"] = py::array_t<float>({F, size_t(3)}, origin.data());
    r["face_normal"] = py::array_t<float>({F, size_t(3)}, normal.data());
    r["face_color"] = py::array_t<float>({F, size_t(3)}, color.data());
    r["face_sides"] = py::array_t<unsigned int>(F, sides.data());
    r["radius"] = radius;
    return r;
}

// The reference stores at most 4 lights (fresnel/common/Light.h:36-40).
unsigned light_slot(unsigned i)
{
    if (i >= 4)
        throw py::index_error("light index out of range (at most 4 lights)");
    return i;
}

}  // namespace

PYBIND11_MODULE(_common, m)
{
    m.doc() = "fresnel_b200 value types (mirror of fresnel._common)";
    m.def("gpu_built", []() { return true; });
    m.def("cpu_built", []() { return false; });
    m.def("find_polyhedron_faces", &find_polyhedron_faces);

    py::class_<RGBf>(m, "RGBf")
        .def(py::init<float, float, float>())
        .def_readwrite("r", &RGBf::r)
        .def_readwrite("g", &RGBf::g)
        .def_readwrite("b", &RGBf::b);

    py::class_<Material>(m, "Material")
        .def(py::init<>())
        .def_readwrite("solid", &Material::solid)
        .def_readwrite("primitive_color_mix", &Material::primitive_color_mix)
        .def_readwrite("roughness", &Material::roughness)
        .def_readwrite("specular", &Material::specular)
        .def_readwrite("spec_trans", &Material::spec_trans)
        .def_readwrite("metal", &Material::metal)
        .def_readwrite("color", &Material::color)
        .def("__repr__", [](const Material& a) {
            std::ostringstream s;
            s << "<fresnel._common.Material: solid=" << a.solid << " color=(" << a.color.r << ", "
              << a.color.g << ", " << a.color.b << ") primitive_color_mix=" << a.primitive_color_mix
              << " roughness=" << a.roughness << " specular=" << a.specular
              << " spec_trans=" << a.spec_trans << " metal=" << a.metal << ">";
            return s.str();
        });

    py::class_<vec3f>(m, "vec3f")
        .def(py::init<float, float, float>())
        .def_readwrite("x", &vec3f::x)
        .def_readwrite("y", &vec3f::y)
        .def_readwrite("z", &vec3f::z)
        .def("__repr__", [](const vec3f& a) {
            std::ostringstream s;
            s << "<fresnel._common.vec3f (" << a.x << ", " << a.y << ", " << a.z << ")>";
            return s.str();
        });

    py::class_<UserCamera>(m, "UserCamera")
        .def(py::init<>())
        .def_readwrite("position", &UserCamera::position)
        .def_readwrite("look_at", &UserCamera::look_at)
        .def_readwrite("up", &UserCamera::up)
        .def_readwrite("h", &UserCamera::h)
        .def_readwrite("f", &UserCamera::f)
        .def_readwrite("f_stop", &UserCamera::f_stop)
        .def_readwrite("focus_distance", &UserCamera::focus_distance)
        .def_readwrite("model", &UserCamera::model);

    py::enum_<CameraModel>(m, "CameraModel")
        .value("orthographic", CameraModel::orthographic)
        .value("perspective", CameraModel::perspective);

    py::class_<CameraBasis>(m, "CameraBasis")
        .def(py::init<const UserCamera&>())
        .def_readwrite("u", &CameraBasis::u)
        .def_readwrite("v", &CameraBasis::v)
        .def_readwrite("w", &CameraBasis::w);

    py::class_<Lights>(m, "Lights")
        .def(py::init<>())
        .def_readwrite("N", &Lights::N)
        .def("getDirection", [](Lights& l, unsigned i) { return l.direction[light_slot(i)]; })
        .def("setDirection",
             [](Lights& l, unsigned i, const vec3f& v) { l.direction[light_slot(i)] = v; })
        .def("getColor", [](Lights& l, unsigned i) { return l.color[light_slot(i)]; })
        .def("setColor", [](Lights& l, unsigned i, const RGBf& v) { l.color[light_slot(i)] = v; })
        .def("getTheta", [](Lights& l, unsigned i) { return l.theta[light_slot(i)]; })
        .def("setTheta", [](Lights& l, unsigned i, float v) { l.theta[light_slot(i)] = v; });
}
