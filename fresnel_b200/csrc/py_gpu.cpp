// py_gpu.cpp -- the `_gpu` extension module: fresnel's GPU backend classes over the C ABI.
//
// Class and method names follow fresnel's `_gpu` module (fresnel/gpu/module-gpu.cc:27-43):
// Device, Scene, Geometry, GeometrySphere, GeometryCylinder, GeometryConvexPolyhedron,
// GeometryMesh, GeometryPolygon, Tracer, TracerDirect, TracerPath and the Array* buffer classes.  Everything
// below is host bookkeeping; all rendering work happens in libfrb200 (include/fresnel_b200.h).
//
// Arrays: geometry arrays keep an authoritative host copy; unmap() marks the array stale and
// the next render uploads stale arrays (a BVH rebuild follows only when a geometric array
// changed), unmapRead() ends a read and marks nothing.  Output arrays are authoritative on the
// device; map() downloads them into the array's buffer, readCopy() into a new numpy array.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "fresnel_b200.h"
#include "host_types.hpp"

#if defined(__SSE2__)
#include <emmintrin.h>
#endif

extern "C" fr_status fr_debug_traversal_compare(fr_scene* sc, const float* rays, uint32_t n,
                                                uint32_t* out);

namespace py = pybind11;
using namespace frh;

namespace {

void check(fr_status s)
{
    if (s != FR_OK)
        throw std::runtime_error(fr_last_error());
}

// ---------------------------------------------------------------------------------------------
// engine objects with shared ownership: an Array keeps the object whose buffer it exposes
// alive (the reference's Array holds its OptiX buffer the same way, fresnel/gpu/Array.h:98-223)
// ---------------------------------------------------------------------------------------------
struct DeviceH;
struct SceneH;

struct TracerCore {
    std::shared_ptr<DeviceH> device;
    fr_tracer* tracer = nullptr;
    ~TracerCore() { fr_tracer_destroy(tracer); }
};

struct GeometryCore {
    std::shared_ptr<SceneH> scene;
    fr_geometry* geom = nullptr;
    ~GeometryCore() { fr_geometry_destroy(geom); }
};

// ---------------------------------------------------------------------------------------------
// arrays
// ---------------------------------------------------------------------------------------------
// Host copy of an array in page-locked memory (fr_host_alloc), so that uploads and downloads
// run at full link speed without a staging copy; plain heap memory if none can be had.
class HostStore {
public:
    HostStore() = default;
    HostStore(const HostStore&) = delete;
    HostStore& operator=(const HostStore&) = delete;
    ~HostStore() { release(); }
    void assign(size_t n)
    {
        release();
        if (n == 0)
            return;
        void* p = nullptr;
        if (fr_host_alloc(n, &p) == FR_OK) {
            ptr_ = static_cast<unsigned char*>(p);
            pinned_ = true;
        } else {
            heap_.assign(n, 0);
            ptr_ = heap_.data();
        }
        n_ = n;
        std::memset(ptr_, 0, n);
    }
    unsigned char* data() { return ptr_; }
    size_t size() const { return n_; }
    bool empty() const { return n_ == 0; }
    bool pinned() const { return pinned_; }

private:
    void release()
    {
        if (pinned_)
            fr_host_free(ptr_);
        heap_.clear();
        heap_.shrink_to_fit();
        ptr_ = nullptr;
        n_ = 0;
        pinned_ = false;
    }
    unsigned char* ptr_ = nullptr;
    size_t n_ = 0;
    bool pinned_ = false;
    std::vector<unsigned char> heap_;
};

// dst[...] = src for two C-contiguous arrays of one shape, written with streaming stores that
// bypass the caches.  A geometry array's page-locked host copy is uploaded right after it is
// written; when several threads had written it with ordinary stores, its lines sat modified in
// those cores' caches and the copy engine read 12 MB at a fifth of the link speed (1.16 against
// 0.23 ms), while after streaming stores, or after one thread's copy, it read at full speed.
// Takes float32 from float32 or float64 (rounded to nearest, as numpy's cast rounds) and uint8
// from uint8, and returns false for any other pair, whose copy is left to the caller.
bool stream_copy(const py::buffer& dst_buf, const py::buffer& src_buf)
{
    const py::buffer_info d = dst_buf.request(true), s = src_buf.request();
    if (d.ndim != s.ndim || d.shape != s.shape)
        return false;
    auto c_order = [](const py::buffer_info& b) {
        py::ssize_t want = b.itemsize;
        for (py::ssize_t k = b.ndim; k-- > 0;) {
            if (b.shape[size_t(k)] > 1 && b.strides[size_t(k)] != want)
                return false;
            want *= b.shape[size_t(k)];
        }
        return true;
    };
    if (!c_order(d) || !c_order(s))
        return false;
    const bool f32 = d.format == "f" && d.itemsize == 4;
    const bool from_f32 = f32 && s.format == "f" && s.itemsize == 4;
    const bool from_f64 = f32 && s.format == "d" && s.itemsize == 8;
    const bool u8 = d.format == "B" && s.format == "B";
    if (!from_f32 && !from_f64 && !u8)
        return false;
    unsigned char* out = static_cast<unsigned char*>(d.ptr);
    const size_t n = size_t(d.size);
    const uintptr_t d0 = reinterpret_cast<uintptr_t>(d.ptr), s0 = reinterpret_cast<uintptr_t>(s.ptr);
    if (d0 < s0 + n * size_t(s.itemsize) && s0 < d0 + n * size_t(d.itemsize))
        return false;  // overlapping storage: numpy buffers the copy
    // bytes to out[0, nbytes) with 16-byte streaming stores where out is aligned
    auto store = [](unsigned char* to, const unsigned char* from, size_t nbytes) {
#if defined(__SSE2__)
        size_t head = (16u - (reinterpret_cast<uintptr_t>(to) & 15u)) & 15u;
        head = std::min(head, nbytes);
        std::memcpy(to, from, head);
        size_t k = head;
        for (; k + 16 <= nbytes; k += 16)
            _mm_stream_si128(reinterpret_cast<__m128i*>(to + k),
                             _mm_loadu_si128(reinterpret_cast<const __m128i*>(from + k)));
        std::memcpy(to + k, from + k, nbytes - k);
#else
        std::memcpy(to, from, nbytes);
#endif
    };
    {
        py::gil_scoped_release nogil;
        if (from_f64) {
            const double* in = static_cast<const double*>(s.ptr);
            float tmp[2048];
            for (size_t i = 0; i < n; i += 2048) {
                const size_t m = std::min<size_t>(2048, n - i);
                for (size_t j = 0; j < m; ++j)
                    tmp[j] = static_cast<float>(in[i + j]);
                store(out + 4 * i, reinterpret_cast<const unsigned char*>(tmp), 4 * m);
            }
        } else {
            store(out, static_cast<const unsigned char*>(s.ptr), n * size_t(d.itemsize));
        }
#if defined(__SSE2__)
        _mm_sfence();
#endif
    }
    return true;
}

// Page-locked blocks that back the arrays returned by whole reads of tracer outputs: the download
// lands in the array handed to numpy, with no copy on the host and no page faults on fresh
// memory, and numpy's release of the array returns the block here.  A block serves requests of
// more than half its size; at most MAX_CACHED bytes wait in the pool, and at most MAX_LIVE bytes
// are held by arrays (a program that keeps many frames gets ordinary memory beyond that, so
// that it does not lock the host's memory).  The pool is never destroyed, since arrays may be
// released after the module is torn down.
class PinnedPool {
public:
    static PinnedPool& get()
    {
        static PinnedPool* pool = new PinnedPool();
        return *pool;
    }
    // a block of at least n bytes (its size in cap), or nullptr when none can be had
    void* take(size_t n, size_t& cap)
    {
        {
            std::lock_guard<std::mutex> lock(m_);
            auto it = free_.lower_bound(n);
            if (it != free_.end() && it->first / 2 < n) {
                cap = it->first;
                void* p = it->second;
                cached_ -= cap;
                live_ += cap;
                free_.erase(it);
                return p;
            }
            if (live_ + n > MAX_LIVE)
                return nullptr;
            live_ += n;  // reserved before the allocation, released if it fails
        }
        void* p = nullptr;
        if (fr_host_alloc(n, &p) != FR_OK) {
            std::lock_guard<std::mutex> lock(m_);
            live_ -= n;
            return nullptr;
        }
        cap = n;
        return p;
    }
    void give(void* p, size_t cap)
    {
        {
            std::lock_guard<std::mutex> lock(m_);
            live_ -= cap;
            if (cached_ + cap <= MAX_CACHED) {
                free_.emplace(cap, p);
                cached_ += cap;
                return;
            }
        }
        fr_host_free(p);
    }

private:
    static constexpr size_t MAX_CACHED = size_t(256) << 20;
    static constexpr size_t MAX_LIVE = size_t(1) << 30;
    std::mutex m_;
    std::multimap<size_t, void*> free_;
    size_t cached_ = 0;
    size_t live_ = 0;
};

struct ArrayBase {
    HostStore data;
    std::vector<py::ssize_t> shape;
    size_t item = 4;        // bytes per scalar
    std::string format;     // python struct format of one scalar
    bool mapped = false;
    bool stale = false;     // host copy newer than the device copy (geometry arrays)
    // owner: a geometry field or a tracer output
    std::shared_ptr<GeometryCore> gcore;
    fr_geometry* geom = nullptr;
    int field = -1;
    std::shared_ptr<TracerCore> tcore;
    fr_tracer* tracer = nullptr;
    int output = -1;  // 0 linear, 1 srgb

    size_t count() const
    {
        size_t n = 1;
        for (auto s : shape)
            n *= size_t(s);
        return n;
    }
    void map()
    {
        if (tracer) {
            if (output == 0)
                check(fr_tracer_read_linear(tracer, reinterpret_cast<float*>(data.data()),
                                            data.size()));
            else
                check(fr_tracer_read_srgb(tracer, data.data(), data.size()));
        }
        mapped = true;
    }
    void unmap()
    {
        mapped = false;
        if (geom)
            stale = true;
    }
    // unmap after a read: the host copy is unchanged, so nothing is uploaded or rebuilt
    void unmap_read() { mapped = false; }
    // A copy of a tracer output as a new numpy array whose storage is a pooled page-locked block
    // that the download writes directly; None for geometry arrays, or when no block can be had.
    py::object read_copy()
    {
        if (!tracer)
            return py::none();
        const size_t nbytes = data.size();
        size_t cap = 0;
        void* p = PinnedPool::get().take(nbytes, cap);
        if (!p)
            return py::none();
        const fr_status s =
            output == 0 ? fr_tracer_read_linear(tracer, static_cast<float*>(p), nbytes)
                        : fr_tracer_read_srgb(tracer, static_cast<uint8_t*>(p), nbytes);
        if (s != FR_OK) {
            PinnedPool::get().give(p, cap);
            check(s);
        }
        auto* block = new std::pair<void*, size_t>(p, cap);
        py::capsule owner(block, [](void* v) {
            auto* b = static_cast<std::pair<void*, size_t>*>(v);
            PinnedPool::get().give(b->first, b->second);
            delete b;
        });
        return py::array(py::dtype(format), shape, strides(), p, owner);
    }
    // push a stale geometry array to the device
    void sync()
    {
        if (geom && stale && !data.empty()) {
            check(fr_geometry_write(geom, field, data.data(), 0, data.size()));
            stale = false;
        }
    }
    std::vector<py::ssize_t> strides() const  // C order, in bytes
    {
        std::vector<py::ssize_t> st(shape.size());
        py::ssize_t s = py::ssize_t(item);
        for (size_t k = shape.size(); k-- > 0;) {
            st[k] = s;
            s *= shape[k];
        }
        return st;
    }
    py::buffer_info buffer()
    {
        if (!mapped)
            throw std::runtime_error("Array must be mapped before it can be accessed");
        return py::buffer_info(data.data(), py::ssize_t(item), format, py::ssize_t(shape.size()),
                               shape, strides());
    }
};

// one C++ type per Python class name (fresnel/cpu/Array.cc:12-78)
template <int K> struct ArrayK : ArrayBase {};
using ArrayRGBAf = ArrayK<0>;
using ArrayRGBAc = ArrayK<1>;
using ArrayRGBf = ArrayK<2>;
using ArrayVec3f = ArrayK<3>;
using ArrayQuat3f = ArrayK<4>;
using Array_f = ArrayK<5>;
using ArrayVec2f = ArrayK<6>;
using ArrayRGBc = ArrayK<7>;

template <class A>
std::shared_ptr<A> make_array(std::vector<py::ssize_t> shape, bool byte_scalar = false)
{
    auto a = std::make_shared<A>();
    a->shape = std::move(shape);
    a->item = byte_scalar ? 1 : 4;
    a->format = byte_scalar ? py::format_descriptor<unsigned char>::format()
                            : py::format_descriptor<float>::format();
    a->data.assign(a->count() * a->item);
    return a;
}

// ---------------------------------------------------------------------------------------------
// device / scene
// ---------------------------------------------------------------------------------------------
struct DeviceH {
    fr_device* dev = nullptr;
    DeviceH(const std::string& /*ptx_root*/, int n) { check(fr_device_create(n, &dev)); }
    ~DeviceH() { fr_device_destroy(dev); }
    std::string describe() const
    {
        char buf[512];
        check(fr_device_describe(dev, buf, sizeof(buf)));
        return buf;
    }
    static std::string all_gpus()
    {
        char buf[4096];
        check(fr_get_all_gpus(buf, sizeof(buf)));
        return buf;
    }
};

struct GeometryH;

struct SceneH {
    std::shared_ptr<DeviceH> device;
    fr_scene* scene = nullptr;
    UserCamera camera;
    RGBf background{0, 0, 0};
    float background_alpha = 0.0f;
    Lights lights;
    std::set<GeometryH*> geoms;

    explicit SceneH(std::shared_ptr<DeviceH> d) : device(std::move(d))
    {
        check(fr_scene_create(device->dev, &scene));
        // default lights (fresnel/gpu/Scene.cc:15-28)
        lights.N = 2;
        lights.direction[0] = vec3f(-1, 0.3f, 1);
        lights.color[0] = RGBf(1, 1, 1);
        lights.direction[1] = vec3f(1, 0, 1);
        lights.color[1] = RGBf(0.1f, 0.1f, 0.1f);
    }
    ~SceneH() { fr_scene_destroy(scene); }
    void sync();
};

struct GeometryH {
    std::shared_ptr<SceneH> scene;
    std::shared_ptr<GeometryCore> core;
    fr_geometry* geom = nullptr;
    bool valid = false;
    Material material, outline;
    float outline_width = 0.0f;
    std::vector<std::shared_ptr<ArrayBase>> arrays;

    explicit GeometryH(std::shared_ptr<SceneH> s) : scene(std::move(s))
    {
        // defaults of the reference's geometry constructors (fresnel/cpu/GeometrySphere.cc:31-33)
        material.solid = 0;
        material.color = RGBf(1, 0, 1);
        material.roughness = 0.1f;
        material.specular = 0.5f;
        outline.solid = 1;
        outline.color = RGBf(0, 0, 0);
        outline.roughness = 0.1f;
        outline.specular = 0.5f;
    }
    // ~Geometry removes the geometry from its scene (fresnel/cpu/Geometry.cc:18-21); its
    // buffers live on while an Array still refers to them.
    virtual ~GeometryH()
    {
        scene->geoms.erase(this);
        if (geom)
            fr_geometry_remove(geom);
    }
    // take ownership of a geometry just created by the engine
    void own(fr_geometry* g)
    {
        geom = g;
        core = std::make_shared<GeometryCore>();
        core->scene = scene;
        core->geom = g;
    }
    void attach()
    {
        valid = true;
        scene->geoms.insert(this);
        push_material();
    }
    template <class A> std::shared_ptr<A> add_array(int field, std::vector<py::ssize_t> shape)
    {
        auto a = make_array<A>(std::move(shape));
        a->gcore = core;
        a->geom = geom;
        a->field = field;
        arrays.push_back(a);
        return a;
    }
    void push_material()
    {
        fr_material m = to_abi(material), o = to_abi(outline);
        check(fr_geometry_set_material(geom, &m, &o, outline_width));
    }
    Material getMaterial() const { return material; }
    void setMaterial(const Material& m)
    {
        material = m;
        push_material();
    }
    Material getOutlineMaterial() const { return outline; }
    void setOutlineMaterial(const Material& m)
    {
        outline = m;
        push_material();
    }
    float getOutlineWidth() const { return outline_width; }
    void setOutlineWidth(float w)
    {
        outline_width = w;
        push_material();
    }
    void enable()
    {
        if (!valid)
            throw std::runtime_error("Cannot enable inactive Geometry");
        check(fr_geometry_set_enabled(geom, 1));
    }
    void disable()
    {
        if (!valid)
            throw std::runtime_error("Cannot disable inactive Geometry");
        check(fr_geometry_set_enabled(geom, 0));
    }
    void remove()
    {
        if (valid) {
            check(fr_geometry_remove(geom));
            valid = false;
        }
    }
    // Array writes are tracked per array (see ArrayBase::unmap); nothing else to record.
    void update() {}
    void sync()
    {
        for (auto& a : arrays)
            a->sync();
    }
};

void SceneH::sync()
{
    for (GeometryH* g : geoms)
        g->sync();
}

struct GeometrySphereH : GeometryH {
    std::shared_ptr<ArrayVec3f> position;
    std::shared_ptr<Array_f> radius;
    std::shared_ptr<ArrayRGBf> color;
    GeometrySphereH(std::shared_ptr<SceneH> s, unsigned n) : GeometryH(std::move(s))
    {
        {
            fr_geometry* g = nullptr;
            check(fr_geometry_create_sphere(scene->scene, n, &g));
            own(g);
        }
        position = add_array<ArrayVec3f>(FR_FIELD_POSITION, {py::ssize_t(n), 3});
        radius = add_array<Array_f>(FR_FIELD_RADIUS, {py::ssize_t(n)});
        color = add_array<ArrayRGBf>(FR_FIELD_COLOR, {py::ssize_t(n), 3});
        attach();
    }
};

struct GeometryCylinderH : GeometryH {
    std::shared_ptr<ArrayVec3f> points;
    std::shared_ptr<Array_f> radius;
    std::shared_ptr<ArrayRGBf> color;
    GeometryCylinderH(std::shared_ptr<SceneH> s, unsigned n) : GeometryH(std::move(s))
    {
        {
            fr_geometry* g = nullptr;
            check(fr_geometry_create_cylinder(scene->scene, n, &g));
            own(g);
        }
        points = add_array<ArrayVec3f>(FR_FIELD_POINTS, {py::ssize_t(n), 2, 3});
        radius = add_array<Array_f>(FR_FIELD_RADIUS, {py::ssize_t(n)});
        color = add_array<ArrayRGBf>(FR_FIELD_COLOR, {py::ssize_t(n), 2, 3});
        attach();
    }
};

using farray = py::array_t<float, py::array::c_style | py::array::forcecast>;

void require_nx3(const farray& a, const char* name, const char* what)
{
    if (a.ndim() != 2)
        throw std::runtime_error(std::string(name) + " must be a 2-dimensional array");
    if (a.shape(1) != 3)
        throw std::runtime_error(std::string(name) + " must be a " + what + " by 3 array");
}

struct GeometryConvexPolyhedronH : GeometryH {
    std::shared_ptr<ArrayVec3f> position;
    std::shared_ptr<ArrayQuat3f> orientation;
    std::shared_ptr<ArrayRGBf> color;
    float color_by_face = 0.0f;
    // argument checks of fresnel/cpu/GeometryConvexPolyhedron.cc:47-78
    GeometryConvexPolyhedronH(std::shared_ptr<SceneH> s, farray origins, farray normals,
                              farray colors, unsigned n, float r)
        : GeometryH(std::move(s))
    {
        require_nx3(origins, "plane_origins", "Nvert");
        require_nx3(normals, "plane_normals", "Nvert");
        if (normals.shape(0) != origins.shape(0))
            throw std::runtime_error("Number of vertices must match in origin and normal arrays");
        require_nx3(colors, "plane_colors", "Nvert");
        if (colors.shape(0) != origins.shape(0))
            throw std::runtime_error("Number of vertices must match in origin and color arrays");
        fr_geometry* g = nullptr;
        check(fr_geometry_create_polyhedron(scene->scene, origins.data(), normals.data(),
                                            colors.data(), unsigned(origins.shape(0)), n, r, &g));
        own(g);
        position = add_array<ArrayVec3f>(FR_FIELD_POSITION, {py::ssize_t(n), 3});
        orientation = add_array<ArrayQuat3f>(FR_FIELD_ORIENTATION, {py::ssize_t(n), 4});
        color = add_array<ArrayRGBf>(FR_FIELD_COLOR, {py::ssize_t(n), 3});
        attach();
    }
    void setColorByFace(float f)
    {
        color_by_face = f;
        check(fr_geometry_set_color_by_face(geom, f));
    }
    float getColorByFace() const { return color_by_face; }
};

struct GeometryMeshH : GeometryH {
    std::shared_ptr<ArrayVec3f> position;
    std::shared_ptr<ArrayQuat3f> orientation;
    std::shared_ptr<ArrayRGBf> color;
    // argument checks of fresnel/cpu/GeometryMesh.cc:27-34
    GeometryMeshH(std::shared_ptr<SceneH> s, farray vertices, unsigned n) : GeometryH(std::move(s))
    {
        if (vertices.ndim() != 2)
            throw std::runtime_error("vertices must be a 2-dimensional array");
        if (vertices.shape(1) != 3)
            throw std::runtime_error("vertices must be a Nvert by 3 array");
        if (vertices.shape(0) % 3 != 0)
            throw std::runtime_error("the number of triangle vertices must be a multiple of three.");
        unsigned nv = unsigned(vertices.shape(0));
        fr_geometry* g = nullptr;
        check(fr_geometry_create_mesh(scene->scene, vertices.data(), nv, n, &g));
        own(g);
        position = add_array<ArrayVec3f>(FR_FIELD_POSITION, {py::ssize_t(n), 3});
        orientation = add_array<ArrayQuat3f>(FR_FIELD_ORIENTATION, {py::ssize_t(n), 4});
        color = add_array<ArrayRGBf>(FR_FIELD_COLOR, {py::ssize_t(nv), 3});
        attach();
    }
};

struct GeometryPolygonH : GeometryH {
    std::shared_ptr<ArrayVec2f> position;
    std::shared_ptr<Array_f> angle;
    std::shared_ptr<ArrayRGBf> color;
    // argument checks of fresnel/cpu/GeometryPolygon.cc:46-52
    GeometryPolygonH(std::shared_ptr<SceneH> s, farray vertices, float rounding_radius, unsigned n)
        : GeometryH(std::move(s))
    {
        if (vertices.ndim() != 2)
            throw std::runtime_error("vertices must be a 2-dimensional array");
        if (vertices.shape(1) != 2)
            throw std::runtime_error("vertices must be a Nvert by 2 array");
        fr_geometry* g = nullptr;
        check(fr_geometry_create_polygon(scene->scene, vertices.data(),
                                         unsigned(vertices.shape(0)), rounding_radius, n, &g));
        own(g);
        position = add_array<ArrayVec2f>(FR_FIELD_POSITION, {py::ssize_t(n), 2});
        angle = add_array<Array_f>(FR_FIELD_ANGLE, {py::ssize_t(n)});
        color = add_array<ArrayRGBf>(FR_FIELD_COLOR, {py::ssize_t(n), 3});
        attach();
    }
    float getRadius() const
    {
        float r = 0.0f;
        check(fr_geometry_get_radius(geom, &r));
        return r;
    }
};

// ---------------------------------------------------------------------------------------------
// tracers
// ---------------------------------------------------------------------------------------------
struct TracerH {
    std::shared_ptr<DeviceH> device;
    std::shared_ptr<TracerCore> core;
    fr_tracer* tracer = nullptr;
    unsigned w = 0, h = 0;
    unsigned seed = 0;
    bool highlight = false;
    RGBf highlight_color{1, 0, 1};
    std::shared_ptr<ArrayRGBAf> linear;
    std::shared_ptr<ArrayRGBAc> srgb;

    TracerH(std::shared_ptr<DeviceH> d, unsigned w_, unsigned h_) : device(std::move(d))
    {
        core = std::make_shared<TracerCore>();
        core->device = device;
        check(fr_tracer_create(device->dev, w_, h_, &core->tracer));
        tracer = core->tracer;
        make_outputs(w_, h_);
    }
    virtual ~TracerH() = default;
    void make_outputs(unsigned w_, unsigned h_)
    {
        w = w_;
        h = h_;
        linear = make_array<ArrayRGBAf>({py::ssize_t(h), py::ssize_t(w), 4});
        linear->tcore = core;
        linear->tracer = tracer;
        linear->output = 0;
        srgb = make_array<ArrayRGBAc>({py::ssize_t(h), py::ssize_t(w), 4}, true);
        srgb->tcore = core;
        srgb->tracer = tracer;
        srgb->output = 1;
    }
    virtual void resize(unsigned w_, unsigned h_)
    {
        if (w_ == 0 || h_ == 0)
            throw std::runtime_error("Invalid dimensions");
        check(fr_tracer_resize(tracer, w_, h_));
        make_outputs(w_, h_);
    }
    fr_render_params params(const SceneH& s) const
    {
        fr_render_params p;
        std::memset(&p, 0, sizeof(p));
        p.camera = to_abi(s.camera);
        p.lights = to_abi(s.lights);
        p.background_color[0] = s.background.r;
        p.background_color[1] = s.background.g;
        p.background_color[2] = s.background.b;
        p.background_alpha = s.background_alpha;
        p.seed = seed;
        p.highlight_warning = highlight ? 1 : 0;
        p.highlight_color[0] = highlight_color.r;
        p.highlight_color[1] = highlight_color.g;
        p.highlight_color[2] = highlight_color.b;
        return p;
    }
    void check_scene(const std::shared_ptr<SceneH>& s) const
    {
        if (s->device != device)
            throw std::runtime_error("Scene and Tracer devices do not match");
    }
    virtual void render(std::shared_ptr<SceneH> s) { check_scene(s); }
    py::dict stats() const
    {
        fr_stats st;
        check(fr_tracer_get_stats(tracer, &st));
        py::dict d;
        d["rays"] = st.rays;
        d["paths"] = st.paths;
        d["dropped"] = st.dropped;
        d["box_tests"] = st.box_tests;
        d["prim_tests"] = st.prim_tests;
        d["kernel_launches"] = st.kernel_launches;
        d["bvh_builds"] = st.bvh_builds;
        d["bvh_refits"] = st.bvh_refits;
        d["grid_builds"] = st.grid_builds;
        d["grid"] = st.last_render_grid;
        d["bvh_build_ms"] = st.bvh_build_ms;
        d["primary_ms"] = st.primary_ms;
        d["shade_ms"] = st.shade_ms;
        d["extend_ms"] = st.extend_ms;
        d["primary_launches"] = st.primary_launches;
        d["shade_launches"] = st.shade_launches;
        d["extend_launches"] = st.extend_launches;
        return d;
    }
};

struct TracerDirectH : TracerH {
    unsigned aa_n = 8;
    using TracerH::TracerH;
    void render(std::shared_ptr<SceneH> s) override
    {
        check_scene(s);
        s->sync();
        fr_render_params p = params(*s);
        check(fr_tracer_render_preview(tracer, s->scene, &p, aa_n, nullptr));
    }
    // Preview render that also returns the closest-hit ids of every primary sample as a
    // [h, w, aa_n^2, 2] uint32 array of (geometry index + 1, primitive index); (0, 0) = miss.
    py::array_t<uint32_t> render_hit_ids(std::shared_ptr<SceneH> s)
    {
        check_scene(s);
        s->sync();
        fr_render_params p = params(*s);
        py::array_t<uint32_t> out({py::ssize_t(h), py::ssize_t(w), py::ssize_t(aa_n * aa_n),
                                   py::ssize_t(2)});
        check(fr_tracer_render_preview(tracer, s->scene, &p, aa_n, out.mutable_data()));
        return out;
    }
};

struct TracerPathH : TracerH {
    unsigned n_samples = 0;
    unsigned light_samples = 1;
    TracerPathH(std::shared_ptr<DeviceH> d, unsigned w_, unsigned h_, unsigned ls)
        : TracerH(std::move(d), w_, h_), light_samples(ls)
    {
        reset();
    }
    // TracerPath::reset (fresnel/cpu/TracerPath.cc:31-47)
    void reset()
    {
        n_samples = 0;
        seed++;
        check(fr_tracer_clear(tracer));
    }
    // TracerPath::resize (fresnel/cpu/TracerPath.h:48-53)
    void resize(unsigned w_, unsigned h_) override
    {
        TracerH::resize(w_, h_);
        n_samples = 0;
        seed++;
    }
    void render(std::shared_ptr<SceneH> s) override { render_samples(s, 1); }
    // `k` consecutive render() calls in one engine call (the sample loop stays on the device).
    void render_samples(std::shared_ptr<SceneH> s, unsigned k)
    {
        check_scene(s);
        if (k == 0)
            return;
        s->sync();
        fr_render_params p = params(*s);
        check(fr_tracer_render_path(tracer, s->scene, &p, n_samples + 1, k, light_samples));
        n_samples += k;
    }
    // The same k renders through the allocation-free entry point (the scene must be built).
    void render_samples_static(std::shared_ptr<SceneH> s, unsigned k)
    {
        check_scene(s);
        s->sync();
        fr_render_params p = params(*s);
        check(fr_tracer_render_path_static(tracer, s->scene, &p, n_samples + 1, k, light_samples));
        n_samples += k;
    }
};

// Batched path renders (fr_batch_*): add() queues Path renders of any tracers and scenes of the
// device; render() traces them together and then advances each tracer's sample count.
struct BatchH {
    std::shared_ptr<DeviceH> device;
    fr_batch* batch = nullptr;
    struct Item {
        std::shared_ptr<TracerPathH> tracer;
        std::shared_ptr<SceneH> scene;
        unsigned k;
    };
    std::vector<Item> items;
    explicit BatchH(std::shared_ptr<DeviceH> d) : device(std::move(d))
    {
        check(fr_batch_create(device->dev, &batch));
    }
    ~BatchH() { fr_batch_destroy(batch); }
    // k more samples of `t` on `s`, numbered after the ones already queued for t
    void add(std::shared_ptr<TracerPathH> t, std::shared_ptr<SceneH> s, unsigned k)
    {
        t->check_scene(s);
        if (t->device != device)
            throw std::runtime_error("Tracer and Batch devices do not match");
        if (k == 0)
            return;
        unsigned queued = 0;
        for (auto& it : items)
            if (it.tracer == t)
                queued += it.k;
        s->sync();
        fr_render_params p = t->params(*s);
        check(fr_batch_add_path(batch, t->tracer, s->scene, &p, t->n_samples + queued + 1, k,
                                t->light_samples));
        items.push_back({t, s, k});
    }
    void render()
    {
        for (auto& it : items)
            it.scene->sync();
        fr_status st = fr_batch_render(batch);
        if (st == FR_OK)
            for (auto& it : items)
                it.tracer->n_samples += it.k;
        clear();
        check(st);
    }
    void clear()
    {
        items.clear();
        check(fr_batch_clear(batch));
    }
    py::dict stats() const
    {
        fr_batch_stats st;
        check(fr_batch_get_stats(batch, &st));
        py::dict d;
        d["renders"] = st.renders;
        d["waves"] = st.waves;
        d["graph_launches"] = st.graph_launches;
        d["graph_captures"] = st.graph_captures;
        d["kernel_launches"] = st.kernel_launches;
        d["shade_extend_pairs"] = st.shade_extend_pairs;
        d["box_tests"] = st.box_tests;
        d["prim_tests"] = st.prim_tests;
        d["last_ms"] = st.last_ms;
        d["total_ms"] = st.total_ms;
        return d;
    }
};

template <class A> void export_array(py::module_& m, const char* name)
{
    py::class_<A, std::shared_ptr<A>>(m, name, py::buffer_protocol())
        .def_buffer([](A& a) { return a.buffer(); })
        .def("map", &A::map)
        .def("unmap", &A::unmap)
        .def("unmapRead", &A::unmap_read)
        .def("readCopy", &A::read_copy)
        .def_static("streamCopy", &stream_copy);
}

}  // namespace

PYBIND11_MODULE(_gpu, m)
{
    m.doc() = "fresnel_b200 GPU backend (mirror of fresnel._gpu) over libfrb200";
    py::module_::import("fresnel_b200._common");

    m.def("get_num_available_devices", []() {
        int n = 0;
        check(fr_get_num_available_devices(&n));
        return n;
    });

    py::class_<DeviceH, std::shared_ptr<DeviceH>>(m, "Device")
        .def(py::init<const std::string&, int>())
        .def("describe", &DeviceH::describe)
        .def("synchronize", [](DeviceH& d) { check(fr_device_synchronize(d.dev)); })
        .def("timerStart", [](DeviceH& d) { check(fr_device_timer_start(d.dev)); })
        .def("timerStop", [](DeviceH& d) {
            float ms = 0.0f;
            check(fr_device_timer_stop(d.dev, &ms));
            return ms;
        })
        .def("setProfiling", [](DeviceH& d, bool on) { check(fr_device_set_profiling(d.dev, on)); })
        .def("setOption", [](DeviceH& d, const std::string& name, double v) {
            check(fr_device_set_option(d.dev, name.c_str(), v));
        })
        .def("getOption", [](DeviceH& d, const std::string& name) {
            double v = 0.0;
            check(fr_device_get_option(d.dev, name.c_str(), &v));
            return v;
        })
        .def_static("getAllGPUs", &DeviceH::all_gpus);

    py::class_<SceneH, std::shared_ptr<SceneH>>(m, "Scene")
        .def(py::init<std::shared_ptr<DeviceH>>())
        .def("getAccel",
             [](SceneH& s) {
                 // (grid kind: 0 BVHs, 1 sphere grid, 2 grid over the scene's parts; why no
                 // grid when one was considered) after the last build
                 int grid = 0;
                 char reason[128];
                 check(fr_scene_get_accel(s.scene, &grid, reason, sizeof(reason)));
                 return py::make_tuple(grid, std::string(reason));
             })
        .def("setCamera", [](SceneH& s, const UserCamera& c) { s.camera = c; })
        .def("getCamera", [](SceneH& s) -> UserCamera& { return s.camera; },
             py::return_value_policy::reference_internal)
        .def("getBackgroundColor", [](SceneH& s) { return s.background; })
        .def("setBackgroundColor", [](SceneH& s, const RGBf& c) { s.background = c; })
        .def("getBackgroundAlpha", [](SceneH& s) { return s.background_alpha; })
        .def("setBackgroundAlpha", [](SceneH& s, float a) { s.background_alpha = a; })
        .def("getLights", [](SceneH& s) -> Lights& { return s.lights; },
             py::return_value_policy::reference_internal)
        .def("setLights", [](SceneH& s, const Lights& l) { s.lights = l; })
        .def("debugTraversalCompare", [](SceneH& s, py::array_t<float, py::array::c_style | py::array::forcecast> rays) {
            s.sync();
            uint32_t n = uint32_t(rays.shape(0));
            py::array_t<uint32_t> out({py::ssize_t(n), py::ssize_t(6)});
            check(fr_debug_traversal_compare(s.scene, rays.data(), n, out.mutable_data()));
            return out;
        })
        .def("build", [](SceneH& s) {
            s.sync();
            check(fr_scene_build(s.scene));
        });

    py::class_<GeometryH, std::shared_ptr<GeometryH>>(m, "Geometry")
        .def("getMaterial", &GeometryH::getMaterial)
        .def("setMaterial", &GeometryH::setMaterial)
        .def("getOutlineMaterial", &GeometryH::getOutlineMaterial)
        .def("setOutlineMaterial", &GeometryH::setOutlineMaterial)
        .def("getOutlineWidth", &GeometryH::getOutlineWidth)
        .def("setOutlineWidth", &GeometryH::setOutlineWidth)
        .def("disable", &GeometryH::disable)
        .def("enable", &GeometryH::enable)
        .def("remove", &GeometryH::remove)
        .def("update", &GeometryH::update);

    py::class_<GeometrySphereH, GeometryH, std::shared_ptr<GeometrySphereH>>(m, "GeometrySphere")
        .def(py::init<std::shared_ptr<SceneH>, unsigned>())
        .def("getPositionBuffer", [](GeometrySphereH& g) { return g.position; })
        .def("getRadiusBuffer", [](GeometrySphereH& g) { return g.radius; })
        .def("getColorBuffer", [](GeometrySphereH& g) { return g.color; });

    py::class_<GeometryCylinderH, GeometryH, std::shared_ptr<GeometryCylinderH>>(m,
                                                                                "GeometryCylinder")
        .def(py::init<std::shared_ptr<SceneH>, unsigned>())
        .def("getPointsBuffer", [](GeometryCylinderH& g) { return g.points; })
        .def("getRadiusBuffer", [](GeometryCylinderH& g) { return g.radius; })
        .def("getColorBuffer", [](GeometryCylinderH& g) { return g.color; });

    py::class_<GeometryConvexPolyhedronH, GeometryH, std::shared_ptr<GeometryConvexPolyhedronH>>(
        m, "GeometryConvexPolyhedron")
        .def(py::init<std::shared_ptr<SceneH>, farray, farray, farray, unsigned, float>())
        .def("getPositionBuffer", [](GeometryConvexPolyhedronH& g) { return g.position; })
        .def("getOrientationBuffer", [](GeometryConvexPolyhedronH& g) { return g.orientation; })
        .def("getColorBuffer", [](GeometryConvexPolyhedronH& g) { return g.color; })
        .def("setColorByFace", &GeometryConvexPolyhedronH::setColorByFace)
        .def("getColorByFace", &GeometryConvexPolyhedronH::getColorByFace);

    py::class_<GeometryMeshH, GeometryH, std::shared_ptr<GeometryMeshH>>(m, "GeometryMesh")
        .def(py::init<std::shared_ptr<SceneH>, farray, unsigned>())
        .def("getPositionBuffer", [](GeometryMeshH& g) { return g.position; })
        .def("getOrientationBuffer", [](GeometryMeshH& g) { return g.orientation; })
        .def("getColorBuffer", [](GeometryMeshH& g) { return g.color; });

    py::class_<GeometryPolygonH, GeometryH, std::shared_ptr<GeometryPolygonH>>(m, "GeometryPolygon")
        .def(py::init<std::shared_ptr<SceneH>, farray, float, unsigned>())
        .def("getPositionBuffer", [](GeometryPolygonH& g) { return g.position; })
        .def("getAngleBuffer", [](GeometryPolygonH& g) { return g.angle; })
        .def("getColorBuffer", [](GeometryPolygonH& g) { return g.color; })
        .def("getRadius", &GeometryPolygonH::getRadius);

    py::class_<TracerH, std::shared_ptr<TracerH>>(m, "Tracer")
        .def("render", &TracerH::render)
        .def("resize", &TracerH::resize)
        .def("getSRGBOutputBuffer", [](TracerH& t) { return t.srgb; })
        .def("getLinearOutputBuffer", [](TracerH& t) { return t.linear; })
        .def("enableHighlightWarning", [](TracerH& t, const RGBf& c) {
            t.highlight = true;
            t.highlight_color = c;
        })
        .def("disableHighlightWarning", [](TracerH& t) { t.highlight = false; })
        .def("getSeed", [](TracerH& t) { return t.seed; })
        .def("setSeed", [](TracerH& t, unsigned s) { t.seed = s; })
        .def("getStats", &TracerH::stats)
        .def("resetStats", [](TracerH& t) { check(fr_tracer_reset_stats(t.tracer)); })
        .def("setLinearOutput",
             [](TracerH& t, py::array_t<float, py::array::c_style | py::array::forcecast> a) {
                 // parity hook (no counterpart in the reference): upload an (h, w, 4) linear
                 // RGBA image into the output buffer
                 if (a.ndim() != 3 || a.shape(0) != py::ssize_t(t.h) ||
                     a.shape(1) != py::ssize_t(t.w) || a.shape(2) != 4)
                     throw std::runtime_error("expected a float32 image of shape (h, w, 4)");
                 check(fr_tracer_write_linear(t.tracer, a.data(), size_t(a.size()) * sizeof(float)));
             })
        .def("histogram", [](TracerH& t) {
            // device-side Tracer.histogram counts, [512][4] uint32 (lightness, R, G, B)
            py::array_t<uint32_t> out({py::ssize_t(512), py::ssize_t(4)});
            check(fr_tracer_histogram(t.tracer, out.mutable_data(), 512 * 4 * sizeof(uint32_t)));
            return out;
        });

    py::class_<TracerDirectH, TracerH, std::shared_ptr<TracerDirectH>>(m, "TracerDirect")
        .def(py::init<std::shared_ptr<DeviceH>, unsigned, unsigned>())
        .def("setAntialiasingN", [](TracerDirectH& t, unsigned n) { t.aa_n = n; })
        .def("getAntialiasingN", [](TracerDirectH& t) { return t.aa_n; })
        .def("renderHitIds", &TracerDirectH::render_hit_ids);

    py::class_<TracerPathH, TracerH, std::shared_ptr<TracerPathH>>(m, "TracerPath")
        .def(py::init<std::shared_ptr<DeviceH>, unsigned, unsigned, unsigned>())
        .def("getNumSamples", [](TracerPathH& t) { return t.n_samples; })
        .def("reset", &TracerPathH::reset)
        .def("setLightSamples", [](TracerPathH& t, unsigned n) { t.light_samples = n; })
        .def("renderSamples", &TracerPathH::render_samples)
        .def("renderSamplesStatic", &TracerPathH::render_samples_static)
        .def("primaryHits", [](TracerPathH& t) {
            py::array_t<uint32_t> out({py::ssize_t(t.h), py::ssize_t(t.w), py::ssize_t(2)});
            check(fr_tracer_read_primary_hits(t.tracer, out.mutable_data(), size_t(t.w) * t.h * 8));
            return out;
        });

    py::class_<BatchH, std::shared_ptr<BatchH>>(m, "Batch")
        .def(py::init<std::shared_ptr<DeviceH>>())
        .def("add", &BatchH::add)
        .def("render", &BatchH::render)
        .def("clear", &BatchH::clear)
        .def("getStats", &BatchH::stats)
        .def("reserve", [](BatchH& b, size_t slots) { check(fr_batch_reserve(b.batch, slots)); })
        .def("__len__", [](const BatchH& b) { return b.items.size(); });

    export_array<ArrayRGBAf>(m, "ArrayRGBAf");
    export_array<ArrayRGBAc>(m, "ArrayRGBAc");
    export_array<ArrayRGBf>(m, "ArrayRGBf");
    export_array<ArrayVec3f>(m, "ArrayVec3f");
    export_array<ArrayQuat3f>(m, "ArrayQuat3f");
    export_array<Array_f>(m, "Array_f");
    export_array<ArrayVec2f>(m, "ArrayVec2f");
    export_array<ArrayRGBc>(m, "ArrayRGBc");
}
