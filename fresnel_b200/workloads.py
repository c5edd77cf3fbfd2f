"""Synthetic scenes for the benchmark configurations and the parity tests.

The reference publishes no benchmark data; these seeded generators stand in for the scenes its
benchmark configurations describe (uniformly placed spheres at a given density, bonds between
neighbours, randomly oriented cubes, icosahedron instances).  Every builder takes a fresnel-API
``device`` and builds the scene with the API of the package that device belongs to: this
package on the GPU engine or the CPU oracle, or fresnel's own Python package (whose scenes the
reference's CPU path renders).  The module imports nothing of its package at load time, so it
can be loaded on its own by file path.
"""

import math
import sys

import numpy


class _Api:
    """The fresnel-API modules of the package that ``device`` belongs to (the package that
    defines its class: fresnel_b200 or fresnel)."""

    def __init__(self, device):
        pkg = sys.modules[type(device).__module__.split(".")[0]]
        self.Scene = pkg.Scene
        self.camera, self.color, self.geometry = pkg.camera, pkg.color, pkg.geometry
        self.light, self.material = pkg.light, pkg.material


def perspective_fit(scene, focal_length=0.5):
    """Perspective camera framing the scene like ``Orthographic.fit``: same position, look_at
    and up; the image-plane height at the focus distance equals the orthographic height."""
    api = _Api(scene.device)
    ortho = api.camera.Orthographic.fit(scene)
    d = float(numpy.linalg.norm(ortho.position - ortho.look_at))
    return api.camera.Perspective(position=ortho.position, look_at=ortho.look_at, up=ortho.up,
                                  focal_length=focal_length, focus_distance=d, f_stop=math.inf,
                                  height=focal_length * ortho.height / d)


def hex_spheres(device):
    """Six spheres on a hexagon with outlines (the reference test fixture scene)."""
    api = _Api(device)
    t1, p1 = 70 * math.pi / 180, 45 * math.pi / 180
    t2, p2 = math.pi / 2, -math.pi / 4
    lights = [api.light.Light(direction=(math.sin(t1) * math.sin(p1), math.cos(t1),
                                         math.sin(t1) * math.cos(p1)),
                              color=(0.75, 0.75, 0.75), theta=math.pi / 8),
              api.light.Light(direction=(math.sin(t2) * math.sin(p2), math.cos(t2),
                                         math.sin(t2) * math.cos(p2)),
                              color=(0.1, 0.1, 0.1), theta=math.pi / 2)]
    scene = api.Scene(device, lights=lights)
    pos = [[2 * math.cos(i * 2 * math.pi / 6), 2 * math.sin(i * 2 * math.pi / 6), 0]
           for i in range(6)]
    g = api.geometry.Sphere(scene, position=pos, radius=1.0)
    g.material = api.material.Material(solid=0.0, color=api.color.linear([1, 0.874, 0.169]))
    g.outline_width = 0.12
    scene.camera = api.camera.Orthographic(position=(0, 0, 10), look_at=(0, 0, 0), up=(0, 1, 0),
                                           height=6)
    return scene


def random_spheres(device, n, box, radius=0.5, seed=0, colors=False, outline_width=0.0,
                   mat=None, lights=None, perspective=True):
    """n spheres uniform in a cube of side ``box`` (float32, numpy default_rng(seed))."""
    api = _Api(device)
    rng = numpy.random.default_rng(seed)
    pos = rng.uniform(-box / 2, box / 2, (n, 3)).astype(numpy.float32)
    scene = api.Scene(device, lights=lights if lights is not None else api.light.cloudy())
    g = api.geometry.Sphere(scene, position=pos, radius=radius, outline_width=outline_width)
    if colors:
        g.color[:] = rng.uniform(0, 1, (n, 3)).astype(numpy.float32)
    g.material = mat if mat is not None else api.material.Material(
        color=api.color.linear((0.1, 0.8, 0.1)), roughness=0.8, specular=0.2)
    scene.camera = perspective_fit(scene) if perspective else api.camera.Orthographic.fit(scene)
    return scene


def config1(device):
    """1000 spheres r=0.5 in a cube of side 20, outline 0.1, cloudy lights (580x580, 64 spp,
    32 light samples in the benchmark)."""
    api = _Api(device)
    return random_spheres(device, 1000, 20.0, 0.5, seed=0, outline_width=0.1,
                          mat=api.material.Material(color=api.color.linear((0.1, 0.8, 0.1)),
                                                    roughness=0.8, specular=0.2))


def config2(device, n=1_000_000, box=140.0):
    """1M spheres r=0.5 in a cube of side 140 with per-particle colours, lightbox
    (1920x1080, 256 spp, 1 light sample in the benchmark).  ``n``/``box`` scale it down at the
    same density for tests."""
    api = _Api(device)
    return random_spheres(device, n, box, 0.5, seed=1, colors=True,
                          mat=api.material.Material(roughness=0.4, metal=0.0, specular=0.5,
                                                    primitive_color_mix=1.0),
                          lights=api.light.lightbox())


def icosahedron(circumradius=0.5):
    """20 triangles (60 vertices, counter-clockwise seen from outside) of a regular icosahedron."""
    p = (1 + math.sqrt(5)) / 2
    v = numpy.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p],
                     [0, -1, -p], [0, 1, -p], [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]],
                    dtype=numpy.float64)
    v *= circumradius / numpy.linalg.norm(v[0])
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    tri = numpy.array([[v[a], v[b], v[c]] for a, b, c in faces])
    # orient every face counter-clockwise seen from outside
    for t in tri:
        n = numpy.cross(t[1] - t[0], t[2] - t[0])
        if numpy.dot(n, t.mean(axis=0)) < 0:
            t[[1, 2]] = t[[2, 1]]
    return tri.reshape(-1, 3).astype(numpy.float32)


def unit_cube_planes():
    """Face planes of a unit cube centred at the origin (radius sqrt(3)/2)."""
    origins, normals = [], []
    for k in range(3):
        for s in (-1, 1):
            n = [0, 0, 0]
            n[k] = s
            o = [0, 0, 0]
            o[k] = 0.5 * s
            origins.append(o)
            normals.append(n)
    return {'face_origin': numpy.array(origins, numpy.float32),
            'face_normal': numpy.array(normals, numpy.float32),
            'face_color': numpy.full((6, 3), 0.9, numpy.float32),
            'radius': math.sqrt(3) / 2}


def random_quaternions(rng, n):
    q = rng.normal(size=(n, 4))
    q /= numpy.linalg.norm(q, axis=1, keepdims=True)
    return q.astype(numpy.float32)


def bonds(rng, pos, n_bonds, cutoff=1.5):
    """Pairs (i, j) with |p_i - p_j| < cutoff, i drawn uniformly (scipy cKDTree)."""
    from scipy.spatial import cKDTree
    tree = cKDTree(pos)
    out = []
    tries = 0
    while len(out) < n_bonds and tries < 50 * n_bonds:
        tries += 1
        i = int(rng.integers(len(pos)))
        nb = [j for j in tree.query_ball_point(pos[i], cutoff) if j != i]
        if nb:
            out.append((i, nb[int(rng.integers(len(nb)))]))
    return numpy.array(out, dtype=numpy.int64).reshape(-1, 2)


# the concave pentagon of fresnel's polygon tests, counter-clockwise
POLYGON_OUTLINE = [[-1, -1], [1, -1], [1, 1], [0, 0], [-1, 1]]


def polygons(device, nx=20, ny=15, spacing=2.5, rounding_radius=0.15, seed=5, spheres=0,
             perspective=True):
    """nx*ny rounded concave pentagons (half size of fresnel's test shape) on a jittered grid in
    the z = 0 plane, random angles and colours, outlined; optionally ``spheres`` spheres floating
    above the plane (a scene of two geometry types, traced through one combined tree)."""
    api = _Api(device)
    rng = numpy.random.default_rng(seed)
    gx, gy = numpy.meshgrid(numpy.arange(nx) - (nx - 1) / 2, numpy.arange(ny) - (ny - 1) / 2)
    pos = numpy.stack([gx.ravel(), gy.ravel()], axis=1) * spacing
    pos += rng.uniform(-0.2, 0.2, pos.shape)
    n = len(pos)
    scene = api.Scene(device, lights=api.light.rembrandt())
    g = api.geometry.Polygon(scene, vertices=numpy.array(POLYGON_OUTLINE, numpy.float32) * 0.5,
                             position=pos.astype(numpy.float32),
                             angle=rng.uniform(-math.pi, math.pi, n).astype(numpy.float32),
                             color=rng.uniform(0, 1, (n, 3)).astype(numpy.float32),
                             rounding_radius=rounding_radius, outline_width=0.05)
    g.material = api.material.Material(roughness=0.5, specular=0.3, primitive_color_mix=1.0)
    if spheres:
        sp = numpy.column_stack([rng.uniform(-nx, nx, spheres), rng.uniform(-ny, ny, spheres),
                                 rng.uniform(0.8, 4.0, spheres)]) * numpy.array([spacing / 2,
                                                                                 spacing / 2, 1])
        api.geometry.Sphere(scene, position=sp.astype(numpy.float32), radius=0.6,
                            material=api.material.Material(color=api.color.linear((0.9, 0.6, 0.2)),
                                                           roughness=0.3))
    if perspective:
        scene.camera = api.camera.Perspective(position=(0, -1.1 * ny * spacing, 0.9 * ny * spacing),
                                              look_at=(0, 0, 0), up=(0, 0, 1), focal_length=0.5,
                                              height=0.35)
    else:
        scene.camera = api.camera.Orthographic(position=(0, 0, 10), look_at=(0, 0, 0), up=(0, 1, 0),
                                               height=ny * spacing)
    return scene


def config3(device, scale=1.0, box=100.0):
    """Mixed scene: 200k spheres (r log-uniform in [0.3, 0.7]), 50k bonds (r = 0.1), 20k unit
    cubes and 10k icosahedra in a cube of side 100 (1280x720, 128 spp in the benchmark).
    ``scale`` shrinks every count (and the box at constant density) for tests."""
    api = _Api(device)
    rng = numpy.random.default_rng(2)
    L = box * scale**(1 / 3)
    ns, nb, nc, nm = (max(1, int(round(x * scale))) for x in (200_000, 50_000, 20_000, 10_000))
    scene = api.Scene(device, lights=api.light.rembrandt())
    pos = rng.uniform(-L / 2, L / 2, (ns, 3)).astype(numpy.float32)
    rad = numpy.exp(rng.uniform(math.log(0.3), math.log(0.7), ns)).astype(numpy.float32)
    api.geometry.Sphere(scene, position=pos, radius=rad, color=(0.6, 0.6, 0.6))
    pairs = bonds(rng, pos, nb)
    if len(pairs):
        pts = numpy.stack([pos[pairs[:, 0]], pos[pairs[:, 1]]], axis=1)
        api.geometry.Cylinder(scene, points=pts, radius=0.1, color=(0.3, 0.3, 0.8))
    cpos = rng.uniform(-L / 2, L / 2, (nc, 3)).astype(numpy.float32)
    poly = api.geometry.ConvexPolyhedron(scene, unit_cube_planes(), position=cpos,
                                         orientation=random_quaternions(rng, nc),
                                         color=(0.8, 0.3, 0.2))
    poly.material = api.material.Material(color=(0.8, 0.3, 0.2), metal=0.5, roughness=0.3)
    mpos = rng.uniform(-L / 2, L / 2, (nm, 3)).astype(numpy.float32)
    verts = icosahedron(0.5)
    api.geometry.Mesh(scene, verts, position=mpos, orientation=random_quaternions(rng, nm),
                      color=numpy.full((len(verts), 3), 0.7, numpy.float32))
    scene.camera = perspective_fit(scene)
    return scene


def config4(device, n_frames=64, seed=3):
    """Trajectory-style frame set: ``n_frames`` independent scenes of the 1M-sphere scene's
    density (1e6 spheres per 140^3), sphere count log-uniform in [1e4, 5e5], r = 0.5, per-particle
    colours, the 1M-sphere scene's material and lights; each frame's resolution drawn from
    512x512, 768x768, 1024x1024 (16 spp, 1 light sample in the benchmark).  Returns a list of
    (scene, width, height)."""
    api = _Api(device)
    rng = numpy.random.default_rng(seed)
    rho = 1e6 / 140.0**3
    frames = []
    for _ in range(n_frames):
        n = int(round(math.exp(rng.uniform(math.log(1e4), math.log(5e5)))))
        box = (n / rho) ** (1.0 / 3.0)
        res = (512, 768, 1024)[int(rng.integers(3))]
        scene = random_spheres(device, n, box, 0.5, seed=int(rng.integers(1 << 31)), colors=True,
                               mat=api.material.Material(roughness=0.4, metal=0.0, specular=0.5,
                                                         primitive_color_mix=1.0),
                               lights=api.light.lightbox())
        frames.append((scene, res, res))
    return frames


def near_bonds(rng, pos, n_bonds, cutoff=1.5):
    """n_bonds pairs (i, j), i uniform, j a uniformly chosen other sphere within ``cutoff`` of i
    (vectorised over candidates with scipy's cKDTree; spheres without a neighbour are redrawn)."""
    from scipy.spatial import cKDTree
    if n_bonds <= 0 or len(pos) < 2:
        return numpy.zeros((0, 2), numpy.int64)
    tree = cKDTree(pos)
    k = min(3, len(pos))
    out = []
    have = 0
    for _ in range(20):
        cand = rng.integers(len(pos), size=int((n_bonds - have) * 1.5) + 16)
        d, idx = tree.query(pos[cand], k=k, workers=-1)
        valid = (d < cutoff) & (idx != cand[:, None]) & (idx < len(pos))
        pick = numpy.argmax(rng.random(valid.shape) * valid, axis=1)
        ok = valid[numpy.arange(len(cand)), pick]
        pairs = numpy.stack([cand[ok], idx[numpy.arange(len(cand)), pick][ok]], axis=1)
        out.append(pairs[:n_bonds - have])
        have += len(out[-1])
        if have >= n_bonds:
            break
    return numpy.concatenate(out).astype(numpy.int64)


def serving_scene(device, n_prims, seed):
    """A serving-request scene of ``n_prims`` primitives: 80% spheres at the mixed scene's
    density (0.2 per unit volume) and radii (log-uniform in [0.3, 0.7]), 20% bonds (r = 0.1)
    between neighbouring spheres; per-sphere colours, the 1M-sphere scene's material, lightbox
    lights, perspective camera fit to the scene."""
    api = _Api(device)
    rng = numpy.random.default_rng(seed)
    ns = max(1, int(round(0.8 * n_prims)))
    nb = max(0, int(n_prims) - ns)
    box = (ns / 0.2) ** (1.0 / 3.0)
    pos = rng.uniform(-box / 2, box / 2, (ns, 3)).astype(numpy.float32)
    rad = numpy.exp(rng.uniform(math.log(0.3), math.log(0.7), ns)).astype(numpy.float32)
    scene = api.Scene(device, lights=api.light.lightbox())
    g = api.geometry.Sphere(scene, position=pos, radius=rad)
    g.color[:] = rng.uniform(0, 1, (ns, 3)).astype(numpy.float32)
    g.material = api.material.Material(roughness=0.4, metal=0.0, specular=0.5,
                                       primitive_color_mix=1.0)
    pairs = near_bonds(rng, pos, nb)
    if len(pairs):
        pts = numpy.stack([pos[pairs[:, 0]], pos[pairs[:, 1]]], axis=1)
        api.geometry.Cylinder(scene, points=pts, radius=0.1, color=(0.3, 0.3, 0.8))
    scene.camera = perspective_fit(scene)
    return scene


def serving_scene_bytes(n_prims):
    """Device bytes of a serving scene (arrays, leaf records, binary and 4-wide BVH nodes)."""
    return int(160 * 0.8 * n_prims + 200 * 0.2 * n_prims) + (1 << 16)


SERVING_RESOLUTIONS = ((256, 256), (640, 480), (1280, 720), (1920, 1080))


def config5(rate, n_requests, n_scenes=32, seed=4):
    """Serving trace: ``n_requests`` Poisson arrivals at ``rate`` per second.  Each request picks
    a scene key (with probability 0.5, or once all ``n_scenes`` keys are in use, one already
    used; else the next new key), a resolution uniformly from SERVING_RESOLUTIONS and a sample
    count round(exp(U(0, ln 64))).  Scene key k has round(exp(U(ln 1e3, ln 2e6))) primitives,
    the same for every rate.  Returns (requests, {key: n_prims})."""
    from .serving import Request, log_uniform_int, poisson_arrivals
    srng = numpy.random.default_rng(seed)
    sizes = {k: log_uniform_int(srng, 1e3, 2e6) for k in range(n_scenes)}
    rng = numpy.random.default_rng([seed, int(round(rate * 1000))])
    arrivals = poisson_arrivals(rate, n_requests, rng)
    used = []
    out = []
    for n, t in enumerate(arrivals):
        if used and (len(used) == n_scenes or rng.random() < 0.5):
            key = used[int(rng.integers(len(used)))]
        else:
            key = len(used)
            used.append(key)
        w, h = SERVING_RESOLUTIONS[int(rng.integers(len(SERVING_RESOLUTIONS)))]
        spp = max(1, int(round(math.exp(rng.uniform(0.0, math.log(64.0))))))
        out.append(Request(key, w, h, spp, seed=1000 + n, arrival=float(t), tag=n))
    return out, sizes


def serving_scene_first(device):
    """The first scene of the serving trace (its per-ray cost stands for the trace's on the CPU):
    config5's scene key 0, round(exp(U(ln 1e3, ln 2e6))) primitives from the trace's seed."""
    srng = numpy.random.default_rng(4)
    n = int(round(math.exp(srng.uniform(math.log(1e3), math.log(2e6)))))
    return serving_scene(device, n, seed=4000)
