"""How many exact sphere tests a warp-shared cone cull would leave in the camera pass of the
1M-sphere 1080p frame (TEST INFRASTRUCTURE: a CPU estimate, not part of the product).

The engine's camera kernel traces the 32 anti-aliasing samples of one pixel in one warp, through
the uniform sphere grid (1.5 cells per sphere over the spheres' bounds, the walk stopping once
the closest hit lies before the current cell's exit).  This script walks the same grid on the
CPU in double precision for the camera rays of random pixels (pinhole camera of the benchmark
scene, fresnel's tent-filtered jitter of width 0.707 pixels, Camera.h:169-269) and reports per
camera ray the spheres tested now (S), the spheres that survive a conservative cull against the
pixel's ray cone (S_cull: the angle between the cone's axis and the sphere's centre at most the
cone's half-angle plus the sphere's angular radius), the tests left when only the steps of a
warp-synchronous walk whose walking lanes all stand in one cell are culled (S_hybrid; the share
of such steps is coop_step_frac), and per warp the references held by the cells its rays visit
(U_refs) and the passes of one reference per lane that culling every distinct cell of every
step would take (cull_rounds: lanes grouped by cell with __match_any_sync).  The look-ahead form
gathers each walking lane's next BATCH cells into one batch, culls the batch's distinct cells in
batch_passes passes and leaves S_batch exact tests per ray (S_batch_max for the warp's
longest).  The hit sphere of every ray is checked to survive the cull.

Run: python oracle/cone_cull_estimate.py [n_pixels]   (default 400)
"""

import json
import math
import os
import sys

import numpy

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

AA_WIDTH = 0.707106781  # Camera.h: importanceSampleAA's tent scaled to this half-width
TNEAR = 1e-5
BATCH = 3  # cells per lane gathered into one cull batch (look-ahead form)
AHEAD = BATCH - 1


class SphereGrid:
    """Uniform grid over sphere bounds, cells in x-fastest order with their sphere lists."""

    def __init__(self, pos, r, cells_per_sphere=1.5):
        n = len(pos)
        self.pos, self.r = pos, r
        self.lo, self.hi = pos.min(0) - r, pos.max(0) + r
        ext = self.hi - self.lo
        h = (ext.prod() / (cells_per_sphere * n)) ** (1.0 / 3.0)
        self.dims = numpy.ceil(ext / h).astype(numpy.int64)
        self.cell = ext / self.dims
        c0 = numpy.floor((pos - r - self.lo) / self.cell).astype(numpy.int64).clip(0, self.dims - 1)
        c1 = numpy.floor((pos + r - self.lo) / self.cell).astype(numpy.int64).clip(0, self.dims - 1)
        span = c1 - c0 + 1
        cnt = span.prod(1)
        owner = numpy.repeat(numpy.arange(n), cnt)
        first = numpy.concatenate([[0], numpy.cumsum(cnt)[:-1]])
        k = numpy.arange(cnt.sum()) - numpy.repeat(first, cnt)
        sx, sy = numpy.repeat(span[:, 0], cnt), numpy.repeat(span[:, 1], cnt)
        ix = numpy.repeat(c0[:, 0], cnt) + k % sx
        iy = numpy.repeat(c0[:, 1], cnt) + (k // sx) % sy
        iz = numpy.repeat(c0[:, 2], cnt) + k // (sx * sy)
        cid = (iz * self.dims[1] + iy) * self.dims[0] + ix
        order = numpy.argsort(cid, kind="stable")
        self.refs = owner[order]
        self.start = numpy.searchsorted(cid[order], numpy.arange(self.dims.prod() + 1))
        self.refs_per_sphere = float(cnt.mean())

    def walk(self, o, d, ahead=0):
        """(cells visited, spheres tested in order, closest hit or -1) of the ray o + t d, and the
        up to `ahead` cells the DDA would reach after the stop (inside the grid)."""
        with numpy.errstate(divide="ignore"):
            inv = numpy.where(d != 0, 1.0 / numpy.where(d != 0, d, 1.0), numpy.inf)
        t0, t1 = (self.lo - o) * inv, (self.hi - o) * inv
        t_in = max(numpy.minimum(t0, t1).max(), 0.0)
        t_out = numpy.maximum(t0, t1).min()
        if not t_in <= t_out:
            return [], [], -1, []
        c = numpy.clip(numpy.floor((o + t_in * d - self.lo) / self.cell).astype(numpy.int64), 0,
                       self.dims - 1)
        step = numpy.where(d >= 0, 1, -1)
        t_next = numpy.array([(self.lo[a] + (c[a] + (d[a] >= 0)) * self.cell[a] - o[a]) * inv[a]
                              for a in range(3)])
        t_delta = numpy.abs(self.cell * inv)
        best, hit, tested, cells = numpy.inf, -1, [], []
        while True:
            ci = int((c[2] * self.dims[1] + c[1]) * self.dims[0] + c[0])
            cells.append(ci)
            for s in self.refs[self.start[ci]:self.start[ci + 1]]:
                s = int(s)
                tested.append(s)
                v = self.pos[s] - o
                b = v @ d
                det = b * b - v @ v + self.r * self.r
                if det >= 0:
                    t = b - math.sqrt(det)
                    if t <= TNEAR:
                        t = b + math.sqrt(det)
                    if TNEAR < t < best or (t == best and s < hit):
                        best, hit = t, s
            a = int(numpy.argmin(t_next))
            if best <= t_next[a] or t_next[a] >= t_out:
                break
            c[a] += step[a]
            if not 0 <= c[a] < self.dims[a]:
                return cells, tested, hit, []
            t_next[a] += t_delta[a]
        extra = []
        while len(extra) < ahead:
            a = int(numpy.argmin(t_next))
            if t_next[a] >= t_out:
                break
            c[a] += step[a]
            if not 0 <= c[a] < self.dims[a]:
                break
            t_next[a] += t_delta[a]
            extra.append(int((c[2] * self.dims[1] + c[1]) * self.dims[0] + c[0]))
        return cells, tested, hit, extra


def _kept(keep, s, pos, p, axis, half, r):
    """Whether sphere s survives the cull against the cone (p, axis, half-angle); memoised."""
    if s not in keep:
        q = pos[s] - p
        dist = numpy.linalg.norm(q)
        ang = math.acos(max(-1.0, min(1.0, float(q @ axis) / dist)))
        keep[s] = ang <= half + math.asin(min(1.0, r / dist)) + 1e-6
    return keep[s]


def _tent(u):
    r = 2.0 * u
    return numpy.where(r < 1.0, numpy.sqrt(r) - 1.0, 1.0 - numpy.sqrt(2.0 - r))


def estimate(n_pixels=400, seed=7):
    import bench
    from oracle import cpu_module
    wl = bench.WORKLOADS["c2"]
    dev = cpu_module.make_device("restated")
    scene = wl.build(dev)
    g = scene.geometry[0]
    pos = numpy.asarray(g.position[:], numpy.float64)
    r = float(numpy.asarray(g.radius[:])[0])
    grid = SphereGrid(pos, r)
    cam = scene.camera
    p = numpy.array(cam.position, numpy.float64)
    fwd = numpy.array(cam.look_at, numpy.float64) - p
    fwd /= numpy.linalg.norm(fwd)
    u = numpy.cross(fwd, numpy.array(cam.up, numpy.float64))
    u /= numpy.linalg.norm(u)
    v = numpy.cross(u, fwd)
    scale = float(cam.height) / float(cam.focal_length)
    w, h = wl.w, wl.h

    def ray(i, j, dx, dy):  # generateRay (Camera.h) for a pinhole: origin p for every sample
        ys = -((j + 0.5 + dy * AA_WIDTH) / h - 0.5)
        xs = (i + 0.5 + dx * AA_WIDTH) / h - 0.5 * w / h
        d = fwd + (ys * v + xs * u) * scale
        return d / numpy.linalg.norm(d)

    rng = numpy.random.default_rng(seed)
    per_ray = {"S": [], "S_cull": [], "S_hybrid": [], "S_batch": [], "cells": [], "hit": []}
    per_warp = {"U_refs": [], "U_cells": [], "S_max": [], "S_cull_max": [], "coop_step_frac": [],
                "cull_rounds": [], "batch_passes": [], "S_batch_max": []}
    for _ in range(n_pixels):
        i, j = int(rng.integers(0, w)), int(rng.integers(0, h))
        dirs = numpy.array([ray(i, j, dx, dy) for dx, dy in
                            zip(_tent(rng.uniform(0, 1, 32)), _tent(rng.uniform(0, 1, 32)))])
        axis = dirs.mean(0)
        axis /= numpy.linalg.norm(axis)
        half = float(numpy.arccos(numpy.clip(dirs @ axis, -1.0, 1.0)).max())
        walks4 = [grid.walk(p, d, AHEAD) for d in dirs]
        walks = [x[:3] for x in walks4]
        cells = set(c for cl, _, _ in walks for c in cl)
        per_warp["U_cells"].append(len(cells))
        per_warp["U_refs"].append(sum(int(grid.start[c + 1] - grid.start[c]) for c in cells))
        keep = {}
        s_all, s_cull = [], []
        for cl, tested, hit in walks:
            kept = sum(1 for x in tested if _kept(keep, x, pos, p, axis, half, r))
            if hit >= 0 and not keep[hit]:
                raise AssertionError("the cull dropped a ray's hit sphere")
            s_all.append(len(tested))
            s_cull.append(kept)
            per_ray["cells"].append(len(cl))
            per_ray["hit"].append(hit >= 0)
        # warp-synchronous walk: a step whose walking lanes all stand in one cell is culled once
        # for the warp; any other step keeps every lane's own tests
        steps = max(len(cl) for cl, _, _ in walks)
        hybrid = [0] * len(walks)
        coop = rounds = 0
        for k in range(steps):
            here = {cl[k] for cl, _, _ in walks if len(cl) > k}
            for lane, (cl, _, _) in enumerate(walks):
                if len(cl) <= k:
                    continue
                refs = grid.refs[grid.start[cl[k]]:grid.start[cl[k] + 1]]
                if len(here) == 1:
                    hybrid[lane] += sum(1 for x in refs if _kept(keep, int(x), pos, p, axis, half, r))
                else:
                    hybrid[lane] += len(refs)
            coop += len(here) == 1
            rounds += sum(-(-int(grid.start[c + 1] - grid.start[c]) // 32) for c in here)
        # look-ahead form: every walking lane contributes its next BATCH cells (past its stop in
        # its last batch), the batch's distinct cells are culled in passes of one reference per
        # lane, and each lane exact-tests the survivors of its own batch cells
        n_batches = max(-(-len(cl) // BATCH) for cl, _, _ in walks) if steps else 0
        passes = 0
        batch_tests = [0] * len(walks)
        for b in range(n_batches):
            distinct = set()
            for lane, (cl, _, _, extra) in enumerate(walks4):
                if len(cl) <= b * BATCH:
                    continue
                mine = (cl + extra)[b * BATCH:(b + 1) * BATCH]
                distinct.update(mine)
                batch_tests[lane] += sum(
                    1 for c in mine for x in grid.refs[grid.start[c]:grid.start[c + 1]]
                    if _kept(keep, int(x), pos, p, axis, half, r))
            passes += -(-sum(int(grid.start[c + 1] - grid.start[c]) for c in distinct) // 32)
        per_warp["batch_passes"].append(passes)
        per_warp["S_batch_max"].append(max(batch_tests))
        per_ray["S_batch"] += batch_tests
        per_warp["coop_step_frac"].append(coop / steps if steps else 1.0)
        per_warp["cull_rounds"].append(rounds)
        per_ray["S_hybrid"] += hybrid
        per_ray["S"] += s_all
        per_ray["S_cull"] += s_cull
        per_warp["S_max"].append(max(s_all))
        per_warp["S_cull_max"].append(max(s_cull))
    out = {k: round(float(numpy.mean(x)), 3) for k, x in {**per_ray, **per_warp}.items()}
    out.update(pixels=n_pixels, rays=32 * n_pixels, grid=[int(x) for x in grid.dims],
               refs_per_sphere=round(grid.refs_per_sphere, 3))
    return out


if __name__ == "__main__":
    print(json.dumps(estimate(int(sys.argv[1]) if len(sys.argv) > 1 else 400)))
