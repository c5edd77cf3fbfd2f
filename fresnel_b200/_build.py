"""Build the native parts of fresnel_b200 in place.

  fresnel_b200/libfrb200.so          CUDA kernels + C ABI (nvcc, sm_100a)
  fresnel_b200/_common<EXT_SUFFIX>   value types (pybind11)
  fresnel_b200/_gpu<EXT_SUFFIX>      backend classes over the C ABI (pybind11)

Device code is compiled with -fmad=false so that every multiply and add in the intersection and
shading arithmetic rounds exactly as the reference's host build does; the few places that want
a fused multiply-add (the BVH slab test) call fmaf explicitly.  Division and square root keep
nvcc's IEEE defaults (no fast math).
"""
import concurrent.futures
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
REPO = os.path.dirname(HERE)
INCLUDE = os.path.join(REPO, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
EXT = sysconfig.get_config_var("EXT_SUFFIX")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "-fmad=false", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC,
    "-Xptxas", "-warn-spills",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fvisibility=hidden",
             "-Wall", "-Wno-unused-function"]


def _cuda_sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC)
           if f.endswith((".h", ".hpp", ".cuh"))]
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def _pybind_includes():
    import pybind11
    return ["-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"]]


def build(verbose=False, force=False):
    """Compile everything that is out of date.  Returns the list of produced libraries."""
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = _headers()
    lib = os.path.join(HERE, "libfrb200.so")
    objs = []
    jobs = []
    for src in _cuda_sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([NVCC, *NVCC_FLAGS, "-c", src, "-o", obj])
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    if objs and (force or jobs or _stale(lib, objs)):
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", lib], verbose)

    out = [lib]
    common = os.path.join(HERE, "_common" + EXT)
    src = os.path.join(CSRC, "py_common.cpp")
    if force or _stale(common, [src] + headers):
        _run(["g++", *CXX_FLAGS, "-shared", *_pybind_includes(), "-I", INCLUDE, src, "-o",
              common], verbose)
    out.append(common)

    gpu = os.path.join(HERE, "_gpu" + EXT)
    src = os.path.join(CSRC, "py_gpu.cpp")
    if force or _stale(gpu, [src, lib] + headers):
        _run(["g++", *CXX_FLAGS, "-shared", *_pybind_includes(), "-I", INCLUDE, src, "-o", gpu,
              "-L", HERE, "-lfrb200", "-Wl,-rpath,$ORIGIN"], verbose)
    out.append(gpu)
    return out


if __name__ == "__main__":
    for p in build(verbose="-v" in sys.argv, force="--force" in sys.argv):
        print(p)
