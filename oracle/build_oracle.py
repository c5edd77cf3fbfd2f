"""Build the CPU oracle (TEST INFRASTRUCTURE; never part of the product).

Outputs
  oracle/_build/liboracle.so      restated math (oracle/restated_math.hpp)
  oracle/_ref/libfresnel_ref.so   the reference's own fresnel/common/*.h math, compiled from the
                                  reference tree when it is present
  oracle/_ref/fresnel_src/        the reference's Python package and test suite, copied
                                  unmodified from the reference tree when it is present
                                  (oracle/reference_package.py)

Both are compiled with g++ -O3 -ffp-contract=off so that no fused multiply-add changes a rounding
the reference does not make.  Run ``python oracle/build_oracle.py``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REFERENCE = os.environ.get("FRESNEL_REFERENCE", "/root/reference")

CXXFLAGS = [
    "-O3", "-std=c++17", "-fPIC", "-shared", "-march=x86-64-v3", "-ffp-contract=off",
    "-fno-math-errno", "-pthread", "-Wall", "-Wno-unused-function",
]

SOURCES = [os.path.join(HERE, "oracle_core.cpp")]
DEPS = SOURCES + [os.path.join(HERE, f) for f in
                  ("oracle.h", "restated_math.hpp", "ref_math_adapter.hpp")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def reference_available():
    return os.path.isfile(os.path.join(REFERENCE, "fresnel", "common", "Camera.h"))


def build(verbose=False, force=False):
    """Compile the oracle libraries; returns the list of built paths."""
    out = []
    lib = os.path.join(HERE, "_build", "liboracle.so")
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    if force or _stale(lib, DEPS):
        _run(["g++", *CXXFLAGS, "-I", HERE, *SOURCES, "-o", lib], verbose)
    out.append(lib)
    if reference_available():
        ref = os.path.join(HERE, "_ref", "libfresnel_ref.so")
        os.makedirs(os.path.dirname(ref), exist_ok=True)
        if force or _stale(ref, DEPS):
            # -w: the reference headers leave some outputs unset on paths they never take
            _run(["g++", *CXXFLAGS, "-w", "-DFR_ORACLE_REFERENCE_MATH",
                  "-I", HERE, "-I", os.path.join(HERE, "ref_shim"),
                  "-I", os.path.join(REFERENCE, "fresnel"),
                  "-I", os.path.join(REFERENCE, "fresnel", "common"),
                  *SOURCES, "-o", ref], verbose)
        out.append(ref)
        sys.path.insert(0, REPO)
        from oracle import reference_package
        staged = reference_package.stage(verbose)
        if staged:
            out.append(staged)
    return out


if __name__ == "__main__":
    for p in build(verbose=True, force="--force" in sys.argv):
        print(p)
