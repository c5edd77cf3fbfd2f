"""Run fresnel's own test suite against the CPU oracle (test infrastructure).

Builds a temporary ``fresnel`` package whose pure-Python modules are the reference's own files
(symlinked, unmodified) and whose compiled backends are replaced by
  _common  -> fresnel_b200._common with cpu_built() True and gpu_built() False
  _cpu     -> oracle.cpu_module (restated or reference-header math)
so that ``pytest <reference>/fresnel/test`` renders every scene with the oracle and compares it
with the reference's golden PNGs.  Needs the reference tree (FRESNEL_REFERENCE, default
/root/reference); the GPU box does not have it, so callers skip when it is absent.
"""

import os
import subprocess
import sys
import tempfile

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = os.environ.get("FRESNEL_REFERENCE", "/root/reference")
PKG = os.path.join(REFERENCE, "fresnel")

# Reference test files left out of the overlay run (none: every geometry is implemented).
EXCLUDED_TESTS = []

_COMMON_SHIM = """from fresnel_b200._common import *  # noqa: F401,F403
from fresnel_b200._common import find_polyhedron_faces  # noqa: F401


def cpu_built():
    return True


def gpu_built():
    return False
"""

_CPU_SHIM = """import sys
sys.path.insert(0, {repo!r})
from oracle import cpu_module as _m
from oracle.cpu_module import *  # noqa: F401,F403


class Device(_m.Device):
    kind = {kind!r}
"""


def available():
    return os.path.isfile(os.path.join(PKG, "__init__.py"))


def make_overlay(root, kind="restated"):
    """Create <root>/fresnel (overlay package) and <root>/test (links to the reference tests)."""
    pkg = os.path.join(root, "fresnel")
    os.makedirs(pkg)
    for name in os.listdir(PKG):
        if name.endswith(".py"):
            os.symlink(os.path.join(PKG, name), os.path.join(pkg, name))
    with open(os.path.join(pkg, "_common.py"), "w") as f:
        f.write(_COMMON_SHIM)
    with open(os.path.join(pkg, "_cpu.py"), "w") as f:
        f.write(_CPU_SHIM.format(repo=REPO, kind=kind))
    test = os.path.join(root, "test")
    os.makedirs(test)
    src = os.path.join(PKG, "test")
    for name in os.listdir(src):
        if name.endswith(".py") and name not in EXCLUDED_TESTS:
            os.symlink(os.path.join(src, name), os.path.join(test, name))
    return test


def run(kind="restated", extra_args=(), timeout=3000):
    """Run the reference suite on the oracle; returns (returncode, output)."""
    with tempfile.TemporaryDirectory() as root:
        test = make_overlay(root, kind)
        env = dict(os.environ)
        env["PYTHONPATH"] = os.pathsep.join([root, REPO, env.get("PYTHONPATH", "")])
        cmd = [sys.executable, "-m", "pytest", test, "-q", "-p", "no:cacheprovider",
               "-p", "no:randomly", "--rootdir", root, *extra_args]
        r = subprocess.run(cmd, cwd=root, env=env, capture_output=True, text=True,
                           timeout=timeout)
        return r.returncode, r.stdout + r.stderr


if __name__ == "__main__":
    kind = sys.argv[1] if len(sys.argv) > 1 else "restated"
    rc, out = run(kind, sys.argv[2:])
    print(out)
    sys.exit(rc)
