"""Run fresnel's own test suite on a stand-in backend (test infrastructure).

The overlay package (oracle/reference_package.py) holds the reference's own pure-Python modules
and tests, unmodified, with the compiled modules replaced:
  backend "oracle"  _common -> fresnel_b200._common (cpu_built True, gpu_built False),
                    _cpu    -> oracle.cpu_module (restated or reference-header math);
  backend "engine"  _common -> fresnel_b200._common, _gpu -> fresnel_b200._gpu (the drop-in).
``pytest <overlay>/test`` then renders every scene of the reference's suite with that backend
and compares it with the reference's golden PNGs.  The reference's files come from the
reference tree (environment variable FRESNEL_REFERENCE, or the container's default location)
or from the copy staged beside the reference-built oracle (oracle/_ref/fresnel_src); callers
skip when neither is present.
"""

import os
import subprocess
import sys
import tempfile

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from oracle import reference_package  # noqa: E402

# Reference test files left out of the overlay run (none: every geometry is implemented).
EXCLUDED_TESTS = []


def available():
    return reference_package.source() is not None


def make_overlay(root, kind="restated", backend="oracle"):
    """Create <root>/fresnel (overlay package) and <root>/test (links to the reference tests)."""
    return reference_package.overlay(root, backend, kind, EXCLUDED_TESTS)


def run(kind="restated", extra_args=(), timeout=3000, backend="oracle"):
    """Run the reference suite on the backend; returns (returncode, output)."""
    with tempfile.TemporaryDirectory() as root:
        test = make_overlay(root, kind, backend)
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
