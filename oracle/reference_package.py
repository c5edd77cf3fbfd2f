"""TEST INFRASTRUCTURE: fresnel's own Python package and test suite over stand-in backends.

``stage()`` copies the reference's pure-Python modules (fresnel/*.py) and its test suite
(fresnel/test/*.py, pytest.ini and the golden images in fresnel/test/reference/) out of the
reference tree, unmodified, into oracle/_ref/fresnel_src/.  Like the oracle library compiled
from the reference's headers beside it, the copy is git-ignored and travels to machines that
have no reference tree.

``overlay(root, backend)`` builds an importable ``fresnel`` package in ``root``: its modules are
links to the reference's files (from the reference tree when present, else from the staged
copy), and its compiled modules are small shims:

  backend "oracle-values"  _common = oracle.values (plain Python), _cpu = oracle.cpu_module
                           -- the reference's Python package on the CPU oracle with no
                           compiled module of this repository loaded;
  backend "oracle"         _common = fresnel_b200._common (cpu_built True, gpu_built False),
                           _cpu = oracle.cpu_module;
  backend "engine"         _common = fresnel_b200._common, _gpu = fresnel_b200._gpu (the
                           drop-in: fresnel's unmodified Python package on this engine).

The oracle backends take ``kind``: "restated" (oracle/_build) or "reference" (oracle/_ref, the
reference's own fresnel/common headers compiled).
"""

import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
STAGED = os.path.join(HERE, "_ref", "fresnel_src")


def reference_tree():
    """The reference tree's fresnel package directory (FRESNEL_REFERENCE, else the default
    mount point), or None when it is absent."""
    root = os.environ.get("FRESNEL_REFERENCE", "/root/reference")
    pkg = os.path.join(root, "fresnel")
    return pkg if os.path.isfile(os.path.join(pkg, "__init__.py")) else None


def source():
    """Directory holding fresnel's *.py and test/ to overlay: the reference tree, else the
    staged copy, else None."""
    ref = reference_tree()
    if ref is not None:
        return ref
    if os.path.isfile(os.path.join(STAGED, "__init__.py")):
        return STAGED
    return None


def stage(verbose=False):
    """Copy the reference's Python package and test suite into oracle/_ref/fresnel_src (when
    the reference tree is present and the copy is missing or older).  Returns the copy's path
    or None."""
    ref = reference_tree()
    if ref is None:
        return None
    files = []
    for name in sorted(os.listdir(ref)):
        if name.endswith(".py"):
            files.append(name)
    test = os.path.join(ref, "test")
    for name in sorted(os.listdir(test)):
        if name.endswith(".py") or name == "pytest.ini":
            files.append(os.path.join("test", name))
    for name in sorted(os.listdir(os.path.join(test, "reference"))):
        files.append(os.path.join("test", "reference", name))
    copied = 0
    for rel in files:
        src = os.path.join(ref, rel)
        dst = os.path.join(STAGED, rel)
        if os.path.exists(dst) and os.path.getmtime(dst) >= os.path.getmtime(src):
            continue
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        shutil.copy2(src, dst)
        copied += 1
    os.makedirs(os.path.join(STAGED, "test", "output"), exist_ok=True)
    if verbose and copied:
        print(f"staged {copied} files of the reference's Python package in {STAGED}")
    return STAGED


_SHIMS = {
    "oracle-values": {
        "_common": ("import sys\nsys.path.insert(0, {repo!r})\n"
                    "from oracle.values import *  # noqa: F401,F403\n"
                    "from oracle.values import cpu_built, gpu_built, find_polyhedron_faces  "
                    "# noqa: F401\n"),
        "_cpu": ("import sys\nsys.path.insert(0, {repo!r})\n"
                 "from oracle import cpu_module as _m\n"
                 "from oracle.cpu_module import *  # noqa: F401,F403\n\n\n"
                 "class Device(_m.Device):\n    kind = {kind!r}\n"),
    },
    "oracle": {
        "_common": ("import sys\nsys.path.insert(0, {repo!r})\n"
                    "from fresnel_b200._common import *  # noqa: F401,F403\n"
                    "from fresnel_b200._common import find_polyhedron_faces  # noqa: F401\n\n\n"
                    "def cpu_built():\n    return True\n\n\n"
                    "def gpu_built():\n    return False\n"),
        "_cpu": ("import sys\nsys.path.insert(0, {repo!r})\n"
                 "from oracle import cpu_module as _m\n"
                 "from oracle.cpu_module import *  # noqa: F401,F403\n\n\n"
                 "class Device(_m.Device):\n    kind = {kind!r}\n"),
    },
    "engine": {
        "_common": ("import sys\nsys.path.insert(0, {repo!r})\n"
                    "from fresnel_b200._common import *  # noqa: F401,F403\n"
                    "from fresnel_b200._common import find_polyhedron_faces  # noqa: F401\n\n\n"
                    "def cpu_built():\n    return False\n\n\n"
                    "def gpu_built():\n    return True\n"),
        "_gpu": ("import sys\nsys.path.insert(0, {repo!r})\n"
                 "from fresnel_b200._gpu import *  # noqa: F401,F403\n"),
    },
}


def overlay(root, backend, kind="restated", excluded_tests=()):
    """Create <root>/fresnel (the overlay package) and <root>/test (links to the reference's
    tests).  Returns the test directory, or None when neither the reference tree nor the staged
    copy exists."""
    src = source()
    if src is None:
        return None
    pkg = os.path.join(root, "fresnel")
    os.makedirs(pkg)
    for name in os.listdir(src):
        if name.endswith(".py"):
            os.symlink(os.path.join(src, name), os.path.join(pkg, name))
    for mod, text in _SHIMS[backend].items():
        with open(os.path.join(pkg, mod + ".py"), "w") as f:
            f.write(text.format(repo=REPO, kind=kind))
    test = os.path.join(root, "test")
    os.makedirs(test)
    tsrc = os.path.join(src, "test")
    for name in os.listdir(tsrc):
        if (name.endswith(".py") or name == "pytest.ini") and name not in excluded_tests:
            os.symlink(os.path.join(tsrc, name), os.path.join(test, name))
    return test


def import_fresnel(root, backend, kind="restated"):
    """Build the overlay in ``root`` and import its ``fresnel`` package in this process."""
    if overlay(root, backend, kind) is None:
        raise FileNotFoundError("neither the reference tree nor its staged copy "
                                "(oracle/_ref/fresnel_src) is present")
    if root not in sys.path:
        sys.path.insert(0, root)
    import fresnel
    return fresnel
