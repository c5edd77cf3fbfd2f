"""List every backend name the reference's Python package uses, for the drop-in check.

Parses fresnel/*.py of the reference tree (source only, nothing is imported; the Qt viewer
interact.py left out) and records:
  * "_gpu": for each backend class, the methods the package calls on objects of that class
    (``self._geometry.X``, ``self._tracer.X``, ``self._scene.X``, ``self._device.X`` inside the
    Python class that constructs it with ``...module.<Class>(...)`` / ``_gpu.<Class>(...)``, plus
    the calls made by its Python base classes), and the module-level names used as
    ``_gpu.<name>``;
  * "_common": the names used as ``_common.<name>``.
Writes backend_names.json beside this script.  Run ``python tests/golden/make_backend_names.py``
where the reference tree is present.
"""

import ast
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference tree: FRESNEL_REFERENCE, else where this container mounts it
PKG = os.path.join(os.environ.get("FRESNEL_REFERENCE", "/root/reference"), "fresnel")
HANDLES = ("_geometry", "_tracer", "_scene", "_device")


def _self_attr(node, name):
    return (isinstance(node, ast.Attribute) and node.attr == name
            and isinstance(node.value, ast.Name) and node.value.id == "self")


def scan():
    classes = {}  # python class -> (bases, backend class or None, {handle: set(methods)})
    gpu_names, common_names = set(), set()
    generic = {h: set() for h in HANDLES}  # x._geometry.m etc. with x not `self`
    static = {}  # _gpu.<Class>.<name>
    for fn in sorted(os.listdir(PKG)):
        # interact.py is the Qt viewer (out of scope); its _tracer is a Python-level tracer
        if not fn.endswith(".py") or fn == "interact.py":
            continue
        tree = ast.parse(open(os.path.join(PKG, fn)).read())
        for node in ast.walk(tree):
            if isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name):
                if node.value.id == "_common":
                    common_names.add(node.attr)
                elif node.value.id == "_gpu":
                    gpu_names.add(node.attr)
            # static methods: _gpu.<Class>.<name>
            if (isinstance(node, ast.Attribute) and isinstance(node.value, ast.Attribute)
                    and isinstance(node.value.value, ast.Name) and node.value.value.id == "_gpu"):
                static.setdefault(node.value.attr, set()).add(node.attr)
            if (isinstance(node, ast.Attribute) and isinstance(node.value, ast.Attribute)
                    and node.value.attr in HANDLES
                    and not (isinstance(node.value.value, ast.Name)
                             and node.value.value.id == "self")):
                generic[node.value.attr].add(node.attr)
        for cls in [n for n in ast.walk(tree) if isinstance(n, ast.ClassDef)]:
            bases = [b.id for b in cls.bases if isinstance(b, ast.Name)]
            backend = None
            calls = {h: set() for h in HANDLES}
            for node in ast.walk(cls):
                if isinstance(node, ast.Assign) and isinstance(node.value, ast.Call):
                    f = node.value.func
                    if (isinstance(f, ast.Attribute) and any(_self_attr(t, h) for t in node.targets
                                                             for h in HANDLES)):
                        if (isinstance(f.value, ast.Attribute) and f.value.attr == "module") or \
                                (isinstance(f.value, ast.Name) and f.value.id == "_gpu"):
                            backend = f.attr
                if isinstance(node, ast.Attribute):
                    for h in HANDLES:
                        if _self_attr(node.value, h):
                            calls[h].add(node.attr)
            classes[cls.name] = (bases, backend, calls)

    def all_calls(name):
        bases, _, calls = classes[name]
        out = {h: set(v) for h, v in calls.items()}
        for b in bases:
            if b in classes:
                for h, v in all_calls(b).items():
                    out[h] |= v
        return out

    gpu = {}
    for name, (_, backend, _) in classes.items():
        if backend is None:
            continue
        methods = set()
        for v in all_calls(name).values():
            methods |= v
        gpu.setdefault(backend, set()).update(methods)
    # classes that hold another object's backend handle (material proxies and the like, neither
    # constructing a backend object nor a base of one that does): their calls are generic too
    bases_of_backends = set()
    for name, (bases, backend, _) in classes.items():
        stack = list(bases) if backend else []
        while stack:
            b = stack.pop()
            if b in classes and b not in bases_of_backends:
                bases_of_backends.add(b)
                stack.extend(classes[b][0])
    for name, (bases, backend, calls) in classes.items():
        if backend is None and name not in bases_of_backends:
            for h, v in calls.items():
                generic[h] |= v
    # calls through another object's handle apply to the whole family of backend classes
    family = {"_geometry": "Geometry", "_tracer": "Tracer", "_scene": "Scene", "_device": "Device"}
    for h, names in generic.items():
        for backend in gpu:
            if backend.startswith(family[h]):
                gpu[backend].update(n for n in names if not n.startswith("_"))
    for cls, names in static.items():
        gpu.setdefault(cls, set()).update(names)
    return ({k: sorted(v) for k, v in sorted(gpu.items())}, sorted(gpu_names),
            sorted(common_names))


def main():
    gpu, gpu_names, common = scan()
    out = {"_gpu_classes": gpu, "_gpu_names": gpu_names, "_common": common}
    with open(os.path.join(HERE, "backend_names.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
