"""Golden vectors for Tracer.histogram, made by the reference's own code.

Reads ``Tracer.histogram`` from the reference tree (fresnel/tracer.py:79-108) as source,
compiles that one function on its own (its module needs fresnel's compiled extensions, which
this container cannot build) and runs it, with numpy, on the crafted images of
``oracle.output_path.crafted_images``.  Writes histogram.npz: for each image, its pixels and
the reference's counts and bin edges.  Run ``python tests/golden/make_histogram_golden.py``
where the reference tree is present.
"""

import ast
import os
import sys

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import output_path  # noqa: E402

# the reference tree: FRESNEL_REFERENCE, else where this container mounts it
REFERENCE = os.path.join(os.environ.get("FRESNEL_REFERENCE", "/root/reference"), "fresnel",
                         "tracer.py")


def reference_histogram():
    tree = ast.parse(open(REFERENCE).read())
    for node in ast.walk(tree):
        if isinstance(node, ast.ClassDef) and node.name == "Tracer":
            for fn in node.body:
                if isinstance(fn, ast.FunctionDef) and fn.name == "histogram":
                    mod = ast.Module(body=[fn], type_ignores=[])
                    scope = {"numpy": numpy}
                    exec(compile(mod, REFERENCE, "exec"), scope)
                    return scope["histogram"]
    raise RuntimeError("Tracer.histogram not found in " + REFERENCE)


class _Image:
    """Stands in for a tracer: ``linear_output[:]`` returns the image."""

    def __init__(self, a):
        self.linear_output = a


def main():
    hist = reference_histogram()
    out = {}
    for name, img in output_path.crafted_images().items():
        counts, edges = hist(_Image(img))
        out[name + "_image"] = img
        out[name + "_counts"] = counts
        out[name + "_edges"] = edges
        print(name, img.shape, int(counts.sum()))
    numpy.savez_compressed(os.path.join(HERE, "histogram.npz"), **out)


if __name__ == "__main__":
    main()
