"""Drop-in check without a GPU: every backend class, method and module name that the
reference's Python package (fresnel/*.py, the Qt viewer aside) uses on ``_gpu`` and ``_common``
exists in this package's extension modules under the same name.  The names were read from the
reference's source by tests/golden/make_backend_names.py into tests/golden/backend_names.json.
"""

import json
import os

import pytest

from fresnel_b200 import _common, _gpu

NAMES = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "backend_names.json")))


@pytest.mark.parametrize("cls", sorted(NAMES["_gpu_classes"]))
def test_gpu_class_has_every_method_the_reference_calls(cls):
    assert hasattr(_gpu, cls), f"_gpu.{cls} missing"
    missing = [m for m in NAMES["_gpu_classes"][cls] if not hasattr(getattr(_gpu, cls), m)]
    assert not missing, f"_gpu.{cls} lacks {missing}"


def test_gpu_module_names():
    missing = [n for n in NAMES["_gpu_names"] if not hasattr(_gpu, n)]
    assert not missing


def test_common_module_names():
    missing = [n for n in NAMES["_common"] if not hasattr(_common, n)]
    assert not missing
