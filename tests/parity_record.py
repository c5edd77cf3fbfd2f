"""Measured parity rates, appended to a record file (test infrastructure).

Parity tests call ``record(test, **fields)`` with what they measured (mismatching samples,
grazing samples, the rate, pixels within tolerance, ...).  When the environment variable
FRB_PARITY_RECORD names a file, each call appends one JSON line to it; otherwise nothing is
written.  tests/parity_rates.jsonl holds the record of a full GPU run.
"""

import json
import os
import time


def record(test, **fields):
    path = os.environ.get("FRB_PARITY_RECORD")
    line = {"test": test, **{k: _plain(v) for k, v in fields.items()}}
    print("parity:", json.dumps(line))
    if not path:
        return
    line["time"] = time.strftime("%Y-%m-%dT%H:%M:%S")
    with open(path, "a") as f:
        f.write(json.dumps(line) + "\n")


def _plain(v):
    """numpy scalars and tuples as JSON values."""
    if hasattr(v, "item") and callable(v.item) and getattr(v, "shape", None) == ():
        return v.item()
    if isinstance(v, (list, tuple)):
        return [_plain(x) for x in v]
    if isinstance(v, dict):
        return {k: _plain(x) for k, x in v.items()}
    return v
