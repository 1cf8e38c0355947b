"""Access to the committed golden fixtures (tests/golden/, made by make_golden.py)."""
import json
import os

import numpy as np

from graphzeppelin_b200 import streams as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)["cases"]


def case_names():
    return [c["name"] for c in manifest()]


def load_case(name):
    c = next(c for c in manifest() if c["name"] == name)
    st = S.read_stream(os.path.join(GOLDEN, c["stream"]))
    labels = np.load(os.path.join(GOLDEN, name + ".labels.npy"))
    trace = np.load(os.path.join(GOLDEN, name + ".trace.npy"))
    return c, st, labels, trace


def xxh3_vectors():
    with open(os.path.join(GOLDEN, "xxh3_vectors.json")) as f:
        return json.load(f)["vectors"]


def params_table():
    with open(os.path.join(GOLDEN, "params.json")) as f:
        return json.load(f)


def canonical(labels):
    """Smallest member id per vertex, from any representative labelling."""
    p = np.asarray(labels).astype(np.int64)
    mn = np.full(p.size, np.iinfo(np.int64).max)
    np.minimum.at(mn, p, np.arange(p.size))
    return mn[p].astype(np.uint32)
