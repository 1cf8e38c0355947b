"""Regenerate the golden fixtures in tests/golden/ from the compiled reference (oracle/_ref).

    GZ_REFERENCE=<reference source tree> python tests/golden/make_golden.py

Needs the reference tree (to build oracle/_ref with oracle/Makefile, and for the stream fixture
the reference's own tests read) and the `xxhash` Python package; the tests only read the files
this writes. Outputs:
  xxh3_vectors.json   XXH3_64bits_withSeed over 8-byte inputs, from libxxhash (python xxhash)
  params.json         sizing from the reference's own Sketch::calc_* functions
  <case>.gzs          seeded streams in the 9-byte binary format
  ref_mult_v1024.data the reference's own test stream test/res/multiples_graph_1024_stream.data,
                      copied byte for byte (read by test/cc_alg_test.cpp:300-350; 78 components)
  <case>.labels.npy   partition from CCSketchAlg::connected_components (smallest member id)
  <case>.trace.npy    every sampled component of every Boruvka round (reference Sketch code)
  manifest.json       per case: vertices, seeds, dump SHA-256, components, rounds
"""
from __future__ import annotations

import hashlib
import json
import os
import random
import shutil
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from graphzeppelin_b200 import streams as S  # noqa: E402
from oracle import oracle as O  # noqa: E402

# name, stream builder, sketch seed, sketches_factor
CASES = [
    ("c0_v1024", lambda: S.planted_partition_stream(1024, 4, seed=1, p=0.25, churn_fraction=0.2,
                                                    uniform_assignment=True)[0], 12345, 1.0),
    ("mult_v1024", lambda: S.edges_to_stream(1024, S.multiples_graph_edges(1024), seed=3,
                                             churn_fraction=0.3), 777, 1.0),
    ("er_v64", lambda: S.erdos_renyi_stream(64, 0.1, seed=5, churn_fraction=0.5), 42, 1.0),
    ("sparse_v300", lambda: S.erdos_renyi_stream(300, 0.006, seed=7, churn_fraction=0.2), 99, 1.0),
    ("planted_v256_f2", lambda: S.planted_partition_stream(256, 3, seed=11, p=0.05,
                                                           churn_fraction=0.1)[0], 2024, 2.0),
    ("cl_v2048", lambda: S.chung_lu_stream(2048, 2.1, 8.0, 256, seed=13), 31337, 1.0),
]


# Stream fixtures of the reference's own test suite, copied unchanged from its tree:
# name, path inside the reference tree, sketch seed, sketches_factor, components its tests expect
REF_FIXTURES = [
    ("ref_mult_v1024", "test/res/multiples_graph_1024_stream.data", 4242, 1.0, 78),
]


def xxh3_vectors(n=256):
    import xxhash
    rng = random.Random(20261203)
    vals = [0, 1, 2**32 - 1, 2**32, 2**64 - 1, (5 << 32) | 9]
    seeds = [0, 1, 5, 2**31, 2**63, 2**64 - 1, 12345]
    out = []
    for v in vals:
        for s in seeds:
            out.append((v, s))
    while len(out) < n:
        out.append((rng.getrandbits(64), rng.getrandbits(rng.choice([8, 32, 64]))))
    return [{"value": v, "seed": s,
             "hash": xxhash.xxh3_64_intdigest(struct.pack("<Q", v), seed=s)} for v, s in out]


def main():
    ref_tree = os.environ.get("GZ_REFERENCE", "")
    assert ref_tree and os.path.isdir(ref_tree), "set GZ_REFERENCE to the reference source tree"
    O.build(reference=ref_tree)
    assert O.have_reference(), "oracle/_ref was not built (reference tree missing?)"
    with open(os.path.join(HERE, "xxh3_vectors.json"), "w") as f:
        json.dump({"source": "python xxhash %s (libxxhash %s)" % (
            __import__("xxhash").VERSION, __import__("xxhash").XXHASH_VERSION),
            "vectors": xxh3_vectors()}, f, indent=0)
    vs = [2, 3, 4, 5, 16, 17, 64, 100, 255, 256, 300, 1000, 1024, 4097, 65535, 65536, 131072,
          262144, 1048576, 2**31]
    params = []
    for f in (1.0, 0.5, 2.0, 3.7):
        out = subprocess.run([O.REF_NOEAGER, "params", repr(f)] + [str(v) for v in vs],
                             check=True, capture_output=True, text=True).stdout
        for line in out.strip().splitlines():
            d = json.loads(line)
            d["sketches_factor"] = f
            params.append(d)
    with open(os.path.join(HERE, "params.json"), "w") as f:
        json.dump(params, f, indent=0)

    manifest = []
    jobs = [(name, builder, seed, factor, name + ".gzs", None) for name, builder, seed, factor in CASES]
    jobs += [(name, rel, seed, factor, name + ".data", want) for name, rel, seed, factor, want in REF_FIXTURES]
    with tempfile.TemporaryDirectory() as td:
        for name, builder, seed, factor, fname, want_cc in jobs:
            spath = os.path.join(HERE, fname)
            if want_cc is None:
                st = builder()
                st.write(spath)
            else:
                shutil.copyfile(os.path.join(ref_tree, builder), spath)
                st = S.read_stream(spath)
            dump = os.path.join(td, name + ".dump")
            lab = os.path.join(td, name + ".labels")
            info = O.ref_ingest(spath, seed, factor, threads=2, dump_path=dump, labels_path=lab)
            eager = O.ref_ingest(spath, seed, factor, threads=2, eager=True)
            tinfo, tlabels, trace = O.ref_trace(dump)
            labels = np.fromfile(lab, np.uint32)
            assert (tlabels == labels).all(), name
            assert tinfo["rounds"] == info["rounds"], name
            assert eager["num_cc"] == info["num_cc"], name
            np.save(os.path.join(HERE, name + ".labels.npy"), labels)
            np.save(os.path.join(HERE, name + ".trace.npy"), trace)
            sha = hashlib.sha256(open(dump, "rb").read()).hexdigest()
            ncc, _ = O.exact_cc(st.num_vertices, st.raw())
            if want_cc is not None:
                assert info["num_cc"] == ncc == want_cc, (name, info["num_cc"], ncc)
            manifest.append({"name": name, "stream": fname, "num_vertices": st.num_vertices,
                             "num_updates": st.num_updates, "seed": seed, "sketches_factor": factor,
                             "dump_sha256": sha, "dump_bytes": os.path.getsize(dump),
                             "num_cc": info["num_cc"], "exact_num_cc": ncc,
                             "rounds": info["rounds"], "trace_len": int(trace.size),
                             "trace_fails": int((trace["result"] == 2).sum())})
            print(name, manifest[-1])
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"generated_by": "tests/golden/make_golden.py from the reference sources "
                                   "compiled by oracle/Makefile", "cases": manifest}, f, indent=1)


if __name__ == "__main__":
    main()
