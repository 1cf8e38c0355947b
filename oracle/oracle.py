"""Python access to the parity oracle (TEST INFRASTRUCTURE ONLY).

Two oracles live under oracle/:
  * liboracle.so -- the plain-C restatement in gz_oracle.c (always buildable with gcc);
  * _ref/gz_ref_noeager, _ref/gz_ref_eager -- the reference's own sources compiled unmodified
    by oracle/Makefile (only where the reference tree is present at build time).
Only tests/, the smoke check and bench.py's CPU-baseline leg import this module, as a checker.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_NOEAGER = os.path.join(REF_DIR, "gz_ref_noeager")
REF_EAGER = os.path.join(REF_DIR, "gz_ref_eager")
REF_CUBE = os.path.join(REF_DIR, "gz_ref_cube")  # -DL0_SAMPLING -DNO_EAGER_DSU

GOOD, ZERO, FAIL = 0, 1, 2
TRACE_DTYPE = np.dtype([("round", "<u4"), ("key", "<u4"), ("result", "<u4"), ("pad", "<u4"),
                        ("idx", "<u8")])

_lib = None


def build(force: bool = False, reference: str | None = None) -> None:
    """Compile liboracle.so, and oracle/_ref from the reference source tree at `reference`
    (default: the GZ_REFERENCE environment variable) when that tree exists."""
    targets = ["oracle"]
    ref = reference or os.environ.get("GZ_REFERENCE", "")
    env = dict(os.environ)
    if ref and os.path.isdir(ref):
        targets.append("ref")
        env["REF"] = ref
    args = ["make", "-C", HERE] + (["-B"] if force else []) + targets
    subprocess.run(args, check=True, env=env, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(LIB_PATH)
        u8p, u32p, u64p = (ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint32),
                           ctypes.POINTER(ctypes.c_uint64))
        L.gzo_xxh3_8b.restype = ctypes.c_uint64
        L.gzo_xxh3_8b.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.gzo_params.restype = ctypes.c_int
        L.gzo_params.argtypes = [ctypes.c_uint32, ctypes.c_double, u32p, u32p]
        L.gzo_apply_records.restype = ctypes.c_int
        L.gzo_apply_records.argtypes = [u8p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint64, u8p, ctypes.c_size_t, u8p]
        L.gzo_apply_batch.restype = ctypes.c_int
        L.gzo_apply_batch.argtypes = [u8p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_uint64, ctypes.c_uint32, u32p, ctypes.c_size_t]
        L.gzo_sample.restype = ctypes.c_int
        L.gzo_sample.argtypes = [u8p, u8p, ctypes.c_uint32, ctypes.c_uint64, u64p]
        L.gzo_boruvka.restype = ctypes.c_int
        L.gzo_boruvka.argtypes = [u8p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_uint64, u32p, u32p, ctypes.c_void_p, ctypes.c_size_t,
                                  ctypes.POINTER(ctypes.c_size_t)]
        L.gzo_exact_cc.restype = ctypes.c_uint32
        L.gzo_exact_cc.argtypes = [ctypes.c_uint32, u8p, ctypes.c_size_t, u32p]
        L.gzo_exact_cc_mt.restype = ctypes.c_uint32
        L.gzo_exact_cc_mt.argtypes = [ctypes.c_uint32, u8p, ctypes.c_size_t, u32p, ctypes.c_int]
        L.gzo_params_alg.restype = ctypes.c_int
        L.gzo_params_alg.argtypes = [ctypes.c_uint32, ctypes.c_double, ctypes.c_int, u32p, u32p, u32p]
        L.gzo_apply_records_alg.restype = ctypes.c_int
        L.gzo_apply_records_alg.argtypes = [u8p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.c_uint64, u8p, ctypes.c_size_t, u8p, ctypes.c_int]
        L.gzo_boruvka_alg.restype = ctypes.c_int
        L.gzo_boruvka_alg.argtypes = [u8p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_void_p,
                                      ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L.gzo_eager_dsu.restype = ctypes.c_size_t
        L.gzo_eager_dsu.argtypes = [ctypes.c_uint32, u8p, ctypes.c_size_t, u32p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def xxh3_8b(value: int, seed: int) -> int:
    return int(lib().gzo_xxh3_8b(value & (2**64 - 1), seed & (2**64 - 1)))


def params_alg(num_vertices: int, sketches_factor: float = 1.0, cube: bool = False):
    """(num_samples, cols_per_sample, bkt_per_col) of CameoSketch or CubeSketch."""
    s, c, b = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    if lib().gzo_params_alg(num_vertices, sketches_factor, int(cube), ctypes.byref(s), ctypes.byref(c),
                            ctypes.byref(b)):
        raise ValueError("num_vertices must be >= 2")
    return s.value, c.value, b.value


def params(num_vertices: int, sketches_factor: float = 1.0):
    """(num_columns, bkt_per_col, num_buckets, sketch_bytes) of CCSketchAlg(V, .., f)."""
    c, b = ctypes.c_uint32(), ctypes.c_uint32()
    if lib().gzo_params(num_vertices, sketches_factor, ctypes.byref(c), ctypes.byref(b)):
        raise ValueError("num_vertices must be >= 2")
    nb = c.value * b.value + 1
    return c.value, b.value, nb, nb * 12


class OracleSketches:
    """V sketches in the reference byte layout, updated by the C restatement."""

    def __init__(self, num_vertices: int, seed: int, sketches_factor: float = 1.0,
                 cube: bool = False):
        self.V, self.seed, self.factor, self.cube = num_vertices, seed, sketches_factor, cube
        samples, self.cps, self.B = params_alg(num_vertices, sketches_factor, cube)
        self.C = samples * self.cps
        self.nb = self.C * self.B + 1
        self.sketch_bytes = self.nb * 12
        self.data = np.zeros(num_vertices * self.sketch_bytes, np.uint8)

    def apply_records(self, raw: np.ndarray, vertex_filter: np.ndarray | None = None) -> int:
        raw = np.ascontiguousarray(raw, np.uint8)
        filt = None
        if vertex_filter is not None:
            vertex_filter = np.ascontiguousarray(vertex_filter, np.uint8)
            filt = _p(vertex_filter, ctypes.c_uint8)
        return lib().gzo_apply_records_alg(_p(self.data, ctypes.c_uint8), self.V, self.C, self.B,
                                           self.seed, _p(raw, ctypes.c_uint8), raw.size // 9, filt,
                                           int(self.cube))

    def apply_batch(self, src: int, dsts) -> int:
        d = np.ascontiguousarray(dsts, np.uint32)
        return lib().gzo_apply_batch(_p(self.data, ctypes.c_uint8), self.V, self.C, self.B,
                                     self.seed, src, _p(d, ctypes.c_uint32), d.size)

    def sketch(self, v: int) -> np.ndarray:
        return self.data[v * self.sketch_bytes:(v + 1) * self.sketch_bytes]

    def boruvka(self, with_trace: bool = True):
        """Returns (status, labels, rounds, trace)."""
        labels = np.zeros(self.V, np.uint32)
        rounds = ctypes.c_uint32()
        cap = self.V * (self.C + 1) if with_trace else 0
        trace = np.zeros(cap, TRACE_DTYPE)
        tl = ctypes.c_size_t()
        rc = lib().gzo_boruvka_alg(_p(self.data, ctypes.c_uint8), self.V, self.C, self.B, self.cps,
                                   self.seed, _p(labels, ctypes.c_uint32), ctypes.byref(rounds),
                                   trace.ctypes.data if with_trace else None, cap, ctypes.byref(tl))
        return rc, labels, rounds.value, trace[:min(tl.value, cap)]

    def dump_bytes(self) -> bytes:
        """CCSketchAlg::write_binary layout: seed u64, V u32, sketches_factor f64, buckets."""
        head = (np.array([self.seed], "<u8").tobytes() + np.array([self.V], "<u4").tobytes()
                + np.array([self.factor], "<f8").tobytes())
        return head + self.data.tobytes()


def exact_cc(num_vertices: int, raw: np.ndarray):
    """(num_components, labels) of the stream's final graph; labels = smallest member id."""
    raw = np.ascontiguousarray(raw, np.uint8)
    labels = np.zeros(num_vertices, np.uint32)
    n = lib().gzo_exact_cc(num_vertices, _p(raw, ctypes.c_uint8), raw.size // 9,
                           _p(labels, ctypes.c_uint32))
    return int(n), labels


def exact_cc_mt(num_vertices: int, raw: np.ndarray, threads: int | None = None):
    """exact_cc on several host threads (full-size streams)."""
    raw = np.ascontiguousarray(raw, np.uint8)
    labels = np.zeros(num_vertices, np.uint32)
    n = lib().gzo_exact_cc_mt(num_vertices, _p(raw, ctypes.c_uint8), raw.size // 9,
                              _p(labels, ctypes.c_uint32), int(threads or os.cpu_count() or 1))
    return int(n), labels


def eager_dsu(num_vertices: int, raw: np.ndarray):
    """The default build's eager DSU over a record stream from singletons: (index of the record
    that invalidated it or None, labels = smallest member id when still valid)."""
    raw = np.ascontiguousarray(raw, np.uint8)
    labels = np.zeros(num_vertices, np.uint32)
    n = raw.size // 9
    pos = lib().gzo_eager_dsu(num_vertices, _p(raw, ctypes.c_uint8), n, _p(labels, ctypes.c_uint32))
    if pos == ctypes.c_size_t(-1).value:
        raise ValueError("record names a vertex >= V")
    return (None, labels) if pos == n else (int(pos), None)


# ---- the compiled reference (oracle/_ref) --------------------------------------------------

def have_reference() -> bool:
    return os.path.exists(REF_NOEAGER) and os.path.exists(REF_EAGER)


def have_cube_reference() -> bool:
    return os.path.exists(REF_CUBE)


def ref_ingest(stream_path: str, seed: int, sketches_factor: float = 1.0, threads: int = 1,
               eager: bool = False, max_records: int = 0, dump_path: str | None = None,
               labels_path: str | None = None, timeout: float | None = None,
               cube: bool = False) -> dict:
    exe = REF_CUBE if cube else (REF_EAGER if eager else REF_NOEAGER)
    out = subprocess.run([exe, "ingest", stream_path, str(seed), repr(float(sketches_factor)),
                          str(threads), str(max_records), dump_path or "-", labels_path or "-"],
                         check=True, capture_output=True, text=True, timeout=timeout)
    return json.loads(out.stdout.strip().splitlines()[-1])


def ref_trace(dump_path: str, cube: bool = False):
    """Boruvka trace from the reference's own Sketch code: (info, labels, trace)."""
    with tempfile.TemporaryDirectory() as td:
        tp, lp = os.path.join(td, "trace.bin"), os.path.join(td, "labels.bin")
        out = subprocess.run([REF_CUBE if cube else REF_NOEAGER, "trace", dump_path, tp, lp], check=True,
                             capture_output=True, text=True)
        info = json.loads(out.stdout.strip().splitlines()[-1])
        return info, np.fromfile(lp, np.uint32), np.fromfile(tp, TRACE_DTYPE)
