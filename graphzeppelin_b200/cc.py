"""Python mirror of the reference's CCSketchAlg / GraphSketchDriver surface over the C ABI.

Names, argument meaning and error behaviour follow include/cc_sketch_alg.h,
include/graph_sketch_driver.h, include/cc_alg_configuration.h, include/driver_configuration.h
and include/return_types.h of the reference; the work itself runs in libgz_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes
import enum
import time
from collections import namedtuple
from typing import Iterable, List, Sequence, Set

import numpy as np

from . import _lib
from .streams import RECORD_DTYPE, Stream, read_stream

# ------------------------------------------------------------------------------------------------
# exceptions (include/sketch.h:193-204, include/cc_sketch_alg.h:25-29,
# include/graph_sketch_driver.h:13-21)
# ------------------------------------------------------------------------------------------------


class GZError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_lib.status_string(status)}: {msg}" if msg else _lib.status_string(status))
        self.status = status


class OutOfSamplesException(GZError):
    pass


class UpdateLockedException(GZError):
    def __str__(self):
        return "Cannot update the algorithm: Connected components currently running"


class BadVertexError(GZError):
    pass


class DriverException(RuntimeError):
    pass


def _check(rc: int):
    if rc == _lib.GZ_OK:
        return
    msg = _lib.last_error()
    if rc == _lib.GZ_ERR_OUT_OF_SAMPLES:
        raise OutOfSamplesException(rc, msg)
    if rc == _lib.GZ_ERR_LOCKED:
        raise UpdateLockedException(rc, msg)
    if rc == _lib.GZ_ERR_BAD_VERTEX:
        raise BadVertexError(rc, msg)
    raise GZError(rc, msg)


# ------------------------------------------------------------------------------------------------
# enums / plain types
# ------------------------------------------------------------------------------------------------

class QueryCode(enum.IntEnum):
    """include/cc_sketch_alg.h:60-63"""
    CONNECTIVITY = 0
    KSPANNINGFORESTS = 1


CONNECTIVITY = QueryCode.CONNECTIVITY
KSPANNINGFORESTS = QueryCode.KSPANNINGFORESTS


class SampleResult(enum.IntEnum):
    """include/sketch.h:20-24"""
    GOOD = 0
    ZERO = 1
    FAIL = 2


class UpdateType(enum.IntEnum):
    INSERT = 0
    DELETE = 1
    BREAKPOINT = 2


Edge = namedtuple("Edge", ["src", "dst"])


class GraphUpdate(namedtuple("GraphUpdate", ["edge", "type"])):
    """include/types.h:12-15"""

    def __new__(cls, edge, type=UpdateType.INSERT):
        return super().__new__(cls, Edge(*edge), UpdateType(type))


def concat_pairing_fn(i: int, j: int) -> int:
    """src/util.cpp:45-51"""
    if i > j:
        i, j = j, i
    return (i << 32) | j


def inv_concat_pairing_fn(idx: int) -> Edge:
    """src/util.cpp:53-57"""
    return Edge(idx >> 32, idx & 0xFFFFFFFF)


class CCAlgConfiguration:
    """include/cc_alg_configuration.h, src/cc_alg_configuration.cpp (fluent setters; a factor
    <= 0 falls back to 1 with a message, as the reference does)."""

    def __init__(self):
        self._disk_dir = "."
        self._sketches_factor = 1.0
        self._batch_factor = 1.0

    def disk_dir(self, d: str) -> "CCAlgConfiguration":
        self._disk_dir = d
        return self

    def sketches_factor(self, f: float) -> "CCAlgConfiguration":
        self._sketches_factor = float(f)
        if self._sketches_factor <= 0:
            print(f"sketches_factor={self._sketches_factor} is out of bounds. (0, infty)"
                  "Defaulting to 1.")
            self._sketches_factor = 1.0
        return self

    def batch_factor(self, f: float) -> "CCAlgConfiguration":
        self._batch_factor = float(f)
        if self._batch_factor <= 0:
            print(f"batch factor={self._batch_factor} is out of bounds. (0, infty)"
                  "Defaulting to 1.")
            self._batch_factor = 1.0
        return self

    def get_disk_dir(self) -> str:
        return self._disk_dir

    def get_sketches_factor(self) -> float:
        return self._sketches_factor

    def get_batch_factor(self) -> float:
        return self._batch_factor

    def __str__(self):
        return ("Connected Components Algorithm Configuration:\n"
                " Sketching algorithm   = CameoSketch\n"
                " Using Eager DSU       = False\n"
                f" Num sketches factor   = {self._sketches_factor:g}\n"
                f" Batch size factor     = {self._batch_factor:g}\n"
                f" On disk data location = {self._disk_dir}")


class GutterSystem(enum.IntEnum):
    """include/driver_configuration.h:5-9, plus DEVICE: the device-resident gutter that every
    choice maps to here (the host guttering systems are replaced, not rebuilt)."""
    GUTTERTREE = 0
    STANDALONE = 1
    CACHETREE = 2
    DEVICE = 3


GUTTERTREE, STANDALONE, CACHETREE = GutterSystem.GUTTERTREE, GutterSystem.STANDALONE, GutterSystem.CACHETREE


class DriverConfiguration:
    """include/driver_configuration.h, src/driver_configuration.cpp"""

    def __init__(self):
        self._gutter_sys = GutterSystem.STANDALONE
        self._disk_dir = "."
        self._num_worker_threads = 1
        self._gutter_capacity = 0

    def gutter_sys(self, g) -> "DriverConfiguration":
        self._gutter_sys = GutterSystem(g)
        return self

    def disk_dir(self, d: str) -> "DriverConfiguration":
        self._disk_dir = d
        return self

    def worker_threads(self, n: int) -> "DriverConfiguration":
        self._num_worker_threads = int(n)
        if self._num_worker_threads < 1:
            print(f"num_worker_threads={self._num_worker_threads} is out of bounds. [1, infty)"
                  "Defaulting to 1.")
            self._num_worker_threads = 1
        return self

    def gutter_capacity(self, endpoint_updates: int) -> "DriverConfiguration":
        """Device gutter size in endpoint updates (0 = the library default)."""
        self._gutter_capacity = int(endpoint_updates)
        return self

    def get_gutter_sys(self):
        return self._gutter_sys

    def get_disk_dir(self):
        return self._disk_dir

    def get_worker_threads(self):
        return self._num_worker_threads

    def __str__(self):
        return ("GraphSketchDriver Configuration:\n"
                " Guttering system      = DeviceGutter\n"
                f" Worker thread count   = {self._num_worker_threads}\n"
                f" On disk data location = {self._disk_dir}")


# ------------------------------------------------------------------------------------------------
# results (include/return_types.h, src/return_types.cpp)
# ------------------------------------------------------------------------------------------------

class ConnectedComponents:
    def __init__(self, parent: np.ndarray, num_cc: int):
        self.parent_arr = parent
        self.num_cc = int(num_cc)

    def size(self) -> int:
        return self.num_cc

    def __len__(self):
        return self.num_cc

    def is_connected(self, a: int, b: int) -> bool:
        return bool(self.parent_arr[a] == self.parent_arr[b])

    def get_component_sets(self) -> List[Set[int]]:
        """Sets ordered by representative, like the std::map walk of get_component_sets."""
        order = np.argsort(self.parent_arr, kind="stable")
        reps = self.parent_arr[order]
        cuts = np.flatnonzero(np.diff(reps)) + 1
        return [set(map(int, g)) for g in np.split(order, cuts)]

    def canonical_labels(self) -> np.ndarray:
        """Smallest member id of each vertex's component (representative-independent)."""
        p = self.parent_arr.astype(np.int64)
        mn = np.full(p.size, np.iinfo(np.int64).max)
        np.minimum.at(mn, p, np.arange(p.size))
        return mn[p].astype(np.uint32)


class SpanningForest:
    def __init__(self, edges: np.ndarray):
        self._edges = edges

    def get_edges(self) -> List[Edge]:
        return [Edge(int(a), int(b)) for a, b in self._edges]


# ------------------------------------------------------------------------------------------------
# CCSketchAlg
# ------------------------------------------------------------------------------------------------

def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


class CCSketchAlg:
    """Connected components of a dynamic graph stream (include/cc_sketch_alg.h:69-258).

    The V vertex sketches live in GPU memory; updates go through the device gutter and queries
    run device Boruvka. The cached-query behaviour is that of the reference built with
    NO_EAGER_DSU: any update invalidates it."""

    SKETCH_ALGORITHMS = {"cameo": _lib.GZ_CAMEO_SKETCH, "cube": _lib.GZ_CUBE_SKETCH}

    def __init__(self, num_vertices: int, seed: int, config: CCAlgConfiguration | None = None,
                 _handle=None, sketch_algorithm: str = "cameo"):
        """sketch_algorithm: "cameo" (CameoSketch, the reference's default build) or "cube"
        (CubeSketch, the reference built with -DL0_SAMPLING)."""
        self.lib = _lib.load()
        self.config = config or CCAlgConfiguration()
        if _handle is None:
            h = ctypes.c_void_p()
            _check(self.lib.gz_create_ex(num_vertices, seed & (2**64 - 1),
                                         self.config.get_sketches_factor(),
                                         self.config.get_batch_factor(),
                                         self.SKETCH_ALGORITHMS[sketch_algorithm], ctypes.byref(h)))
            _handle = h
        self._h = _handle
        p = _lib.gz_params_t()
        _check(self.lib.gz_get_params(self._h, ctypes.byref(p)))
        self.params = p
        self.cc_alg_start = self.cc_alg_end = 0.0

    # -- construction / teardown ---------------------------------------------------------------
    @classmethod
    def construct_from_serialized_data(cls, input_file: str,
                                       config: CCAlgConfiguration | None = None,
                                       sketch_algorithm: str = "cameo") -> "CCSketchAlg":
        """src/cc_sketch_alg.cpp:30-43 (the file's sketches_factor replaces the config's)."""
        lib = _lib.load()
        config = config or CCAlgConfiguration()
        h = ctypes.c_void_p()
        _check(lib.gz_create_from_serialized_ex(input_file.encode(), config.get_batch_factor(),
                                                cls.SKETCH_ALGORITHMS[sketch_algorithm],
                                                ctypes.byref(h)))
        obj = cls.__new__(cls)
        p = _lib.gz_params_t()
        _check(lib.gz_get_params(h, ctypes.byref(p)))
        config.sketches_factor(p.sketches_factor)
        CCSketchAlg.__init__(obj, p.num_vertices, p.seed, config, _handle=h)
        return obj

    def close(self):
        if getattr(self, "_h", None):
            self.lib.gz_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- driver contract (include/graph_sketch_driver.h:28-69) -----------------------------------
    def allocate_worker_memory(self, num_workers: int) -> None:
        _check(self.lib.gz_allocate_worker_memory(self._h, num_workers))

    def get_desired_updates_per_batch(self) -> int:
        return int(self.params.desired_updates_per_batch)

    def get_num_vertices(self) -> int:
        return int(self.params.num_vertices)

    def pre_insert(self, upd: GraphUpdate, thr_id: int = 0) -> None:
        _check(self.lib.gz_pre_insert(self._h, upd.edge.src, upd.edge.dst, int(upd.type), thr_id))

    def apply_update_batch(self, thr_id: int, src_vertex: int, dst_vertices: Sequence[int]) -> None:
        d = np.ascontiguousarray(dst_vertices, dtype=np.uint32)
        _check(self.lib.gz_apply_update_batch(self._h, thr_id, src_vertex, _ptr(d), d.size))

    def has_cached_query(self, query_code: int) -> bool:
        out = ctypes.c_int()
        _check(self.lib.gz_has_cached_query(self._h, int(query_code), ctypes.byref(out)))
        return bool(out.value)

    def print_configuration(self) -> None:
        print(self.config)

    # -- updates --------------------------------------------------------------------------------
    def apply_raw_buckets_update(self, src_vertex: int, raw_buckets: np.ndarray) -> None:
        raw = np.ascontiguousarray(raw_buckets).view(np.uint8).reshape(-1)
        if raw.size != self.params.sketch_bytes:
            raise ValueError("raw bucket buffer must hold num_buckets * 12 bytes")
        _check(self.lib.gz_apply_raw_buckets_update(self._h, src_vertex, _ptr(raw)))

    def update(self, upd: GraphUpdate) -> None:
        _check(self.lib.gz_update(self._h, upd.edge.src, upd.edge.dst, int(upd.type)))

    def ingest_records(self, records) -> None:
        """Ingest packed 9-byte records (a RECORD_DTYPE array, a raw uint8 array or a Stream)
        from host memory through the device gutter."""
        raw = _as_raw(records)
        _check(self.lib.gz_ingest_records(self._h, _ptr(raw), raw.size // 9))

    def ingest_records_device(self, ptr: int, n_records: int) -> None:
        """Ingest n_records packed records already resident in GPU memory at address ptr."""
        _check(self.lib.gz_ingest_records_device(self._h, ctypes.c_void_p(ptr), n_records))

    def flush(self) -> None:
        _check(self.lib.gz_flush(self._h))

    # -- queries ---------------------------------------------------------------------------------
    def connected_components(self) -> ConnectedComponents:
        self.cc_alg_start = time.perf_counter()
        parent = np.empty(self.params.num_vertices, np.uint32)
        n = ctypes.c_uint32()
        _check(self.lib.gz_connected_components(self._h, _ptr(parent), ctypes.byref(n)))
        self.cc_alg_end = time.perf_counter()
        return ConnectedComponents(parent, n.value)

    def query_submit(self) -> int:
        """Snapshot the sketches (after every update so far) and start their connectivity query
        on the device; updates made afterwards proceed meanwhile. Returns a ticket."""
        t = ctypes.c_uint64()
        _check(self.lib.gz_query_submit(self._h, ctypes.byref(t)))
        return int(t.value)

    def query_wait(self, ticket: int):
        """(ConnectedComponents, rounds) of the state at the ticket's submission."""
        parent = np.empty(self.params.num_vertices, np.uint32)
        n = ctypes.c_uint32()
        r = ctypes.c_size_t()
        _check(self.lib.gz_query_wait(self._h, ticket, _ptr(parent), ctypes.byref(n), ctypes.byref(r)))
        return ConnectedComponents(parent, n.value), int(r.value)

    def num_connected_components(self) -> int:
        n = ctypes.c_uint32()
        _check(self.lib.gz_connected_components(self._h, None, ctypes.byref(n)))
        return int(n.value)

    def point_query(self, a: int, b: int) -> bool:
        out = ctypes.c_int()
        _check(self.lib.gz_point_query(self._h, a, b, ctypes.byref(out)))
        return bool(out.value)

    def calc_spanning_forest(self) -> SpanningForest:
        n = ctypes.c_size_t()
        _check(self.lib.gz_spanning_forest(self._h, None, 0, ctypes.byref(n)))
        buf = np.zeros((max(n.value, 1), 2), np.uint32)
        _check(self.lib.gz_spanning_forest(self._h, _ptr(buf), n.value, ctypes.byref(n)))
        return SpanningForest(buf[:n.value])

    @property
    def last_query_rounds(self) -> int:
        out = ctypes.c_size_t()
        _check(self.lib.gz_last_query_rounds(self._h, ctypes.byref(out)))
        return int(out.value)

    def get_seed(self) -> int:
        return int(self.params.seed)

    def max_rounds(self) -> int:
        return int(self.params.max_rounds)

    # -- checkpoint --------------------------------------------------------------------------------
    def write_binary(self, filename: str) -> None:
        _check(self.lib.gz_write_binary(self._h, filename.encode()))

    def clear(self) -> None:
        """Sketch::zero_contents on every vertex sketch: back to the empty graph."""
        _check(self.lib.gz_clear(self._h))

    def dump_sketches(self) -> np.ndarray:
        buf = np.empty(self.params.sketch_bytes * self.params.num_vertices, np.uint8)
        _check(self.lib.gz_dump_sketches(self._h, _ptr(buf), buf.size))
        return buf

    # -- instrumentation ---------------------------------------------------------------------------
    def set_trace(self, enable: bool = True) -> None:
        _check(self.lib.gz_set_trace(self._h, int(enable)))

    def get_trace(self) -> np.ndarray:
        """Every sampled component of the last Boruvka: records sorted by (round, key)."""
        dt = np.dtype([("round", "<u4"), ("key", "<u4"), ("result", "<u4"), ("pad", "<u4"),
                       ("idx", "<u8")])
        n = ctypes.c_size_t()
        _check(self.lib.gz_get_trace(self._h, None, 0, ctypes.byref(n)))
        buf = np.zeros(n.value, dt)
        if n.value:
            _check(self.lib.gz_get_trace(self._h, _ptr(buf), n.value, ctypes.byref(n)))
        return np.sort(buf, order=["round", "key"])

    def set_profiling(self, enable: bool = True) -> None:
        _check(self.lib.gz_set_profiling(self._h, int(enable)))

    def get_profile(self) -> dict:
        p = _lib.gz_profile_t()
        _check(self.lib.gz_get_profile(self._h, ctypes.byref(p)))
        return {f: getattr(p, f) for f, _ in p._fields_}

    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        _check(self.lib.gz_get_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def set_eager_dsu(self, enable: bool = True) -> None:
        """The reference's default eager DSU (gz_set_eager_dsu): pre_insert keeps a union-find
        and spanning forest on the host so queries stay cached until a forest edge changes."""
        _check(self.lib.gz_set_eager_dsu(self._h, int(enable)))

    def set_tuning(self, vertices_per_tile: int = 0, threads_per_block: int = 0,
                   tiles_per_bin: int = 0, entry_form: int = 0) -> None:
        """0 keeps defaults; entry_form 1 = plain entries (hashed per endpoint), 2 = coded entries
        (each record hashed once, applied through bucket planes), 3 = coded entries with 3-bit
        depth codes (gz_set_tuning)."""
        _check(self.lib.gz_set_tuning(self._h, vertices_per_tile, threads_per_block,
                                      tiles_per_bin, entry_form))
        p = _lib.gz_params_t()
        _check(self.lib.gz_get_params(self._h, ctypes.byref(p)))
        self.params = p

    def set_direct_factor(self, factor: float) -> None:
        """Sparse tiles below factor x the staging break-even go in place (gz_set_direct_factor);
        0 always stages."""
        _check(self.lib.gz_set_direct_factor(self._h, float(factor)))

    def set_pipeline(self, mode: int = -1) -> None:
        """Sketch-update kernel: 1 tile pipeline (2..4: with that many tile buffers), 0 one
        staged tile at a time, -1 the handle's choice (gz_set_pipeline). Re-picks the default
        tiling."""
        _check(self.lib.gz_set_pipeline(self._h, int(mode)))
        p = _lib.gz_params_t()
        _check(self.lib.gz_get_params(self._h, ctypes.byref(p)))
        self.params = p

    def set_query_graph(self, mode=-1) -> None:
        """How queries run (gz_set_query_graph): 2 one cooperative kernel, 1 (or True) a CUDA
        graph of per-phase kernels, 0 (or False) those kernels with the round loop on the host
        (for profilers), -1 by size (the default: 2 up to 2^18 vertices, 1 above)."""
        _check(self.lib.gz_set_query_graph(self._h, int(mode)))

    def set_gutter_capacity(self, endpoint_updates: int) -> None:
        _check(self.lib.gz_set_gutter_capacity(self._h, endpoint_updates))


def measure_hash_rate(repeats: int = 5) -> float:
    """Peak 8-byte XXH3 + depth evaluations per second of the current GPU (register-only)."""
    lib = _lib.load()
    out = ctypes.c_double()
    _check(lib.gz_measure_hash_rate(repeats, ctypes.byref(out)))
    return out.value


def measure_update_rate(repeats: int = 5) -> float:
    """Peak shared-memory 12-byte bucket XOR updates per second of the current GPU."""
    lib = _lib.load()
    out = ctypes.c_double()
    _check(lib.gz_measure_update_rate(repeats, ctypes.byref(out)))
    return out.value


def _as_raw(records) -> np.ndarray:
    if isinstance(records, Stream):
        records = records.records
    a = np.asarray(records)
    if a.dtype == RECORD_DTYPE:
        a = a.view(np.uint8).reshape(-1)
    a = np.ascontiguousarray(a, dtype=np.uint8).reshape(-1)
    if a.size % 9:
        raise ValueError("record buffer length must be a multiple of 9 bytes")
    return a


# ------------------------------------------------------------------------------------------------
# streams + driver
# ------------------------------------------------------------------------------------------------

END_OF_STREAM = -1


class BinaryFileStream:
    """Reader of the reference's binary stream format (StreamingUtilities BinaryFileStream)."""

    def __init__(self, file_name: str | None = None, stream: Stream | None = None):
        self._s = stream if stream is not None else read_stream(file_name)
        self._pos = 0
        self._break = self._s.num_updates

    def vertices(self) -> int:
        return self._s.num_vertices

    def edges(self) -> int:
        return self._s.num_updates

    def set_break_point(self, break_idx: int) -> bool:
        if break_idx == END_OF_STREAM or break_idx > self._s.num_updates:
            break_idx = self._s.num_updates
        if break_idx < self._pos:
            return False
        self._break = break_idx
        return True

    def get_update_is_thread_safe(self) -> bool:
        return True

    def take_until_break(self) -> np.ndarray:
        """Records from the current position to the break point (zero-copy view)."""
        out = self._s.records[self._pos:self._break]
        self._pos = self._break
        return out


class GraphSketchDriver:
    """include/graph_sketch_driver.h:70-229 with the GutteringSystem and worker threads replaced
    by the device gutter: process_stream_until hands raw records to the GPU, prep_query folds
    the gutter into the sketches and synchronizes."""

    def __init__(self, sketching_alg: CCSketchAlg, stream: BinaryFileStream,
                 config: DriverConfiguration | None = None, num_stream_threads: int = 1):
        config = config or DriverConfiguration()
        self.sketching_alg = sketching_alg
        self.stream = stream
        self.num_stream_threads = num_stream_threads
        sketching_alg.allocate_worker_memory(config.get_worker_threads())
        if config._gutter_capacity:
            sketching_alg.set_gutter_capacity(config._gutter_capacity)
        self.total_updates = 0
        self.flush_start = self.flush_end = 0.0

    def process_stream_until(self, break_edge_idx: int) -> None:
        if not self.stream.set_break_point(break_edge_idx):
            raise DriverException(f"Could not correctly set breakpoint: {break_edge_idx}")
        recs = self.stream.take_until_break()
        if recs.size:
            # ingest_records also performs pre_insert's work (it invalidates the cached answer)
            self.sketching_alg.ingest_records(recs)
            self.total_updates += 2 * recs.size  # both directions, as the gutters see them

    def prep_query(self, query_code: int = CONNECTIVITY) -> None:
        if self.sketching_alg.has_cached_query(query_code):
            self.flush_start = self.flush_end = time.perf_counter()
            return
        self.flush_start = time.perf_counter()
        self.sketching_alg.flush()
        self.flush_end = time.perf_counter()

    def batch_callback(self, thr_id: int, src_vertex: int, dst_vertices: Sequence[int]) -> None:
        self.total_updates += len(dst_vertices)
        self.sketching_alg.apply_update_batch(thr_id, src_vertex, dst_vertices)

    def get_total_updates(self) -> int:
        return self.total_updates
