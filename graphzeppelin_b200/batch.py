"""Many independent graph streams on one GPU (the gz_batch_* entry points of include/gz_b200.h).

A CCSketchBatch holds G CCSketchAlg instances (include/cc_sketch_alg.h:69), each with its own
vertex count and seed. Records of all graphs are ingested by one gutter pass and one persistent
sketch-update launch; connected_components() runs Boruvka for every graph at once. Per graph
the sketches, partition, last_query_rounds and out-of-samples outcome equal those of a
CCSketchAlg with the same V and seed fed the same records.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence

import numpy as np

from . import _lib
from .cc import ConnectedComponents, OutOfSamplesException, _as_raw, _check, _ptr

GZ_ERR_OUT_OF_SAMPLES = 3


class BatchResult:
    """Per-graph outcome of one batched query."""

    def __init__(self, labels: List[np.ndarray], num_cc: np.ndarray, rounds: np.ndarray,
                 status: np.ndarray):
        self.labels = labels
        self.num_cc = num_cc
        self.rounds = rounds
        self.status = status

    def out_of_samples(self, g: int) -> bool:
        return int(self.status[g]) == GZ_ERR_OUT_OF_SAMPLES

    def connected_components(self, g: int) -> ConnectedComponents:
        """Graph g's answer; raises OutOfSamplesException where CCSketchAlg would have."""
        if self.out_of_samples(g):
            raise OutOfSamplesException(GZ_ERR_OUT_OF_SAMPLES,
                                        f"graph {g} ran out of sketch columns")
        return ConnectedComponents(self.labels[g], int(self.num_cc[g]))


class CCSketchBatch:
    def __init__(self, num_vertices: Sequence[int], seeds: Sequence[int],
                 sketches_factor: float = 1.0, vertices_per_tile: Sequence[int] | None = None):
        self.lib = _lib.load()
        self.num_vertices = np.ascontiguousarray(num_vertices, dtype=np.uint32)
        g = self.num_vertices.size
        if len(seeds) != g:
            raise ValueError("one seed per graph")
        seeds_a = np.array([int(s) & (2**64 - 1) for s in seeds], dtype=np.uint64)
        vpt = None
        if vertices_per_tile is not None:
            vpt = np.ascontiguousarray(vertices_per_tile, dtype=np.uint32)
            if vpt.size != g:
                raise ValueError("one vertices_per_tile entry per graph")
        h = ctypes.c_void_p()
        _check(self.lib.gz_batch_create(g, _ptr(self.num_vertices), _ptr(seeds_a),
                                        float(sketches_factor),
                                        _ptr(vpt) if vpt is not None else None, ctypes.byref(h)))
        self._h = h
        self.num_graphs = g
        self._refresh_params()
        self.vbase = np.concatenate([[0], np.cumsum(self.num_vertices.astype(np.int64))])

    def close(self):
        if getattr(self, "_h", None):
            self.lib.gz_batch_destroy(self._h)
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

    # -- ingest -------------------------------------------------------------------------------------
    def ingest(self, streams: Sequence) -> None:
        """Fold every graph's records (one record array or Stream per graph, host memory)."""
        if len(streams) != self.num_graphs:
            raise ValueError("one record array per graph")
        raws = [_as_raw(s) for s in streams]
        offsets = np.zeros(self.num_graphs + 1, np.uint64)
        offsets[1:] = np.cumsum([r.size // 9 for r in raws])
        buf = np.concatenate(raws) if raws else np.zeros(0, np.uint8)
        _check(self.lib.gz_batch_ingest(self._h, _ptr(buf) if buf.size else None, _ptr(offsets)))

    def ingest_packed(self, raw: np.ndarray, offsets: Sequence[int]) -> None:
        """Records of all graphs back to back in one host uint8 array (graph g's are records
        [offsets[g], offsets[g+1])); pinned memory makes the copy faster."""
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        if off.size != self.num_graphs + 1:
            raise ValueError("offsets needs num_graphs + 1 entries")
        buf = np.ascontiguousarray(raw, dtype=np.uint8).reshape(-1)
        if buf.size < 9 * int(off[-1]):
            raise ValueError("record buffer shorter than the offsets say")
        _check(self.lib.gz_batch_ingest(self._h, _ptr(buf) if buf.size else None, _ptr(off)))

    def ingest_device(self, ptr: int, offsets: Sequence[int]) -> None:
        """Records already on the GPU at ptr; graph g's are records [offsets[g], offsets[g+1])."""
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        if off.size != self.num_graphs + 1:
            raise ValueError("offsets needs num_graphs + 1 entries")
        _check(self.lib.gz_batch_ingest_device(self._h, ctypes.c_void_p(ptr), _ptr(off)))

    def clear(self) -> None:
        _check(self.lib.gz_batch_clear(self._h))

    # -- queries ------------------------------------------------------------------------------------
    def connected_components(self, labels: bool = True) -> BatchResult:
        g = self.num_graphs
        lab = np.empty(int(self.vbase[-1]), np.uint32) if labels else None
        ncc = np.zeros(g, np.uint32)
        rounds = np.zeros(g, np.uint32)
        status = np.zeros(g, np.int32)
        _check(self.lib.gz_batch_connected_components(
            self._h, _ptr(lab) if labels else None, _ptr(ncc), _ptr(rounds), _ptr(status)))
        per = [lab[self.vbase[i]:self.vbase[i + 1]] for i in range(g)] if labels else []
        return BatchResult(per, ncc, rounds, status)

    def dump_sketches(self, g: int) -> np.ndarray:
        p = self.params[g]
        buf = np.empty(p.sketch_bytes * p.num_vertices, np.uint8)
        _check(self.lib.gz_batch_dump_sketches(self._h, g, _ptr(buf), buf.size))
        return buf

    def load_sketches(self, g: int, data: np.ndarray) -> None:
        """Replace graph g's sketches (V * sketch_bytes bytes, dump_sketches' layout)."""
        buf = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
        _check(self.lib.gz_batch_load_sketches(self._h, g, _ptr(buf), buf.size))

    def set_tuning(self, threads_per_block: int = 0, ctas_per_sm: int = 0,
                   vertices_per_tile: Sequence[int] | None = None) -> None:
        """Shape of the batched sketch-update launch (see gz_batch_set_tuning)."""
        vpt = None
        if vertices_per_tile is not None:
            vpt = np.ascontiguousarray(vertices_per_tile, dtype=np.uint32)
            if vpt.size != self.num_graphs:
                raise ValueError("one vertices_per_tile entry per graph")
        _check(self.lib.gz_batch_set_tuning(self._h, threads_per_block, ctas_per_sm,
                                            _ptr(vpt) if vpt is not None else None))
        self._refresh_params()

    def set_route(self, sparse_factor: float) -> None:
        """Per-call routing between in-place and staged ingest (gz_batch_set_route)."""
        _check(self.lib.gz_batch_set_route(self._h, float(sparse_factor)))

    def autotune(self, records_per_vertex: int = 0) -> np.ndarray:
        """Run the autotuner (gz_batch_autotune); returns the vertices per tile chosen per graph."""
        out = np.zeros(self.num_graphs, np.uint32)
        _check(self.lib.gz_batch_autotune(self._h, records_per_vertex, _ptr(out)))
        self._refresh_params()
        return out

    def _refresh_params(self):
        self.params = []
        for i in range(self.num_graphs):
            p = _lib.gz_params_t()
            _check(self.lib.gz_batch_get_params(self._h, i, ctypes.byref(p)))
            self.params.append(p)

    def set_profiling(self, enable: bool = True) -> None:
        _check(self.lib.gz_batch_set_profiling(self._h, int(enable)))

    def get_profile(self) -> dict:
        p = _lib.gz_profile_t()
        _check(self.lib.gz_batch_get_profile(self._h, ctypes.byref(p)))
        return {f: getattr(p, f) for f, _ in p._fields_}
