#!/usr/bin/env python
"""Benchmark of the B200 sketch-ingest + Boruvka connected-components path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--small]

Workload (one replica per GPU): the dense planted-partition stream -- V = 2^17 vertices in 64
planted components (sizes uniform, >= 256), intra-component edges, 10% insert-then-delete
churn over random non-edges, ~1.4e8 packed 9-byte records (1.26 GB), one connectivity query at
the end. A step = clear the sketches, ingest every record (device gutter + sketch update), run
the query. `value` = updates / device time of the step with the records already in HBM;
`e2e` = the same through the public API from pinned host memory (copies inside the timing).

Under torchrun (N > 1) every rank runs an independent replica (the path is single-GPU; there is
no data-path collective); timing is the max over ranks.

`--impl reference` times the reference's own CCSketchAlg (compiled from its sources into
oracle/_ref) on the host cores over bounded samples of the same stream.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edge updates/sec + CC query ms on 1 B200"
UNIT = "updates/s"

FULL = dict(workload="dense_planted_v131072_c64_deg1780_churn10", num_vertices=1 << 17,
            components=64, min_size=256, mean_degree=1780.0, churn=0.10, stream_seed=1,
            sketch_seed=0x5EED5EED)
SMALL = dict(workload="dense_planted_v16384_c16_deg800_churn10", num_vertices=1 << 14,
             components=16, min_size=256, mean_degree=800.0, churn=0.10, stream_seed=1,
             sketch_seed=0x5EED5EED)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def gen_stream(cfg, out=None):
    from graphzeppelin_b200 import streams as S
    return S.planted_partition_stream_fast(cfg["num_vertices"], cfg["components"],
                                           cfg["stream_seed"], mean_degree=cfg["mean_degree"],
                                           min_size=cfg["min_size"],
                                           churn_fraction=cfg["churn"], out=out)


# ------------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.first = threading.Event()
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to print its first sample: the timed region starts after it
            self.first.wait(timeout=3.0)
            self.lines.clear()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ------------------------------------------------------------------------------------------------
# CPU baseline: the reference's CCSketchAlg on the host cores
# ------------------------------------------------------------------------------------------------
def cpu_reference_run(stream, cfg, n_records: int, threads: int, timeout=600, path=None,
                      eager=True, dump_path=None, labels_path=None):
    """Ingest the first n_records through the reference's CCSketchAlg compiled from its sources
    (oracle/_ref: gz_ref_eager = the default eager-DSU build, timed as the baseline;
    gz_ref_noeager = the -DNO_EAGER_DSU build whose query always runs Boruvka) with the stand-in
    gutter, and return its JSON (ingest_s, query_s, num_cc, rounds, ...). `path`: the stream
    already written to a file."""
    from oracle import oracle as O
    from graphzeppelin_b200 import streams as S
    if O.have_reference():
        with tempfile.TemporaryDirectory() as td:
            if path is None:
                path = os.path.join(td, "sample.gzs")
                S.Stream(stream.num_vertices, stream.records[:n_records]).write(path)
                n_arg = 0
            else:
                n_arg = n_records if n_records < stream.num_updates else 0
            r = O.ref_ingest(path, cfg["sketch_seed"], 1.0, threads=threads, eager=eager,
                             max_records=n_arg, dump_path=dump_path, labels_path=labels_path,
                             timeout=timeout)
        r["kind"] = "reference"
        return r
    # the compiled reference is unavailable: time the C restatement (single thread)
    osk = O.OracleSketches(stream.num_vertices, cfg["sketch_seed"])
    t0 = time.perf_counter()
    osk.apply_records(stream.records[:n_records].view("u1").reshape(-1))
    t1 = time.perf_counter()
    rc, lab, rounds, _ = osk.boruvka(with_trace=False)
    t2 = time.perf_counter()
    return {"ingest_s": t1 - t0, "query_s": t2 - t1, "threads": 1, "kind": "port",
            "updates": n_records, "rounds": rounds}


def sha256_file(path):
    import hashlib
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 24), b""):
            h.update(blk)
    return h.hexdigest()


def cpu_baseline_and_parity(alg, stream, cfg, cc, threads=None):
    """The reference on the host cores over the whole stream, twice: the default eager-DSU
    build timed (the CPU baseline), and the -DNO_EAGER_DSU build (whose query runs Boruvka) for
    parity. Parity: the GPU's write_binary file against the reference's (SHA-256; the format of
    src/cc_sketch_alg.cpp:614-623), the partition and the Boruvka rounds against the reference's
    connected_components (src/cc_sketch_alg.cpp:515-557), and the partition against an exact
    union-find over the stream's final edge set."""
    import numpy as np
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    n = stream.num_updates
    V = stream.num_vertices
    with tempfile.TemporaryDirectory() as td:
        spath = os.path.join(td, "stream.gzs")
        stream.write(spath)
        r = cpu_reference_run(stream, cfg, n, threads, path=spath, eager=True)
        value = n / (r["ingest_s"] + r["query_s"])
        cpu = {"value": value, "unit": UNIT, "cores": int(r.get("threads", threads)),
               "kind": r["kind"],
               "sample": f"all {n} records of the same stream (ingest {r['ingest_s']:.3f} s + "
                         f"query {r['query_s']:.3f} s, {r.get('num_cc', '?')} components)",
               "ingest_updates_per_s": n / r["ingest_s"], "query_ms": r["query_s"] * 1e3}
        parity = {"reference": "unavailable"}
        if r["kind"] == "reference":
            gpath, rdump, rlab = (os.path.join(td, x) for x in ("gpu.bin", "ref.bin", "ref.labels"))
            alg.write_binary(gpath)
            ref = cpu_reference_run(stream, cfg, n, threads, path=spath, eager=False,
                                    dump_path=rdump, labels_path=rlab)
            gsha, rsha = sha256_file(gpath), sha256_file(rdump)
            labels = cc.canonical_labels()
            rlabels = np.fromfile(rlab, np.uint32)
            n_exact, exact = O.exact_cc_mt(V, stream.raw(), threads)
            parity = {
                "sketch_sha256_equal": gsha == rsha, "partition_equal": bool((labels == rlabels).all()),
                "rounds_equal": int(alg.last_query_rounds) == int(ref["rounds"]),
                "exact_partition_equal": bool((labels == exact).all()),
                "components": {"gpu": cc.size(), "reference": int(ref["num_cc"]), "exact": n_exact},
                "rounds": {"gpu": int(alg.last_query_rounds), "reference": int(ref["rounds"])},
                "sketch_sha256": gsha,
                "reference": "reference CCSketchAlg compiled from its sources (-DNO_EAGER_DSU) on "
                             "the whole stream; exact union-find over the final edge set"}
    return cpu, parity


# ------------------------------------------------------------------------------------------------
def roofline(alg, n, prof, steps, ingest_ms, hash_peak, hbm_peak_gbs, update_peak):
    """Roofline of the ingest (one pass of the hot path over the step's records) per the
    algorithmic work of one record: 1 + C XXH3 hashes (one per column and the checksum, hashed
    once per edge), 9 B of stream read, and the touched sketches read and written once. The path
    is bound by the slower of the hash term (over the measured hash rate) and the HBM term.
    Per kernel: the gutter phase (count + hash sort-scatter) against its own hashes (C columns per
    record, once) and bytes, the sketch update against the shared-memory slot rate (2 (C + 1)
    bucket updates per record, made as 2 x 32 slot steps), its hashes (the checksum, per
    endpoint) and its bytes."""
    p = alg.params
    V, C, B, sb = p.num_vertices, p.num_columns, p.bkt_per_col, p.sketch_bytes
    t_ing = statistics.mean(ingest_ms) / 1e3
    hashes = n * (C + 1)
    path_bytes = 9 * n + 2 * V * sb
    t_hash, t_hbm = hashes / hash_peak, path_bytes / (hbm_peak_gbs * 1e9)
    bound = "int" if t_hash >= t_hbm else "hbm"
    kernels = {}
    t_g = prof["gutter_ms"] / max(1, prof["gutter_launches"]) / 1e3
    t_u = prof["sketch_update_ms"] / max(1, prof["sketch_update_launches"]) / 1e3
    if p.entry_form == 2:
        coded = C  # every column hashed once per record in the gutter pass
        g_bytes = 9 * n + 9 * n + 2 * n * 16
        kernels["gutter"] = {
            "kernels": "k_gutter (count) + k_hash_sort_scatter", "launch_ms": t_g * 1e3,
            "bound": "int", "hashes_per_launch": n * coded,
            "int": {"achieved": n * coded / t_g / 1e9, "peak": hash_peak / 1e9, "unit": "Ghash/s",
                    "frac": n * coded / t_g / hash_peak},
            "hbm": {"achieved": g_bytes / t_g / 1e9, "peak": hbm_peak_gbs, "unit": "GB/s",
                    "frac": g_bytes / t_g / 1e9 / hbm_peak_gbs, "bytes_per_launch": g_bytes}}
        rows = min(B, 11)
        u_bytes = 2 * n * 16 + 2 * V * 12 * (C * rows + 1)
        slots = 2 * n * 32
        u_hashes = 2 * n  # the checksum, per endpoint
        kernels["sketch_update"] = {
            "kernels": "k_plane_update", "launch_ms": t_u * 1e3, "bound": "smem",
            "bucket_updates_per_launch": 2 * n * (C + 1), "slot_steps_per_launch": slots,
            "hashes_per_launch": u_hashes,
            "smem": {"achieved": slots / t_u / 1e9, "peak": update_peak / 1e9,
                     "unit": "Gslot/s", "frac": slots / t_u / update_peak,
                     "useful_frac": 2 * n * (C + 1) / t_u / update_peak},
            "int": {"achieved": u_hashes / t_u / 1e9, "peak": hash_peak / 1e9, "unit": "Ghash/s",
                    "frac": u_hashes / t_u / hash_peak},
            "hbm": {"achieved": u_bytes / t_u / 1e9, "peak": hbm_peak_gbs, "unit": "GB/s",
                    "frac": u_bytes / t_u / 1e9 / hbm_peak_gbs, "bytes_per_launch": u_bytes}}
    else:
        kernels["gutter"] = {"kernels": "k_gutter (count) + k_gutter_sort_scatter", "launch_ms": t_g * 1e3}
        kernels["sketch_update"] = {"kernels": "k_sketch_update (staged tiles, hashed per endpoint)",
                                    "launch_ms": t_u * 1e3, "hashes_per_launch": 2 * n * (C + 1),
                                    "int": {"achieved": 2 * n * (C + 1) / t_u / 1e9,
                                            "frac": 2 * n * (C + 1) / t_u / hash_peak}}
    achieved = hashes / t_ing if bound == "int" else path_bytes / t_ing
    peak = hash_peak if bound == "int" else hbm_peak_gbs * 1e9
    return {"bound": bound, "achieved": achieved / 1e9, "peak": peak / 1e9,
            "unit": "Ghash/s" if bound == "int" else "GB/s", "frac": achieved / peak,
            "kernel": "ingest = " + " + ".join(k["kernels"] for k in kernels.values()),
            "launch_ms": t_ing * 1e3,
            "units_per_launch": {"records": n, "hashes": hashes, "bytes": path_bytes},
            "terms_ms": {"int": t_hash * 1e3, "hbm": t_hbm * 1e3},
            "kernels": kernels}


def load_traffic(workload):
    """DRAM bytes per sketch-update launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "sketch_update_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(workload)
    except Exception:
        return None


def combine_ranks(local_total_ms: float, records_per_rank: int, steps: int, world: int, dist=None,
                  device=None):
    """Whole-job result over replicas: the slowest rank's device time, every rank's records."""
    total_ms = local_total_ms
    if dist is not None and world > 1:
        import torch
        tt = torch.tensor([local_total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    return total_ms, world * records_per_rank * steps / (total_ms / 1e3)


def run_b200(args, cfg):
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    import graphzeppelin_b200 as gz
    from graphzeppelin_b200 import cc as gzcc

    t = time.time()
    # the records live in pinned host memory (for e2e) and are copied once into HBM (for value)
    from graphzeppelin_b200 import streams as S
    probe, _ = gen_stream(cfg)
    n = probe.num_updates
    pinned = torch.empty(n * 9, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = probe.raw()
    stream = S.Stream(cfg["num_vertices"], pinned.numpy().view(S.RECORD_DTYPE))
    del probe
    d_rec = pinned.cuda(non_blocking=False)
    torch.cuda.synchronize()
    log(f"[rank {rank}] stream: {n} records ({n * 9 / 1e9:.2f} GB) in {time.time() - t:.1f} s")

    V = cfg["num_vertices"]
    alg = gz.CCSketchAlg(V, cfg["sketch_seed"])
    if args.host_rounds:
        alg.set_query_graph(False)
    if args.pipeline is not None:
        alg.set_pipeline(args.pipeline)
    alg.set_gutter_capacity(2 * n + 1024)
    lib_stream = torch.cuda.ExternalStream(alg.stream_handle())
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def step():
        e0, e1, e2 = ev(), ev(), ev()
        e0.record(lib_stream)
        alg.clear()
        alg.ingest_records_device(d_rec.data_ptr(), n)
        alg.flush()
        e1.record(lib_stream)
        ncc = alg.num_connected_components()
        e2.record(lib_stream)
        return e0, e1, e2, ncc

    # the clock sampler runs from before the warm-up (its first sample takes a moment); only the
    # samples taken from the start of the timed steps are kept
    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        *_, ncc = step()
    torch.cuda.synchronize()
    if ncc != cfg["components"]:
        raise SystemExit(f"wrong answer: {ncc} components, expected {cfg['components']}")

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.lines.clear()
    alg.set_profiling(True)
    marks = []
    tw0 = time.perf_counter()
    for _ in range(args.steps):
        marks.append(step())
    torch.cuda.synchronize()
    tw1 = time.perf_counter()
    prof = alg.get_profile()
    alg.set_profiling(False)
    clocks = sampler.stop()
    ingest_ms = [a.elapsed_time(b) for a, b, c, _ in marks]
    query_ms = [b.elapsed_time(c) for a, b, c, _ in marks]
    total_ms = sum(a.elapsed_time(c) for a, b, c, _ in marks)
    total_ms, value = combine_ranks(total_ms, n, args.steps, world, dist, device="cuda")
    ms_per_step = total_ms / args.steps

    # end to end through the public API: pinned host records in, partition out
    e2e_s = []
    for i in range(0 if args.no_e2e else max(1, min(args.steps, 3)) + 1):
        alg.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        alg.ingest_records(stream.records)
        cc = alg.connected_components()
        t1 = time.perf_counter()
        if i:
            e2e_s.append(t1 - t0)
    if args.no_e2e:
        e2e_s = [float("nan")]
    else:
        assert cc.size() == cfg["components"]
    # the ceiling e2e works against: one plain pinned host -> HBM copy of the step's records
    copy_ms = []
    for _ in range(0 if args.no_e2e else 3):
        c0, c1 = ev(), ev()
        c0.record()
        d_rec.copy_(pinned, non_blocking=True)
        c1.record()
        c1.synchronize()
        copy_ms.append(c0.elapsed_time(c1))
    e2e = {"value": world * n / max(e2e_s), "unit": UNIT, "h2d_bytes_per_step": n * 9,
           "d2h_bytes_per_step": V * 4 + 4,
           "h2d_copy_gbs": round(n * 9 / (min(copy_ms) * 1e6), 1) if copy_ms else None,
           "copy_bound_value": world * n / (min(copy_ms) / 1e3) if copy_ms else None,
           "note": "pinned host records -> gz_ingest_records (pipelined H2D) -> "
                   "gz_connected_components -> parent array on host; wall clock, max of steps; "
                   "copy_bound_value = updates/s of the records' plain host->device copy alone"}

    line = None
    if rank == 0:
        hbm_peak = 6546.2
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                hbm_peak = float(json.load(f)["hbm_gbs"])
            peak_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
        except Exception:
            peak_src = "fallback 6546.2 GB/s"
        hash_peak = gzcc.measure_hash_rate(5)
        update_peak = gzcc.measure_update_rate(5)
        roof = roofline(alg, n, prof, args.steps, ingest_ms, hash_peak, hbm_peak, update_peak)
        roof["traffic"] = load_traffic(cfg["workload"])
        roof["peaks"] = {"hbm": peak_src,
                         "int": "measured here: gz_measure_hash_rate (register-only per-column "
                                "XXH3-8B of premixed input and seed + depth ctz, best of 5)",
                         "smem": "measured here: gz_measure_update_rate (bucket-plane slot "
                                 "steps, two conflict-free red.shared.xor each, best of 5)"}
        p = alg.params
        cpu, parity = None, None
        if world == 1 and not args.no_cpu_baseline:
            log("[rank 0] timing the CPU reference baseline and checking full-size parity ...")
            cpu, parity = cpu_baseline_and_parity(alg, stream, cfg, cc)
        checks = None
        if world == 1 and not args.no_checks:
            log("[rank 0] full-size parity of the power-law and many-graph workloads ...")
            checks = {}
            for name, fn in (("powerlaw", powerlaw_check), ("many_graphs", many_graphs_check)):
                try:
                    checks[name] = fn()
                except Exception as e:  # reported in the line, the headline stands
                    checks[name] = {"error": repr(e)}
        serving = None
        if world == 1 and not args.no_serving:
            log("[rank 0] short serving replay with the admission queue in use ...")
            try:
                serving = serving_short()
            except SystemExit:
                raise
            except Exception as e:  # reported in the line, the headline stands
                serving = {"error": repr(e)}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded planted-partition stream, C generator)",
            "config": {"workload": cfg["workload"], "num_vertices": V, "num_updates": n,
                       "components": cfg["components"], "num_columns": p.num_columns,
                       "bkt_per_col": p.bkt_per_col, "sketch_bytes_total": V * p.sketch_bytes,
                       "entry_form": "coded (each record hashed once), bucket planes"
                       if p.entry_form == 2 else "plain (hashed per endpoint), staged tiles",
                       "stream_seed": cfg["stream_seed"], "sketch_seed": cfg["sketch_seed"],
                       "l2": "inputs larger than L2: 1.26 GB records + 1.29 GB sketches per step",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "query_ms": statistics.mean(query_ms),
            "ingest_ms": statistics.mean(ingest_ms),
            "ingest_updates_per_s": n / (statistics.mean(ingest_ms) / 1e3),
            "parity": parity,
            "checks": checks,
            "serving": serving,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks,
            "gpu_launches": int(prof["kernel_launches"]),
            "profile": {k: prof[k] for k in ("gutter_ms", "sketch_update_ms", "query_ms",
                                             "sketch_update_launches", "gutter_launches")},
            "wall_s_timed": tw1 - tw0,
        }
    alg.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return line


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if rank != 0:
        return None
    stream, _ = gen_stream(cfg)
    n_total = stream.num_updates
    threads = os.cpu_count() or 1
    # every step ingests the whole stream and answers the query, as the GPU arm's step does
    n = n_total
    with tempfile.TemporaryDirectory() as td:
        spath = os.path.join(td, "stream.gzs")
        stream.write(spath)
        for _ in range(args.warmup):
            cpu_reference_run(stream, cfg, n, threads, path=spath)
        runs = [cpu_reference_run(stream, cfg, n, threads, path=spath) for _ in range(args.steps)]
    total = sum(x["ingest_s"] + x["query_s"] for x in runs)
    value = n * args.steps / total
    kind = runs[0]["kind"]
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded planted-partition stream, C generator)",
        "config": {"workload": cfg["workload"], "num_vertices": cfg["num_vertices"],
                   "num_updates": n_total,
                   "parallelism": f"{runs[0].get('threads', threads)} host threads"},
        "impl": "reference",
        "query_ms": statistics.mean(x["query_s"] for x in runs) * 1e3,
        "ingest_updates_per_s": n / statistics.mean(x["ingest_s"] for x in runs),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": int(runs[0].get("threads", threads)),
                         "kind": kind,
                         "sample": f"all {n} records of the stream per step, then the query "
                                   f"(reference CCSketchAlg, eager DSU, stand-in gutter)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


MANY = dict(workload="many_graphs_g512_v2e8-2e16_deg8-256_c1-16_churn10", num_graphs=512,
            stream_seed=3)


def run_many_graphs(args):
    """Many independent graph streams on one GPU: the batched engine (one gutter pass, one
    persistent sketch-update launch, CUDA-graph Boruvka rounds for all graphs) against the plain
    single-graph path run graph by graph on the same device-resident records. Each step = clear
    every sketch, ingest every graph's records, query every graph."""
    import numpy as np
    import torch

    import graphzeppelin_b200 as gz
    from graphzeppelin_b200 import streams as S

    torch.cuda.set_device(0)
    G = args.graphs or MANY["num_graphs"]
    t = time.time()
    Vs, seeds, raw, off = S.many_graph_streams(G, MANY["stream_seed"])
    n = int(off[-1])
    pinned = torch.empty(raw.size, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = raw
    del raw
    d_rec = pinned.cuda()
    torch.cuda.synchronize()
    log(f"[many] {G} graphs, {int(Vs.sum())} vertices, {n} records ({n * 9 / 1e9:.2f} GB) "
        f"in {time.time() - t:.1f} s")
    base = d_rec.data_ptr()

    # --- plain path, graph by graph (one CCSketchAlg per graph, created once) ---
    plain_ms, plain_ncc = [], None
    if not args.no_plain:
        algs = []
        for g in range(G):
            a = gz.CCSketchAlg(int(Vs[g]), int(seeds[g]))
            a.set_gutter_capacity(2 * int(off[g + 1] - off[g]) + 1024)
            algs.append(a)

        def plain_step():
            out = np.zeros(G, np.uint32)
            for g, a in enumerate(algs):
                a.clear()
                cnt = int(off[g + 1] - off[g])
                if cnt:
                    a.ingest_records_device(base + 9 * int(off[g]), cnt)
                out[g] = a.num_connected_components()
            return out

        for _ in range(args.warmup):
            plain_ncc = plain_step()
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            plain_ncc = plain_step()
            torch.cuda.synchronize()
            plain_ms.append((time.perf_counter() - t0) * 1e3)
        for a in algs:
            a.close()
        del algs
        torch.cuda.empty_cache()

    # --- batched engine ---
    b = gz.CCSketchBatch(Vs, seeds)
    tune = None
    if not args.no_autotune:
        t0 = time.perf_counter()
        chosen = b.autotune(int(round(2 * n / max(1, int(Vs.sum())))))
        hist = {int(v): int(c) for v, c in zip(*np.unique(chosen, return_counts=True))}
        tune = {"seconds": time.perf_counter() - t0, "vertices_per_tile_hist": hist}
        log(f"[many] autotune {tune}")

    def batch_step():
        b.clear()
        b.ingest_device(base, off)
        return b.connected_components(labels=False)

    for _ in range(args.warmup):
        res = batch_step()
    if plain_ncc is not None and not (res.num_cc == plain_ncc).all():
        raise SystemExit("batched and plain answers differ")
    sampler = ClockSampler(0)
    sampler.start()
    b.set_profiling(True)
    batch_ms = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = batch_step()
        torch.cuda.synchronize()
        batch_ms.append((time.perf_counter() - t0) * 1e3)
    prof = b.get_profile()
    b.set_profiling(False)
    clocks = sampler.stop()

    # end to end: pinned host records through gz_batch_ingest, answers back on the host (the
    # first pass is an untimed warm-up: it sizes the batch's record staging buffer)
    e2e_ms = []
    for i in range(0 if args.no_e2e else 4):
        b.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.ingest_packed(pinned.numpy(), off)
        r = b.connected_components(labels=True)
        if i:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    sketch_bytes_total = int(sum(p.sketch_bytes * p.num_vertices for p in b.params))
    b.close()

    steps = args.steps
    ms = statistics.mean(batch_ms)
    line = {
        "metric": "edge updates/sec, many graphs batched on 1 B200", "value": n / (ms / 1e3),
        "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded planted-partition streams, C generator)",
        "config": {"workload": MANY["workload"] if G == 512 else f"many_graphs_g{G}",
                   "num_graphs": G, "total_vertices": int(Vs.sum()), "num_updates": n,
                   "v_min": int(Vs.min()), "v_max": int(Vs.max()),
                   "sketch_bytes_total": sketch_bytes_total,
                   "l2": "inputs larger than L2 (GB of records and sketches per step)"},
        "timing": "wall clock between device synchronisations (each call is synchronous)",
        "batched": {"ms_per_step": ms, "ms_min": min(batch_ms),
                    "gutter_ms": prof["gutter_ms"] / steps,
                    "sketch_update_ms": prof["sketch_update_ms"] / steps,
                    "query_ms": prof["query_ms"] / steps,
                    "query_rounds": prof["query_rounds"] / steps,
                    "kernel_launches_per_step": prof["kernel_launches"] / (steps + args.warmup)},
        "plain_graph_by_graph": ({"ms_per_step": statistics.mean(plain_ms),
                                  "value": n / (statistics.mean(plain_ms) / 1e3),
                                  "speedup_of_batched": statistics.mean(plain_ms) / ms}
                                 if plain_ms else None),
        "e2e": ({"value": n / (max(e2e_ms) / 1e3), "unit": UNIT, "h2d_bytes_per_step": n * 9,
                 "d2h_bytes_per_step": int(Vs.sum()) * 4 + 12 * G,
                 "note": "pinned host records -> gz_batch_ingest -> "
                         "gz_batch_connected_components with labels; wall clock, max of 3 after one untimed pass"}
                if e2e_ms else None),
        "autotune": tune,
        "components_total": int(res.num_cc.sum()),
        "clocks": clocks,
        "gpu_launches": int(prof["kernel_launches"]),
    }
    return line


SERVING = dict(workload="serving_t2000_v2e10-2e18_chunglu2.3_budget120GB", num_tenants=2000,
               trace_seed=7, budget_bytes=120 * 10**9, snapshot_bytes=40 * 10**9)


# The serving check of the default run: a short trace whose sketch demand exceeds the budget, so
# that tenants queue for admission while query latency is measured.
SERVING_SHORT = dict(num_tenants=400, trace_seed=11, budget_bytes=16 * 10**9,
                     snapshot_bytes=8 * 10**9, time_scale=5.0)
# records per tick of the saturated (throughput) replays; the paced ones use the replay's default,
# a smaller cap that bounds how long a released query waits behind one ingest call
SERVING_SAT_TICK = 1 << 21


def serving_short():
    """Paced replay of a 400-tenant serving trace through the batched server (continuous
    batching, in-place queries, ticks of at most 2^19 records with queries first) under a 16 GB
    sketch budget, and the same trace saturated through the batched server (ticks of up to 2^21
    records) and through the plain per-tenant path; answers must agree."""
    from graphzeppelin_b200 import serve as SV
    cfg = SERVING_SHORT
    tr = SV.serving_trace(cfg["num_tenants"], cfg["trace_seed"])
    demand = sum(SV.tenant_bytes(int(v)) for v in tr.num_vertices)
    kw = dict(snapshot_bytes=cfg["snapshot_bytes"])
    warm = SV.serving_trace(60, cfg["trace_seed"] + 1000)
    SV.replay(warm, "batched", cfg["budget_bytes"], time_scale=1e12, **kw)
    SV.replay(warm, "plain", cfg["budget_bytes"], time_scale=1e12, **kw)
    paced = SV.replay(tr, "batched", cfg["budget_bytes"], time_scale=cfg["time_scale"], **kw)
    sat = SV.replay(tr, "batched", cfg["budget_bytes"], time_scale=1e12,
                    max_tick_updates=SERVING_SAT_TICK, **kw)
    plain = SV.replay(tr, "plain", cfg["budget_bytes"], time_scale=1e12, **kw)
    if not (paced.answers == sat.answers == plain.answers):
        raise SystemExit("serving answers differ between the batched server and the plain path")
    p, s_, pl = paced.summary(), sat.summary(), plain.summary()
    return {"workload": f"serving_t{cfg['num_tenants']}_v2e10-2e18_chunglu2.3_budget16GB",
            "tenants": cfg["num_tenants"], "requests": int(tr.time.size), "updates": tr.num_updates,
            "budget_bytes": cfg["budget_bytes"], "sketch_demand_bytes": int(demand),
            "time_scale": cfg["time_scale"],
            "query_p50_ms": p["query_p50_ms"], "query_p99_ms": p["query_p99_ms"],
            "service_p50_ms": p["service_p50_ms"], "service_p99_ms": p["service_p99_ms"],
            "tenants_waited_for_budget": p["tenants_waited_for_budget"],
            "max_waiting_tenants": p["max_waiting_tenants"],
            "paced_updates_per_s": p["updates_per_s"],
            "saturated_updates_per_s": s_["updates_per_s"],
            "plain_path_updates_per_s": pl["updates_per_s"],
            "saturated_over_plain": s_["updates_per_s"] / max(pl["updates_per_s"], 1e-9),
            "paced_over_plain": p["updates_per_s"] / max(pl["updates_per_s"], 1e-9),
            "tick_records_paced": SV.REPLAY_TICK_RECORDS, "tick_records_saturated": SERVING_SAT_TICK,
            "answers_equal": True,
            "note": "query_* from release, service_* from release or admission; wall clock; "
                    "plain path = one CCSketchAlg per tenant, requests one at a time"}


def run_serving(args):
    """Serving loop: a seeded trace of tenants (V log-uniform 2^10..2^18, Chung-Lu endpoints,
    exponent 2.3) whose requests are update batches of 1k-64k records (20% deletions of live
    edges), connectivity queries and point queries, served by the batched server (continuous
    batching, in-place queries) and by the plain per-tenant CCSketchAlg path, both admitting
    tenants against a 120 GB sketch budget. Each arm runs the trace twice: paced (requests
    released at their arrival times, compressed by --time-scale) for query latency, and saturated
    (every request released at once) for throughput."""
    import numpy as np
    import torch

    from graphzeppelin_b200 import serve as SV

    torch.cuda.set_device(0)
    T = args.tenants or SERVING["num_tenants"]
    t = time.time()
    tr = SV.serving_trace(T, SERVING["trace_seed"])
    log(f"[serving] {T} tenants, {tr.time.size} requests, {tr.num_updates} updates "
        f"({tr.raw.size / 1e9:.2f} GB) over {tr.time[-1]:.1f} s of trace in {time.time() - t:.1f} s")
    # the request payloads are page-locked by each replay (outside its timing), as a server's
    # receive buffers would be
    budget = SERVING["budget_bytes"]
    kw = dict(snapshot_bytes=SERVING["snapshot_bytes"])
    arms = {}
    # warm-up (untimed): a 200-tenant trace of its own through both paths, so that module loading,
    # first allocations and pinned staging of this process are not charged to the measured replays
    warm = SV.serving_trace(200, SERVING["trace_seed"] + 1000)
    for mode in ("batched", "plain"):
        if mode == "plain" and args.no_plain:
            continue
        SV.replay(warm, mode, budget, time_scale=1e12, **kw)
    sampler = ClockSampler(0)
    sampler.start()
    for mode in ("batched", "plain"):
        if mode == "plain" and args.no_plain:
            continue
        paced = SV.replay(tr, mode, budget, time_scale=args.time_scale, **kw)
        sat = SV.replay(tr, mode, budget, time_scale=1e12, max_tick_updates=SERVING_SAT_TICK, **kw)
        arms[mode] = {"paced": paced, "saturated": sat}
        log(f"[serving] {mode}: paced {paced.summary()}; saturated {sat.summary()}")
        torch.cuda.empty_cache()
    clocks = sampler.stop()
    b = arms["batched"]
    equal = None
    if "plain" in arms:
        equal = (b["paced"].answers == arms["plain"]["paced"].answers ==
                 b["saturated"].answers == arms["plain"]["saturated"].answers)
    else:
        equal = b["paced"].answers == b["saturated"].answers
    if equal is False:
        raise SystemExit("batched and plain serving answers differ")
    sat = b["saturated"].summary()
    paced = b["paced"].summary()
    line = {
        "metric": "edge updates/sec + p50/p99 query ms, serving on 1 B200",
        "value": sat["updates_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": sat["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded serving trace: Poisson arrivals, Chung-Lu update batches)",
        "config": {"workload": SERVING["workload"] if T == 2000 else f"serving_t{T}",
                   "tenants": T, "requests": int(tr.time.size), "updates": tr.num_updates,
                   "budget_bytes": budget, "snapshot_bytes": SERVING["snapshot_bytes"],
                   "trace_seconds": float(tr.time[-1]), "time_scale": args.time_scale},
        "timing": "wall clock of the replay loop (host + GPU), from the first release to the "
                  "last answer, after an untimed 200-tenant warm-up replay",
        "batched": {"saturated": sat, "paced": paced},
        "plain_per_tenant": ({"saturated": arms["plain"]["saturated"].summary(),
                              "paced": arms["plain"]["paced"].summary()} if "plain" in arms else None),
        "answers_equal": equal,
        "query_p50_ms": paced["query_p50_ms"], "query_p99_ms": paced["query_p99_ms"],
        "service_p50_ms": paced["service_p50_ms"], "service_p99_ms": paced["service_p99_ms"],
        "admitted_tenants": paced["admitted_tenants"],
        "clocks": clocks,
    }
    return line


POWERLAW = dict(workload="powerlaw_v1048576_chunglu2.1_deg200_max16384_q10", num_vertices=1 << 20,
                exponent=2.1, mean_degree=200.0, max_degree=1 << 14, stream_seed=2, queries=10,
                sketch_seed=0x9E37)


# profiling case of the same kind: V = 2^18 (2.8 GB of sketches, 3.2e7 records)
POWERLAW_SMALL = dict(POWERLAW, workload="powerlaw_v262144_chunglu2.1_deg200_max16384_q10",
                      num_vertices=1 << 18)


def powerlaw_check(threads=None):
    """The power-law workload at full size (V = 2^20, 10 segments, a snapshot query after each),
    checked in the CPU-baseline leg: every snapshot answer equals the blocking query's at the same
    point, and the final partition equals the exact union-find over the stream's final edge set
    and the reference's connected_components (-DNO_EAGER_DSU build, src/cc_sketch_alg.cpp:515-557)
    over the whole stream, with the same Boruvka rounds."""
    import numpy as np
    import torch

    import graphzeppelin_b200 as gz
    from graphzeppelin_b200 import streams as S
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    cfg = POWERLAW
    V, Q = cfg["num_vertices"], cfg["queries"]
    t0 = time.perf_counter()
    st = S.chung_lu_stream_fast(V, cfg["exponent"], cfg["mean_degree"], cfg["max_degree"],
                                cfg["stream_seed"])
    n = st.num_updates
    d_rec = torch.from_numpy(st.raw()).cuda()
    cuts = np.linspace(0, n, Q + 1).astype(np.int64)
    alg = gz.CCSketchAlg(V, cfg["sketch_seed"])
    alg.set_gutter_capacity(2 * int(cuts[1] - cuts[0]) + 1024)
    base = d_rec.data_ptr()
    snap, tickets, final = [], [], None
    for k in range(Q):
        alg.ingest_records_device(base + 9 * int(cuts[k]), int(cuts[k + 1] - cuts[k]))
        tickets.append(alg.query_submit())
    for t in tickets:
        final, rounds = alg.query_wait(t)
        snap.append(final.size())
    alg.clear()
    block = []
    for k in range(Q):
        alg.ingest_records_device(base + 9 * int(cuts[k]), int(cuts[k + 1] - cuts[k]))
        block.append(alg.num_connected_components())
    labels = final.canonical_labels()
    alg.close()
    del d_rec
    torch.cuda.empty_cache()
    out = {"workload": cfg["workload"], "num_updates": n, "components_at_each_query": snap,
           "snapshot_equals_blocking": snap == block}
    n_exact, exact = O.exact_cc_mt(V, st.raw(), threads)
    out["exact_partition_equal"] = bool((labels == exact).all())
    out["components"] = {"gpu": snap[-1], "exact": n_exact}
    if O.have_reference():
        with tempfile.TemporaryDirectory() as td:
            spath, rlab = os.path.join(td, "stream.gzs"), os.path.join(td, "ref.labels")
            st.write(spath)
            ref = cpu_reference_run(st, cfg, n, threads, path=spath, eager=False, labels_path=rlab)
            rlabels = np.fromfile(rlab, np.uint32)
        out["reference_partition_equal"] = bool((labels == rlabels).all())
        out["rounds_equal"] = int(rounds) == int(ref["rounds"])
        out["rounds"] = {"gpu": int(rounds), "reference": int(ref["rounds"])}
        out["components"]["reference"] = int(ref["num_cc"])
    out["seconds"] = round(time.perf_counter() - t0, 1)
    return out


def many_graphs_check(num_graphs=64):
    """The many-graph engine checked graph by graph against the single-graph path on the
    many-graph workload's generator (the first num_graphs graphs' streams): each graph's sketch
    bytes (SHA-256 of its dump), partition and Boruvka rounds are the same."""
    import hashlib

    import numpy as np
    import torch

    import graphzeppelin_b200 as gz
    from graphzeppelin_b200 import streams as S
    t0 = time.perf_counter()
    Vs, seeds, raw, off = S.many_graph_streams(num_graphs, MANY["stream_seed"])
    d_rec = torch.from_numpy(raw).cuda()
    base = d_rec.data_ptr()
    b = gz.CCSketchBatch(Vs, seeds)
    b.ingest_device(base, off)
    res = b.connected_components(labels=True)
    same_sketch = same_labels = same_rounds = 0
    for g in range(num_graphs):
        a = gz.CCSketchAlg(int(Vs[g]), int(seeds[g]))
        cnt = int(off[g + 1] - off[g])
        if cnt:
            a.ingest_records_device(base + 9 * int(off[g]), cnt)
        cc = a.connected_components()
        h1 = hashlib.sha256(a.dump_sketches().tobytes()).hexdigest()
        h2 = hashlib.sha256(b.dump_sketches(g).tobytes()).hexdigest()
        same_sketch += h1 == h2
        same_labels += bool((cc.canonical_labels() == res.connected_components(g).canonical_labels()).all())
        same_rounds += int(a.last_query_rounds) == int(res.rounds[g])
        a.close()
    b.close()
    del d_rec
    torch.cuda.empty_cache()
    return {"graphs": num_graphs, "vertices": int(Vs.sum()), "num_updates": int(off[-1]),
            "sketch_sha256_equal": same_sketch == num_graphs,
            "partition_equal": same_labels == num_graphs, "rounds_equal": same_rounds == num_graphs,
            "graphs_equal": {"sketch": same_sketch, "partition": same_labels, "rounds": same_rounds},
            "seconds": round(time.perf_counter() - t0, 1)}


def run_powerlaw(args):
    """Power-law graph with interleaved queries: a Chung-Lu stream (V = 2^20, exponent 2.1, mean
    degree 200 after a 2^14 degree cap; shuffled inserts, deletes of 15% of them, re-inserts of
    half of those) ingested in 10 segments with a connectivity query after each. Arm
    "snapshot": each query runs on a device snapshot (gz_query_submit) while the next segment is
    ingested. Arm "blocking": each query (gz_connected_components) stops ingest until it ends.
    A step = clear + the whole stream with its 10 queries."""
    import numpy as np
    import torch

    import graphzeppelin_b200 as gz
    from graphzeppelin_b200 import streams as S

    torch.cuda.set_device(0)
    cfg = POWERLAW_SMALL if args.small else POWERLAW
    V, Q = cfg["num_vertices"], cfg["queries"]
    t = time.time()
    probe = S.chung_lu_stream_fast(V, cfg["exponent"], cfg["mean_degree"], cfg["max_degree"],
                                   cfg["stream_seed"])
    n = probe.num_updates
    pinned = torch.empty(n * 9, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = probe.raw()
    del probe
    host = pinned.numpy().view(S.RECORD_DTYPE)
    d_rec = pinned.cuda()
    torch.cuda.synchronize()
    log(f"[powerlaw] {n} records ({n * 9 / 1e9:.2f} GB) in {time.time() - t:.1f} s")
    cuts = np.linspace(0, n, Q + 1).astype(np.int64)
    alg = gz.CCSketchAlg(V, cfg["sketch_seed"])
    if args.host_rounds:
        alg.set_query_graph(False)
    if args.entry_form:
        alg.set_tuning(entry_form=args.entry_form)
    if args.pipeline is not None:
        alg.set_pipeline(args.pipeline)
    alg.set_gutter_capacity(2 * int(cuts[1] - cuts[0]) + 1024)
    base = d_rec.data_ptr()

    def step_snapshot(from_host=False):
        alg.clear()
        answers, tickets = [], []
        for k in range(Q):
            if from_host:
                alg.ingest_records(host[cuts[k]:cuts[k + 1]])
            else:
                alg.ingest_records_device(base + 9 * int(cuts[k]), int(cuts[k + 1] - cuts[k]))
            tickets.append(alg.query_submit())
            if k:
                answers.append(alg.query_wait(tickets[k - 1])[0].size())
        answers.append(alg.query_wait(tickets[-1])[0].size())
        return answers

    def step_blocking():
        alg.clear()
        answers = []
        for k in range(Q):
            alg.ingest_records_device(base + 9 * int(cuts[k]), int(cuts[k + 1] - cuts[k]))
            answers.append(alg.num_connected_components())
        return answers

    def timed(fn, steps):
        out, ms = None, []
        for _ in range(steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ms.append((time.perf_counter() - t0) * 1e3)
        return out, ms

    for _ in range(args.warmup):
        a_snap = step_snapshot()
        a_block = step_blocking()
    if a_snap != a_block:
        raise SystemExit(f"snapshot and blocking answers differ: {a_snap} vs {a_block}")
    sampler = ClockSampler(0)
    sampler.start()
    alg.set_profiling(True)
    a_snap, snap_ms = timed(step_snapshot, args.steps)
    prof = alg.get_profile()
    alg.set_profiling(True)  # resets the counters: the blocking arm's queries are timed here
    a_block, block_ms = timed(step_blocking, args.steps)
    prof_block = alg.get_profile()
    alg.set_profiling(False)
    clocks = sampler.stop()
    assert a_snap == a_block
    e2e_ms = []
    if not args.no_e2e:
        a_host, e2e_ms = timed(lambda: step_snapshot(from_host=True), max(1, min(args.steps, 3)))
        assert a_host == a_snap
    p = alg.params
    alg.close()
    ms = statistics.mean(snap_ms)
    return {
        "metric": "edge updates/sec with interleaved CC queries on 1 B200", "value": n / (ms / 1e3),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded Chung-Lu stream, C generator)",
        "config": {"workload": cfg["workload"], "num_vertices": V, "num_updates": n, "queries": Q,
                   "num_columns": p.num_columns, "bkt_per_col": p.bkt_per_col,
                   "sketch_bytes_total": V * p.sketch_bytes,
                   "l2": "inputs larger than L2 (GB of records and sketches)"},
        "timing": "wall clock between device synchronisations, whole stream with its queries",
        "snapshot_queries": {"ms_per_step": ms, "updates_per_s": n / (ms / 1e3),
                             "ingest_ms_per_step": (prof["gutter_ms"] + prof["sketch_update_ms"]) / args.steps},
        "blocking_queries": {"ms_per_step": statistics.mean(block_ms),
                             "updates_per_s": n / (statistics.mean(block_ms) / 1e3),
                             "query_ms": prof_block["query_ms"] / (args.steps * Q),
                             "ingest_ms_per_step": (prof_block["gutter_ms"] + prof_block["sketch_update_ms"]) / args.steps},
        "query_ms": prof_block["query_ms"] / (args.steps * Q),
        "components_at_each_query": a_snap,
        "e2e": ({"value": n / (max(e2e_ms) / 1e3), "unit": UNIT, "h2d_bytes_per_step": n * 9,
                 "d2h_bytes_per_step": Q * V * 4,
                 "note": "pinned host records -> gz_ingest_records in 10 segments, snapshot query "
                         "after each (labels to host); wall clock, max of steps"} if e2e_ms else None),
        "clocks": clocks,
        "gpu_launches": int(prof["kernel_launches"]),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--small", action="store_true",
                    help="profiling sizes: dense V=2^14, powerlaw V=2^18")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--entry-form", type=int, default=0, choices=[0, 1, 2, 3],
                    help="power-law workload: gutter entry form (0 the handle's choice, 1 plain, "
                         "2 coded, 3 coded with 3-bit depth codes)")
    ap.add_argument("--pipeline", type=int, default=None, choices=[-1, 0, 1, 2, 3, 4],
                    help="sketch-update kernel: 1 tile pipeline (2..4: with that many buffers), "
                         "0 one tile at a time, -1 the handle's choice (default)")
    ap.add_argument("--host-rounds", action="store_true",
                    help="queries with the Boruvka round loop on the host (profilers cannot see "
                         "kernels inside the conditional query graph)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-checks", action="store_true",
                    help="skip the full-size parity checks of the power-law and many-graph "
                         "workloads in the default run")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the short serving replay of the default run")
    ap.add_argument("--workload", default="dense",
                    choices=["dense", "many_graphs", "serving", "powerlaw"],
                    help="dense: one V=2^17 graph (the headline); many_graphs: 512 uneven graphs; "
                         "serving: 2000 tenants behind a 120 GB sketch budget; powerlaw: V=2^20 "
                         "Chung-Lu stream with 10 interleaved queries")
    ap.add_argument("--graphs", type=int, default=0, help="graphs of the many_graphs workload")
    ap.add_argument("--tenants", type=int, default=0, help="tenants of the serving workload")
    ap.add_argument("--time-scale", type=float, default=4.0,
                    help="serving: trace seconds per wall second in the paced replay")
    ap.add_argument("--no-autotune", action="store_true",
                    help="many_graphs: keep the default tiling instead of running the autotuner")
    ap.add_argument("--no-plain", action="store_true",
                    help="many_graphs / serving: skip the plain-path comparison")
    args = ap.parse_args()
    if args.warmup < 3 and not args.small:
        log("note: at least 3 warm-up steps are required for a valid number; using 3")
        args.warmup = 3
    cfg = SMALL if args.small else FULL
    if args.workload == "many_graphs":
        line = run_many_graphs(args)
    elif args.workload == "serving":
        line = run_serving(args)
    elif args.workload == "powerlaw":
        line = run_powerlaw(args)
    else:
        line = run_reference(args, cfg) if args.impl == "reference" else run_b200(args, cfg)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
