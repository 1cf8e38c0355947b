"""CPU checks of the figures bench.py puts in its JSON line: the roofline arithmetic of the ingest
path (per record: 1 + C hashes, 9 B of stream, the touched sketches read and written once), and
the committed per-launch DRAM traffic that fills roofline.traffic."""
import bench


class _Params:
    num_vertices = 1 << 17
    num_columns = 24
    bkt_per_col = 34
    sketch_bytes = 9804
    entry_form = 2


class _Alg:
    params = _Params()


def test_roofline_arithmetic():
    n = 139_997_155
    prof = {"gutter_ms": 30.0, "gutter_launches": 10, "sketch_update_ms": 25.0,
            "sketch_update_launches": 10}
    ingest_ms = [6.0, 6.0]
    r = bench.roofline(_Alg(), n, prof, 10, ingest_ms, hash_peak=1358e9, hbm_peak_gbs=6550.4,
                       update_peak=3667e9)
    hashes = n * 25  # one hash per record per column, plus the checksum: hashed once per edge
    assert r["units_per_launch"]["hashes"] == hashes
    assert r["units_per_launch"]["bytes"] == 9 * n + 2 * (1 << 17) * 9804
    # the hash term (3.5e9 hashes at 1358 G/s = 2.58 ms) is slower than the HBM term (0.58 ms)
    assert r["bound"] == "int"
    assert abs(r["achieved"] - hashes / 6e-3 / 1e9) < 1e-6
    assert abs(r["frac"] - (hashes / 1358e9) / 6e-3) < 1e-12
    assert abs(r["terms_ms"]["int"] - hashes / 1358e9 * 1e3) < 1e-9
    g, u = r["kernels"]["gutter"], r["kernels"]["sketch_update"]
    assert g["hashes_per_launch"] == n * 24 and abs(g["launch_ms"] - 3.0) < 1e-12
    assert u["hashes_per_launch"] == 2 * n
    assert u["slot_steps_per_launch"] == 2 * n * 32
    assert u["bucket_updates_per_launch"] == 2 * n * 25
    assert abs(u["smem"]["frac"] - (2 * n * 32 / 2.5e-3) / 3667e9) < 1e-12


def test_committed_traffic_is_per_step_of_each_workload():
    traffic = bench.load_traffic(bench.FULL["workload"])
    if traffic is None:
        return
    n, V, sb = 139_997_155, 1 << 17, 9804
    algorithmic = 9 * n + 2 * V * sb
    # DRAM bytes of the ingest kernels of one step: the coded entries (16 B per endpoint) are
    # written and read once on top of the path's algorithmic bytes
    assert algorithmic < traffic < algorithmic + 2 * 2 * n * 16 * 1.1
