"""CPU checks of the figures bench.py puts in its JSON line: the roofline arithmetic of the
sketch-update kernel, and the committed per-launch DRAM traffic that fills roofline.traffic."""
import bench


class _Params:
    num_vertices = 1 << 17
    num_columns = 24
    sketch_bytes = 9804


class _Alg:
    params = _Params()


def test_roofline_terms_arithmetic():
    n = 139_997_155
    t_launch = 0.01406
    terms, bound = bench.roofline_terms(_Alg(), n, t_launch, hash_peak=676e9, hbm_peak_gbs=6550.4,
                                        update_peak=857e9)
    entries = 2 * n
    assert terms["hbm"]["bytes_per_launch"] == entries * 8 + 2 * (1 << 17) * 9804
    assert terms["int"]["hashes_per_launch"] == entries * 25
    assert terms["smem_atomic"]["bucket_updates_per_launch"] == entries * 25
    for k, peak in (("int", 676.0), ("smem_atomic", 857.0)):
        assert abs(terms[k]["frac"] - terms[k]["achieved"] / peak) < 1e-12
    # the bound is the term with the longest ideal time: 7.0e9 hashes at 676 G/s
    assert bound == "int"
    assert 0.70 < terms["int"]["frac"] < 0.80


def test_committed_traffic_is_per_launch_of_each_workload():
    for cfg, n, V, sb in ((bench.FULL, 139_997_155, 1 << 17, 9804),
                        (bench.SMALL, 7_863_052, 1 << 14, 6396)):
        traffic = bench.load_traffic(cfg["workload"])
        assert traffic is not None and traffic > 0, cfg["workload"]
        algorithmic = 2 * n * 8 + 2 * V * sb
        # DRAM bytes of one launch: no re-reads, and at most the sketches' L2-resident share less
        assert 0.8 * algorithmic < traffic < 1.05 * algorithmic, (cfg["workload"], traffic, algorithmic)
