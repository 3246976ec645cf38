"""Host arithmetic of bench.py that needs no GPU: the roofline of the
dominant kernel reported for each workload."""
import bench
from matter_tests_b200.abi import default_params


def test_roofline_picks_the_slowest_kernel_and_divides_its_bytes_by_its_time():
    p = default_params(3, 2)
    Np, Ga, G = 1_000_000, 150_000, 180_000
    kms = {"k_p2g": 0.30, "k_g2p": 0.50, "k_grid": 0.03, "memset(v2)": 0.9}  # memsets are not kernels
    r = bench.roofline_of(kms, p, Np, Ga, G, 8.0)
    assert r["kernel"] == "k_g2p" and r["bound"] == "hbm" and r["unit"] == "GB/s"
    b = bench.kernel_bytes("k_g2p", p, Np, Ga, G, 8.0)
    assert r["kernel_algorithmic_bytes"] == b
    assert abs(r["achieved"] - b / 0.5e-3 / 1e9) < 1e-9 * r["achieved"]
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert r["active_nodes"] == Ga and r["grid_nodes"] == G


def test_mixed_kernels_count_four_bytes_per_value_except_positions():
    p = default_params(3, 2)
    b8 = bench.kernel_bytes("k_p2g", p, 1000, 0, 0, 8.0)
    b4 = bench.kernel_bytes("k_p2g", p, 1000, 0, 0, 4.0)
    assert b8 > b4 > b8 / 2  # positions stay FP64 on the mixed path


def test_capture_figures_are_used_only_on_the_kernel_sources_they_were_taken_on(monkeypatch):
    """profiles/dram_traffic.json: DRAM bytes and pipe utilisation of the C2
    tile kernels, reported while the kernel headers hash as at capture."""
    for prec in ("fp64", "mixed"):
        for k in ("k_p2g", "k_g2p_musl", "k_defgrad"):
            b, src = bench.measured_traffic("collapse3d_mui", 1.0, k, prec)
            assert b and b > 0 and src.startswith("ncu capture"), (k, prec, src)
            pipes = bench.measured_pipes("collapse3d_mui", 1.0, k, prec)
            assert 0 < pipes["issue_active_pct"] <= 100 and pipes["top_stalls"]
    assert bench.measured_pipes("incline3d_mcc", 1.0, "k_g2p", "fp64") is None
    monkeypatch.setattr(bench, "kernel_source_hash", lambda: "0" * 16)
    b, why = bench.measured_traffic("collapse3d_mui", 1.0, "k_p2g", "fp64")
    assert b is None and "predates" in why
    assert bench.measured_pipes("collapse3d_mui", 1.0, "k_p2g", "fp64") is None
