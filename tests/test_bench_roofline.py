"""The benchmark's roofline arithmetic (bench.roofline): the top kernel of a
profile, its algorithmic bytes (components x real size x owned cells, the
allocated range for the primitive-variable pass), achieved GB/s and the
fraction of the peak, and the committed DRAM traffic figure it scales."""
import pytest


def test_roofline_of_the_top_kernel():
    import bench

    prof = {"k_fluid": 2.0, "k_bface": 0.1, "k_sync": 5.0}  # k_sync is not a roofline kernel
    cells = [(32, 32, 32), (16, 16, 64)]
    r = bench.roofline(prof, cells, 6000.0, "measured", precision=1)
    owned = 32 ** 3 + 16 * 16 * 64
    algo = bench.kernel_bytes_per_cell("k_fluid", 1) * owned
    assert r["kernel"] == "k_fluid" and r["algo_bytes_per_launch"] == algo
    assert r["achieved"] == pytest.approx(algo / 2e-3 / 1e9, rel=1e-3)
    assert r["frac"] == pytest.approx(r["achieved"] / 6000.0, abs=1e-4)
    assert r["share_of_step"] == pytest.approx(2.0 / 7.1, abs=1e-4)
    assert r["traffic"] is None


def test_primitive_pass_counts_its_allocated_range():
    import bench

    r = bench.roofline({"k_pv_uplus": 1.0}, [(8, 8, 8)], 6000.0, "measured", precision=0)
    assert r["algo_bytes_per_launch"] == bench.kernel_bytes_per_cell("k_pv_uplus", 0) * 16 ** 3


def test_traffic_from_the_committed_ncu_summary():
    import bench

    per_cell = bench.load_traffic("k_fluid_mixed_ensemble")
    assert per_cell and per_cell > 0
    r = bench.roofline({"k_fluid": 1.0}, [(10, 10, 10)], 6000.0, "measured", precision=1,
                       traffic_key="k_fluid_mixed_ensemble")
    assert r["traffic"] == int(per_cell * 1000)


def test_replicas_value():
    import bench

    assert bench.replicas_value(4, 1_000_000, 10, 100.0) == pytest.approx(400.0)
