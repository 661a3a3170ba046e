"""bench.py host helpers on the CPU: the clock sampler's fallback without a
GPU and the grid roofline's work counts (no GPU needed)."""
import bench


def test_clock_sampler_without_a_gpu_reports_instead_of_raising():
    cs = bench.ClockSampler(0)
    cs.start()
    out = cs.stop()
    assert set(out) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    # no device here: no clock, and no throttle reason invented
    assert out["sm_mhz"] is None or out.get("samples", 0) > 0


def test_grid_roofline_counts_the_documented_work():
    nmb, R = 8160, 32
    out = bench._grid_roofline(nmb, R, {"sad": 0.5, "satd": 4.0}, 18000.0)
    cands = nmb * (2 * R + 1) ** 2
    assert out["sad"]["ops"] == cands * 128  # 2 lane ops per 4 pixels of a 16x16 candidate
    assert out["satd"]["ops"] == cands * 16 * 112  # 112 ops per 4x4 Hadamard block
    assert abs(out["sad"]["frac"] - out["sad"]["achieved"] / 18000.0) < 1e-3
    assert out["kernels"] == {"sad": "fullpel_sad_kernel", "satd": "fullpel_satd_kernel"}
