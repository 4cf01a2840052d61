"""bench.py's accounting on CPU: which transform each QC size takes, the
fp64 flop and butterfly counts of the QC report, and the LPN L1-wavefront
roofline model (no device needed)."""
import bench


def test_qc_leaves_follow_the_backend_split():
    assert [bench.qc_leaves(e) for e in (10, 16, 20, 21, 22)] == [1, 1, 1, 1, 1]
    assert bench.qc_leaves(23) == 3 and bench.qc_leaves(24) == 9
    assert bench.qc_leaves(25) == 0


def test_qc_work_counts():
    n = 1 << 20
    w = bench.qc_transform_work([n])
    # both roles, 32 four-plane transforms forward and inverse, 5 n log n each, + 6n products
    assert w == {"fft_fp64_flops": 2 * 32 * (2 * 5 * n * 20 + 6 * n), "ntt_butterflies": 0}
    m = 1 << 22
    w22 = bench.qc_transform_work([m])
    assert w22["fft_fp64_flops"] == 2 * 32 * (2 * 5 * m * 22 + 6 * m)
    assert bench.qc_transform_work([1 << 23])["fft_fp64_flops"] == 3 * w22["fft_fp64_flops"]
    w25 = bench.qc_transform_work([1 << 25])
    assert w25 == {"fft_fp64_flops": 0, "ntt_butterflies": 2 * 128 * 2 * (1 << 24) * 25}


def test_qc_report_rate_only_for_pure_fft():
    r = bench.qc_transform_report([1 << 20], 1.0)
    assert abs(r["fp64_tflops"] - r["fft_fp64_flops"] / 1e-3 / 1e12) < 1e-9
    assert "fp64_tflops" not in bench.qc_transform_report([1 << 20, 1 << 25], 1.0)
    assert "frac_of_measured" not in r
    m = bench.qc_transform_report([1 << 20], 1.0, fp64_peak=40.0)
    assert abs(m["frac_of_measured"] - m["fp64_tflops"] / 40.0) < 1e-12
    f = bench.fp64_roofline(m)
    assert f["peak"] == 40.0 and f["frac"] == m["frac_of_measured"] and f["unit"] == "TFLOP/s"
    assert bench.fp64_roofline(r) is None


def test_lpn_l1_roofline_model():
    class Props:
        multi_processor_count = 148
    # the dual-role kernel: one index computation per row pair, 2d gathers, both rows read and written
    r = bench.lpn_l1_roofline(2 * 10485760, 10, 1.275, {"sm_mhz": 1965.0}, Props())
    assert abs(r["wavefronts_per_row"] - ((145 * 10 + 15) / 4 / 32 + 2 * 10 + 0.5) / 2) < 1e-12
    assert abs(r["peak_rows_per_s"] - 148 * 1965e6 / r["wavefronts_per_row"]) < 1.0
    assert 0.85 < r["frac"] < 0.95
