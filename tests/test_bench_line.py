"""bench.py's roofline object for each kind of dominant kernel, built from
synthetic profile counters on the CPU: the keys the JSON line carries, the
fraction as achieved / peak, and the deferred-update traffic scaled by the
entries the launches update."""
import math

import pytest

import bench

PEAKS = {"hbm_gbs": 6555.2, "bf16_tflops": 1640.3}
ARM = {"factor_ms": 44.0}


def _check(roof, bound, unit):
    assert roof["bound"] == bound and roof["unit"] == unit
    assert roof["achieved"] > 0 and roof["peak"] > 0
    assert math.isclose(roof["frac"], roof["achieved"] / roof["peak"])
    assert "traffic" in roof and roof["kernel"]


def test_deferred_update_dominant():
    prof = {"gemm_ms": 20.0, "schur_ms": 5.0, "defer_bytes": 402 * 40e6, "gemm_launches": 402,
            "defer_updates": 1352, "defer_small": 0, "tc_ms": 0.0, "panel_ms": 18.0}
    roof = bench.dominant_roofline(prof, "fp64", ARM, PEAKS)
    _check(roof, "hbm", "GB/s")
    assert math.isclose(roof["achieved"], 402 * 40e6 / 15e-3 / 1e9)
    # 40 MB of algorithmic traffic per launch = 2.5 M entries at 13.7 bytes
    assert math.isclose(roof["traffic"], bench.DEFER_DRAM_BYTES_PER_ENTRY * 2.5e6)
    assert roof["peak_source"].startswith("MEASURED_PEAKS.json")


def test_tensor_core_dominant():
    prof = {"gemm_ms": 1.0, "schur_ms": 1.0, "tc_ms": 4.0, "tc_flops": 2e12, "tc_passes": 10}
    roof = bench.dominant_roofline(prof, "mixed", ARM, PEAKS)
    _check(roof, "tensor", "TFLOP/s")
    assert math.isclose(roof["peak"], 1640.3 / 2 / 3)


def test_fp64_update_dominant():
    prof = {"gemm_ms": 3.0, "schur_ms": 3.0, "gemm_flops": 1e11, "gemm_launches": 7}
    roof = bench.dominant_roofline(prof, "fp64", ARM, PEAKS, dgemm_peak=lambda: 50.0)
    _check(roof, "tensor", "TFLOP/s")
    assert roof["peak"] == 50.0


@pytest.mark.parametrize("peaks", [PEAKS, {}], ids=["measured", "fallback"])
def test_small_fronts_only(peaks):
    prof = {"arena_bytes": 4.28e9}
    roof = bench.dominant_roofline(prof, "fp64", ARM, peaks)
    _check(roof, "hbm", "GB/s")
    assert roof["traffic"] is None
    assert roof["peak"] == (6555.2 if peaks else 6650.0)


def test_solves_dominant():
    """Four solves a step (one, three refinement) outweigh the factor's
    kernels: the solves are the named kernel, against HBM."""
    prof = {"gemm_ms": 6.0, "schur_ms": 0.3, "defer_bytes": 1e9, "gemm_launches": 40, "tc_ms": 3.8,
            "tc_flops": 1e12, "tc_passes": 5, "panel_ms": 19.0}
    solve = {"ms": 9.3, "count": 4, "bytes": 1.51e9}
    roof = bench.dominant_roofline(prof, "mixed", ARM, PEAKS, solve=solve)
    _check(roof, "hbm", "GB/s")
    assert math.isclose(roof["achieved"], 1.51e9 / 9.3e-3 / 1e9)
    assert roof["kernel_ms"]["solves"] == 4 * 9.3
