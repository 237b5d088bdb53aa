"""Host-side checks of bench.py's roofline arithmetic (no GPU)."""
import importlib.util
import math
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_under_test"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_roofline_reports_the_busier_unit_and_scales_by_scanned_cells():
    b = load_bench()
    clocks = {"sm_mhz": 1965.0}
    t = 1.0e-4
    full = b.roofline(b.SL_CELLS_PER_LAUNCH, t, clocks)
    half = b.roofline(b.SL_CELLS_PER_LAUNCH // 2, t / 2, clocks)
    # achieved rates are counts per launch, scaled by the counted cells, over the launch time
    smem = b.SL_SMEM_WAVEFRONTS_PER_LAUNCH / t / 1e9
    alu = b.SL_ALU_WARP_INST_PER_LAUNCH / t / 1e9
    smem_peak = b.SM_COUNT * b.SMEM_WAVEFRONTS_PER_SM_CLK * 1965.0e6 / 1e9
    alu_peak = b.SM_COUNT * b.ALU_WARP_INST_PER_SM_CLK * 1965.0e6 / 1e9
    fr = {"smem": smem / smem_peak, "alu": alu / alu_peak}
    bound = max(fr, key=fr.get)
    assert full["bound"] == bound
    assert math.isclose(full["frac"], fr[bound], rel_tol=1e-9)
    other = "alu" if bound == "smem" else "smem"
    assert math.isclose(full[other]["frac"], fr[other], rel_tol=1e-9)
    # half the cells in half the time: the same rates
    assert math.isclose(half["frac"], full["frac"], rel_tol=1e-6)
    assert math.isclose(full["cells_per_s"], b.SL_CELLS_PER_LAUNCH / t, rel_tol=1e-12)


def test_counted_cells_per_cds():
    b = load_bench()
    # the upper triangle of pairs (r, c) with c - r >= 5: (n-5)(n-4)/2
    for n in (5, 6, 7, 100, 3003):
        k = n - 5
        assert b.hairpin_cells_per_cds(n) == (k * (k + 1) // 2 if k > 0 else 0)
    assert b.SL_CELLS_PER_LAUNCH == b.SL_CDS_PER_LAUNCH * b.hairpin_cells_per_cds(3003)
