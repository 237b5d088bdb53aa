"""Host-side checks of bench.py's roofline arithmetic and of the ncu counts it
uses (no GPU)."""
import hashlib
import importlib.util
import math
import re
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PROFILES = {"hairpin": ROOT / "profiles" / "k_sl_L1000_m8_N1024.md",
            "lrcs": ROOT / "profiles" / "k_sl_lrcs_L3000_m4_N4096.md"}


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_under_test"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("kind", ["hairpin", "lrcs"])
def test_roofline_reports_the_busiest_unit_and_scales_by_scans(kind):
    b = load_bench()
    c = b.SL_NCU[kind]
    clocks = {"sm_mhz": 1965.0}
    t = 1.0e-4
    full = b.roofline(c["scans"], c["cells"], t, clocks, kind)
    half = b.roofline(c["scans"] / 2, c["cells"] / 2, t / 2, clocks, kind)
    # achieved rates are counts per launch, scaled by the scans run, over the launch time
    hz = 1965.0e6
    fr = {"issue": c["warp_inst"] / t / (b.SM_COUNT * b.ISSUE_WARP_INST_PER_SM_CLK * hz),
          "alu": c["alu_warp_inst"] / t / (b.SM_COUNT * b.ALU_WARP_INST_PER_SM_CLK * hz),
          "smem": c["smem_wavefronts"] / t / (b.SM_COUNT * b.SMEM_WAVEFRONTS_PER_SM_CLK * hz)}
    bound = max(fr, key=fr.get)
    assert full["bound"] == bound
    assert math.isclose(full["frac"], fr[bound], rel_tol=1e-9)
    for other in fr:
        if other != bound:
            assert math.isclose(full[other]["frac"], fr[other], rel_tol=1e-9)
    # half the scans in half the time: the same rates
    assert math.isclose(half["frac"], full["frac"], rel_tol=1e-6)
    assert math.isclose(full["cells_per_s"], c["cells"] / t, rel_tol=1e-12)
    assert math.isclose(full["traffic"], c["dram_bytes"], rel_tol=1e-12)


def test_counted_cells_per_cds():
    b = load_bench()
    # the upper triangle of pairs (r, c) with c - r >= 5: (n-5)(n-4)/2
    for n in (5, 6, 7, 100, 3003):
        k = n - 5
        assert b.hairpin_cells_per_cds(n) == (k * (k + 1) // 2 if k > 0 else 0)
    assert b.SL_NCU["hairpin"]["cells"] == 2311 * b.hairpin_cells_per_cds(3003)


@pytest.mark.parametrize("kind", ["hairpin", "lrcs"])
def test_ncu_constants_equal_the_committed_profile(kind):
    """bench.py's counts are the ones the committed profile summary reports."""
    b = load_bench()
    line = next(x for x in PROFILES[kind].read_text().splitlines() if x.startswith("bench: "))
    got = dict(kv.split("=") for kv in line[len("bench: "):].split())
    c = b.SL_NCU[kind]
    for k, v in got.items():
        if k == "source":
            assert c[k] == v
        else:
            assert math.isclose(float(c[k]), float(v), rel_tol=0, abs_tol=1e-9), k


def test_ncu_constants_match_the_kernel_source():
    """The counts were captured from the current kernel source: any change to the
    string-objective kernel's section needs a new capture (and new constants)."""
    b = load_bench()
    src = (ROOT / "protein_encoding_v2_nsga-iii_b200" / "csrc" / "pe_eval.cu").read_text()
    i = src.index("// k_sl: hairpin-stem scan on bit planes")
    digest = hashlib.sha256(src[i:].encode()).hexdigest()[:16]
    for kind, c in b.SL_NCU.items():
        assert c["source"] == digest, f"{kind}: k_sl source changed since its ncu capture"
