"""Host arithmetic of bench.py (no GPU): the algorithmic word count per
cell-step, the words of the fused kernel families, and the roofline of the
dominant family from per-family event times."""
import json
import os

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_words_per_cell_step():
    # phases A 15, B 6 + 7 + 8, C 4, D 4 + 4 + 2, E 7, F 9 per substep
    assert sum(bench.WORDS.values()) == 66
    assert bench.WORDS_PER_CELL_STEP == 198
    assert bench.WORDS_PER_CELL_STEP * 8 == 1584


def test_family_words_of_fused_kernels():
    fused = {"rhs": (1.0, 3), "uppres": (1.0, 3)}
    assert bench.family_words("rhs", fused) == 15 + 6  # the theta sweep runs inside
    assert bench.family_words("uppres", fused) == 9 + 7  # upsol runs inside
    apart = {"rhs": (1.0, 3), "tsweep": (1.0, 3), "uppres": (1.0, 3), "upsol": (1.0, 3)}
    assert bench.family_words("rhs", apart) == 15
    assert bench.family_words("uppres", apart) == 9
    assert bench.family_words("zsweep", fused) == 8
    # the forward theta transform takes divq from dq when divq is not timed apart
    assert bench.family_words("fft", {"fft": (1.0, 6)}) == 4 + 4
    assert bench.family_words("fft", {"fft": (1.0, 6), "divq": (1.0, 3)}) == 4


def test_roofline_of_the_dominant_field_family():
    steps, ncell = 10, 256 * 128 * 512
    # per-family (total ms, launches) over the timed steps; the particles take
    # the most time but carry no field words, so the right-hand side leads
    prof = {"part": (18.0, 2 * steps), "rhs": (15.0, 3 * steps), "uppres": (11.0, 3 * steps),
            "dct": (4.0, 6 * steps), "zsweep": (7.5, 9 * steps)}
    r = bench.roofline(prof, steps, ncell, 6500.0, "measured", {"rhs": 1.97e9}, 7.3)
    assert r["kernel"] == "rhs"
    per_launch_ms = 15.0 / (3 * steps)
    algo = 21 * 8 * ncell  # one launch per substep covers 21 words per cell
    assert r["algorithmic_bytes_per_launch"] == pytest.approx(algo)
    assert r["achieved"] == pytest.approx(algo / (per_launch_ms / 1e3) / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6500.0)
    assert r["traffic"] == 1.97e9
    floor_ms = 1584 * ncell / 6500e9 * 1e3
    assert r["step_frac"] == pytest.approx(floor_ms / 7.3)
    # a family launched several times per substep spreads its words over them
    prof2 = {"zsweep": (9.0, 9 * steps)}
    r2 = bench.roofline(prof2, steps, ncell, 6500.0, "measured", {}, 7.3)
    assert r2["algorithmic_bytes_per_launch"] == pytest.approx(8 / 3 * 8 * ncell)
    assert r2["traffic"] is None


def test_peaks_and_traffic_tables_are_readable():
    peak, kind = bench.peaks()
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        assert kind == "measured" and peak == float(d["hbm_gbs"])
    else:
        assert kind == "fallback"
    t = bench.traffic_table()
    assert t.get("rhs", 0) > 0 and t.get("uppres", 0) > 0
