"""The bench line's roofline figures on the CPU: the DRAM traffic and FP64
FLOP per cell and stage come from the committed ncu summary, scale with the
event, and agree with the figures its text quotes."""
import json
import os
import re
import sys

import vahlib as V

sys.path.insert(0, V.ROOT)

import bench  # noqa: E402

PROFILE = os.path.join(V.ROOT, "profiles", "split_stage_dram.json")
SUMMARY = os.path.join(V.ROOT, "profiles", "split_stage_121x121x81.md")
CELLS = 121 * 121 * 81


def test_fp64_peak_is_the_vector_dfma_rate():
    assert abs(bench.FP64_PEAK_TFLOPS - 64 * 2 * 148 * 1.965e-3) < 1e-9


def test_roofline_figures_scale_with_the_event_and_match_the_summary():
    with open(PROFILE) as f:
        prof = json.load(f)
    with open(SUMMARY) as f:
        text = f.read()
    for prec in ("fp64", "fp32"):
        per_b = prof["dram_bytes_per_cell_per_stage"][prec]
        assert bench.traffic_per_launch(CELLS, "per_cell", prec) == per_b * CELLS
        assert bench.traffic_per_launch(2 * CELLS, "per_cell", prec) == 2 * per_b * CELLS
    # the text quotes the same per-cell traffic and FLOP count as the JSON
    assert f"= {round(prof['dram_bytes_per_cell_per_stage']['fp64'])} B per interior cell" in text
    assert f"{prof['fp64_flop_per_cell_per_stage']['fp64']} FP64 FLOP" in text
    # FP64 roofline of a 1 ms stage: FLOP per cell x cells / 1 ms, against the peak
    r = bench.fp64_roofline(CELLS, "per_cell", "fp64", 1e-3)
    flop = prof["fp64_flop_per_cell_per_stage"]["fp64"]
    assert abs(r["achieved"] - flop * CELLS / 1e-3 / 1e12) < 1e-9
    assert r["flop_per_cell_update"] == 2 * flop
    assert 0 < r["frac"] < 1 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    # no FLOP figure for the modes the summary does not cover
    assert bench.fp64_roofline(CELLS, "shared", "fp64", 1e-3) is None
    assert bench.fp64_roofline(CELLS, "fused", "fp64", 1e-3) is None
    assert re.search(r"\| cell_kernel<double, 2, 1, 1, 3> \| 4 \|", text)
