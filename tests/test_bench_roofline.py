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
TILE_PROFILE = os.path.join(V.ROOT, "profiles", "tile_stage_dram.json")
TILE_SUMMARY = os.path.join(V.ROOT, "profiles", "tile_kernel_fp32_121x121x81.md")
CELLS = 121 * 121 * 81


def test_fp64_peak_is_the_vector_dfma_rate():
    assert abs(bench.FP64_PEAK_TFLOPS - 64 * 2 * 148 * 1.965e-3) < 1e-9


def test_roofline_figures_scale_with_the_event_and_match_the_summary():
    with open(PROFILE) as f:
        prof = json.load(f)
    with open(SUMMARY) as f:
        text = f.read()
    per_b = prof["dram_bytes_per_cell_per_stage"]["fp64"]
    assert bench.traffic_per_launch(CELLS, "per_cell", "fp64") == per_b * CELLS
    assert bench.traffic_per_launch(2 * CELLS, "per_cell", "fp64") == 2 * per_b * CELLS
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


def test_fp32_form_roofline_comes_from_the_tile_kernel_summary():
    """The FP32 form runs the tile kernel whatever the face option: its
    traffic and FP64 FLOP per cell and stage are the tile summary's."""
    with open(TILE_PROFILE) as f:
        prof = json.load(f)
    with open(TILE_SUMMARY) as f:
        text = f.read()
    per = prof["dram_bytes_per_cell_per_stage"]
    assert abs(per["mean"] - (per["stage1"] + per["stage2"]) / 2) < 0.05
    for flux in ("per_cell", "shared"):
        assert bench.traffic_per_launch(CELLS, flux, "fp32") == per["mean"] * CELLS
    assert f"| dram bytes per interior cell | {per['stage1']} B | {per['stage2']} B |" in text
    r = bench.fp64_roofline(CELLS, "per_cell", "fp32", 1e-3)
    assert r["flop_per_cell_update"] == 2 * prof["fp64_flop_per_cell_per_stage"]
    assert re.search(r"\| tile_kernel<2, 1> \| 4 \|", text)
