"""Consistency of the bench's roofline constants with the committed ncu
summaries (CPU only): the DRAM traffic per point that bench.py reports as
`roofline.traffic` must be the figure of the summary it comes from, and the
algorithmic bytes must follow the per-point state the kernels read and write.
"""
import os
import re
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

# summary of the capture each traffic constant comes from
SOURCES = {
    ("ensemble", "fp64"): "k_g2p2g_ensemble96_fp64.md",
    ("ensemble", "mixed"): "k_g2p2g_ensemble96_mixed.md",
    ("column", "fp64"): "k_g2p2g_column_fp64.md",
    ("column", "mixed"): "k_g2p2g_column_mixed.md",
}


def _summary_bytes_per_point(name):
    text = open(os.path.join(ROOT, "profiles", name)).read()
    m = re.search(r"\*\*([0-9.]+) B per point\*\*", text)
    assert m, f"{name}: no DRAM bytes per point"
    return float(m.group(1))


def _summary_algorithmic(name):
    text = open(os.path.join(ROOT, "profiles", name)).read()
    m = re.search(r"algorithmic bytes \| ([0-9]+) \+ 112 x ([0-9.]+) active nodes per point = ([0-9.]+) B", text)
    return None if m is None else (float(m.group(1)), float(m.group(2)), float(m.group(3)))


def test_every_traffic_constant_has_a_summary():
    assert set(bench.TRAFFIC_BYTES_PER_POINT) == set(SOURCES)


@pytest.mark.parametrize("key", sorted(SOURCES))
def test_traffic_constant_matches_its_summary(key):
    assert bench.TRAFFIC_BYTES_PER_POINT[key] == pytest.approx(_summary_bytes_per_point(SOURCES[key]), abs=0.05)


@pytest.mark.parametrize("key", sorted(SOURCES))
def test_algorithmic_bytes_match_the_summaries(key):
    alg = _summary_algorithmic(SOURCES[key])
    assert alg is not None
    base, ratio, total = alg
    mixed = key[1] == "mixed"
    assert base == (192.0 if mixed else 276.0)
    assert bench.bytes_per_point_step(ratio, mixed) == pytest.approx(total, abs=0.05)


def test_algorithmic_bytes_per_form():
    # FP64: read x, v (24 each), m, V (8 each), sigma (48), u (24), extent (8),
    # active (4); written x, v, V, sigma, u
    fp64 = (24 + 24 + 8 + 8 + 48 + 24 + 8 + 4) + (24 + 24 + 8 + 48 + 24)
    # mixed: x, x_t, m in two FP32 words, the rest FP32
    mixed = (24 + 24 + 8 + 4 + 24 + 12 + 4 + 4) + (24 + 24 + 4 + 24 + 12)
    assert bench.bytes_per_point_step(0.0) == fp64 == 276
    assert bench.bytes_per_point_step(0.0, mixed=True) == mixed == 192
    assert bench.bytes_per_point_step(1.0) - bench.bytes_per_point_step(0.0) == 112
