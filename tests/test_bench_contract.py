"""The constants bench.py computes its roofline figures from (CPU).

The maps kernel's FLOP count and the algorithmic bytes of the SSIMULACRA2 kernels follow the
pyramid of the workload's 1920x1080 frames and the library's pruning of (plane, scale) maps.
These tests recompute both from the weight table the kernels use (a map is computed when the
weight of its 1-norm or 4-norm feature exceeds the pruning threshold), so the bench line's
figures cannot drift from what the kernels do.
"""
import importlib.util
import os
import re

from tests import tables

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
W, H = 1920, 1080


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _prune_threshold():
    text = open(os.path.join(ROOT, "vship_b200", "csrc", "metric_tables.h")).read()
    return float(re.search(r"#define VSHIP_SSIMU2_PRUNE ([0-9.]+)f", text).group(1))


def _planes_per_scale():
    w, prune = tables.weights(), _prune_threshold()
    out = []
    for scale in range(6):
        n = 0
        for plane in range(3):
            base = plane * 36 + scale * 6
            if any(w[base + m] > prune or w[base + 3 + m] > prune for m in range(3)):
                n += 1
        out.append(n)
    return out


def _levels(w, h):
    for _ in range(6):
        yield w, h
        w, h = (w - 1) // 2 + 1, (h - 1) // 2 + 1


def test_pruning_leaves_eleven_planes():
    assert _planes_per_scale() == [1, 2, 2, 3, 3, 0]


def test_maps_flop_count_follows_the_pyramid():
    tiles = sum(n * -(-w // 32) * -(-h // 32) for n, (w, h) in zip(_planes_per_scale(), _levels(W, H)))
    assert tiles == 3486
    assert _bench().maps_flop_per_pair(W, H) == tiles * 1024 * 370


def test_algorithmic_bytes_are_the_unpruned_planes():
    floats = sum(n * w * h for n, (w, h) in zip(_planes_per_scale(), _levels(W, H)))
    b = _bench()
    assert b.ALGO_BYTES["ssimu2_maps"] == 2 * 4 * floats == 27_930_240
    raw = 2 * (W * H * 2 + 2 * (W // 2) * (H // 2) * 2)
    assert b.ALGO_BYTES["ssimu2_front"] == raw + 2 * 4 * floats == 40_371_840
