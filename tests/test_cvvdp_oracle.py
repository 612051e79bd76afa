"""CPU checks of the CVVDP oracle and of the library's host-side CVVDP logic.

* The castleCSF table the library and the oracle share (vship_b200/csrc/cvvdp_csf_table.h) is
  regenerated from the reference's own table and must be identical (when the reference
  sources are present).
* The FP64 oracle (oracle/cvvdp.c) reproduces the JOD scores and distortion maps the
  reference library produced on a B200 for the seeded sequences of tests/golden/cvvdp_cases.py
  (committed in tests/golden/cvvdp_vectors.json by tests/golden/make_golden_cvvdp.py):
  |dJOD| <= 2e-4 (the reference computes in FP32).
* Display models (VshipExt_CVVDPDisplayModel, host only): built-in models, the JSON override
  and its errors, as src/cvvdp/display_models.hpp defines them.
* Oracle invariants: identical clips score exactly 10, and the temporal pooling follows the
  reference's formula (src/cvvdp/main.hpp:376-388).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from tests.golden.cvvdp_cases import CVVDP_CASES, run_oracle
from vship_b200 import api

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden", "cvvdp_vectors.json")
TABLE = os.path.join(ROOT, "vship_b200", "csrc", "cvvdp_csf_table.h")

JOD_TOL = 2e-4


def test_csf_table_matches_reference_source():
    from tests.golden import cvvdp_csf_table as gen
    src = gen.default_source()
    if not os.path.exists(src):
        pytest.skip("reference sources not present")
    assert gen.render(*gen.parse(src)) == open(TABLE).read()


@pytest.fixture(scope="module")
def golden():
    if not os.path.exists(GOLDEN):
        pytest.skip("cvvdp_vectors.json not generated yet")
    return json.load(open(GOLDEN))["cases"]


@pytest.mark.parametrize("case", CVVDP_CASES, ids=lambda c: c["name"])
def test_oracle_matches_reference_vectors(golden, case):
    if case["name"] not in golden:
        pytest.skip("no reference vectors for this case yet")
    want = golden[case["name"]]
    got = run_oracle(case)
    assert [e["op"] for e in got] == [e["op"] for e in want]
    for g, w in zip(got, want):
        if "score" in w:
            assert abs(g["score"] - w["score"]) <= JOD_TOL, (g["score"], w["score"])
        if "dmap" in w:
            assert abs(g["dmap"]["mean"] - w["dmap"]["mean"]) <= 1e-4 * max(1.0, abs(w["dmap"]["mean"]))
            for (x, y, a), (_, _, b) in zip(g["dmap"]["samples"], w["dmap"]["samples"]):
                assert abs(a - b) <= 2e-4, (x, y, a, b)


def test_identical_clips_score_ten():
    case = next(c for c in CVVDP_CASES if c["name"] == "c_identical")
    assert [e["score"] for e in run_oracle(case)] == [10.0, 10.0, 10.0]


def _to_jod(a):
    a = np.float32(a)
    if a > np.float32(0.1):
        return float(np.float32(10.0) - np.float32(0.0439569391310215) * np.float32(a ** np.float32(0.9302042722702026)))
    return float(10.0 - 0.0439569391310215 * 0.1 ** (0.9302042722702026 - 1.0) * a)


def test_temporal_pooling_formula():
    """JOD after frame k from the per-frame pooled values q_0..q_k: q_0 * image_int for the
    first frame, then sqrt(sum(q^2) / k) (the frame counter before its increment)."""
    rng = np.random.default_rng(5)
    o = oracle.CVVDP(80, 64, 24.0)
    a = rng.random((3, 64, 80))
    qs, scores = [], []
    for k in range(5):
        b = np.clip(a + (0.02 + 0.01 * k) * rng.standard_normal(a.shape), 0, 1)
        scores.append(o.frame(a, b))
        qs.append(o.bands()[1])
    for k, s in enumerate(scores):
        resq = qs[0] * 0.577918291091919 if k == 0 else np.sqrt(np.sum(np.square(qs[:k + 1])) / k)
        assert abs(s - _to_jod(resq)) < 1e-5, (k, s, _to_jod(resq))


def test_reset_semantics():
    """ResetScore keeps the ring, Reset empties it: a reset handler scores like a fresh one."""
    rng = np.random.default_rng(6)
    frames = [(rng.random((3, 48, 64)), rng.random((3, 48, 64))) for _ in range(4)]
    o = oracle.CVVDP(64, 48, 24.0)
    for a, b in frames[:3]:
        o.frame(a, b)
    o.reset()
    after_reset = o.frame(*frames[3])
    fresh = oracle.CVVDP(64, 48, 24.0)
    assert after_reset == fresh.frame(*frames[3])
    o2 = oracle.CVVDP(64, 48, 24.0)
    for a, b in frames[:3]:
        o2.frame(a, b)
    o2.reset(only_score=True)
    first_after = o2.frame(*frames[3])
    assert abs(first_after - _to_jod(o2.bands()[1] * 0.577918291091919)) < 1e-5
    assert first_after != after_reset  # the ring still holds the earlier frames


def test_filter_taps():
    o = oracle.CVVDP(64, 48, 24.0)
    f = o.filters()
    assert o.taps == 7 and f.shape == (4, 7)
    np.testing.assert_allclose(f, f[:, ::-1], atol=1e-7)  # symmetric taps
    assert oracle.CVVDP(64, 48, 60.0).taps == 17


# ---- display models (host-side code of the library; no GPU needed) --------------------------

def test_builtin_displays():
    fhd = api.cvvdp_display("standard_fhd")
    assert (fhd["width"], fhd["height"], fhd["hdr"]) == (1920, 1080, 0)
    assert abs(fhd["ppd"] - 37.8425) < 1e-3
    assert abs(fhd["black_level"] - 0.2) < 1e-6 and abs(fhd["reflected_level"] - 250 * 0.005 / np.pi) < 1e-5
    k4 = api.cvvdp_display("standard_4k")
    assert abs(k4["ppd"] - 75.4025) < 1e-3
    for name in ("standard_hdr_pq", "standard_hdr_hlg", "standard_hdr_linear", "standard_hdr_dark",
                 "standard_hdr_linear_zoom"):
        d = api.cvvdp_display(name)
        assert d["hdr"] == 1 and (d["width"], d["height"]) == (3840, 2160)
    assert api.cvvdp_display("standard_hdr_linear_zoom")["max_luminance"] == 10000.0
    assert api.cvvdp_display("standard_hdr_dark")["E_ambient"] == 0.0


def _code(fn):
    with pytest.raises(api.VshipError) as e:
        fn()
    return e.value.code


def test_display_json(tmp_path):
    p = str(tmp_path / "displays.json")
    mine = {"name": "x", "colorspace": "BT.2020-PQ", "resolution": [2560, 1440], "viewing_distance_meters": 0.5,
            "diagonal_size_inches": 27, "max_luminance": 400, "contrast": 5000, "E_ambient": 50, "exposure": 2}
    json.dump({"other": {"resolution": [1, 2], "nested": {"a": "}"}}, "mine": mine}, open(p, "w"), indent=2)
    d = api.cvvdp_display("mine", p)
    assert (d["width"], d["height"], d["hdr"], d["exposure"], d["k_refl"]) == (2560, 1440, 1, 2.0, np.float32(0.005))
    # a built-in name present in the file is overridden field by field
    json.dump({"standard_fhd": {"max_luminance": 350}}, open(p, "w"))
    d = api.cvvdp_display("standard_fhd", p)
    assert d["max_luminance"] == 350.0 and d["width"] == 1920
    # a built-in name absent from the file keeps its values
    assert api.cvvdp_display("standard_4k", p)["width"] == 3840


def test_display_errors(tmp_path):
    p = str(tmp_path / "d.json")
    assert _code(lambda: api.cvvdp_display("no_such_display")) == api.abi.BadDisplayModel
    json.dump({"mine": {"resolution": [640, 480]}}, open(p, "w"))
    assert _code(lambda: api.cvvdp_display("mine", p)) == api.abi.BadDisplayModel  # missing fields
    assert _code(lambda: api.cvvdp_display("absent", p)) == api.abi.BadDisplayModel
    json.dump({"mine": {"resolution": [640, 480], "refresh_rate": 60}}, open(p, "w"))
    assert _code(lambda: api.cvvdp_display("mine", p)) == api.abi.BadJson
    json.dump({"mine": {"colorspace": "P3"}}, open(p, "w"))
    assert _code(lambda: api.cvvdp_display("mine", p)) == api.abi.BadJson
    open(p, "w").write('{"mine": {"resolution": [640, 480]')
    assert _code(lambda: api.cvvdp_display("mine", p)) == api.abi.BadJson
    assert _code(lambda: api.cvvdp_display("mine", p + ".missing")) == api.abi.BadPath
