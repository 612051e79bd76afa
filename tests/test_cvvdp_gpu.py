"""GPU parity of the CVVDP path through the C ABI.

Every seeded sequence of tests/golden/cvvdp_cases.py (SDR and HDR displays, 8/10/16-bit and
float inputs, 4:2:0 chroma, crop, display downscale and upscale, 24/30/60 fps rings,
LoadTemporal / Reset / ResetScore, distortion maps) is run through this library and compared
with
  * the FP64 oracle (oracle/cvvdp.c): |dJOD| <= 1e-4 per scored frame; distortion maps within
    2e-4 absolute (maps are 1 - JOD/10 per pixel);
  * the reference library built from its own sources (oracle/_ref/libvship_ref.so) on the same
    GPU, live, and its committed results (tests/golden/cvvdp_vectors.json): |dJOD| <= 2e-4.
Plus: identical clips score exactly 10, geometry (bands, ring length, distortion-map size)
agrees with the oracle, and the error paths of Init / Compute.
"""
import json
import os

import numpy as np
import pytest

import oracle
from tests.golden.cases import colorspace_of
from tests.golden.cvvdp_cases import CVVDP_CASES, build_frame, run_library, run_oracle
from vship_b200 import abi, api

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libvship_ref.so")
GOLDEN = os.path.join(HERE, "golden", "cvvdp_vectors.json")

ORACLE_TOL = 1e-4
REF_TOL = 2e-4


def _compare(got, want, tol, map_tol):
    assert [e["op"] for e in got] == [e["op"] for e in want]
    worst = 0.0
    for g, w in zip(got, want):
        if "score" in w:
            worst = max(worst, abs(g["score"] - w["score"]))
            assert abs(g["score"] - w["score"]) <= tol, (g["score"], w["score"])
        if "dmap" in w:
            for (x, y, a), (_, _, b) in zip(g["dmap"]["samples"], w["dmap"]["samples"]):
                assert abs(a - b) <= map_tol, (x, y, a, b)
            assert abs(g["dmap"]["mean"] - w["dmap"]["mean"]) <= map_tol
    return worst


@pytest.mark.parametrize("case", CVVDP_CASES, ids=lambda c: c["name"])
def test_cases_match_oracle(gpu, tmp_path, case):
    got = run_library(case, directory=str(tmp_path), keep_maps=True)
    want = run_oracle(case, keep_maps=True)
    _compare(got, want, ORACLE_TOL, 2e-4)
    for g, w in zip(got, want):
        if "map" in w:
            np.testing.assert_allclose(g["map"], w["map"], rtol=0, atol=2e-4)


@pytest.fixture(scope="module")
def ref_lib(gpu):
    if not os.path.exists(REF):
        pytest.skip("reference library not built (oracle/build_ref.sh needs the reference sources)")
    return api.load_library(REF)


@pytest.mark.parametrize("case", CVVDP_CASES, ids=lambda c: c["name"])
def test_cases_match_reference_library(gpu, ref_lib, tmp_path, case):
    got = run_library(case, directory=str(tmp_path))
    want = run_library(case, lib=ref_lib, directory=str(tmp_path))
    _compare(got, want, REF_TOL, 5e-4)


@pytest.mark.parametrize("case", CVVDP_CASES, ids=lambda c: c["name"])
def test_cases_match_golden_vectors(gpu, tmp_path, case):
    if not os.path.exists(GOLDEN):
        pytest.skip("cvvdp_vectors.json not generated yet")
    golden = json.load(open(GOLDEN))["cases"]
    if case["name"] not in golden:
        pytest.skip("no reference vectors for this case yet")
    want = golden[case["name"]]
    _compare(run_library(case, directory=str(tmp_path)), want, REF_TOL, 5e-4)


def test_identical_is_ten(gpu, tmp_path):
    case = next(c for c in CVVDP_CASES if c["name"] == "c_identical")
    assert [e["score"] for e in run_library(case, directory=str(tmp_path))] == [10.0, 10.0, 10.0]


@pytest.mark.parametrize("size,fps,display,resize", [
    ((128, 96), 24.0, "standard_fhd", False),
    ((1920, 1080), 60.0, "standard_fhd", False),
    ((3840, 2160), 30.0, "standard_4k", False),
    ((3840, 2160), 24.0, "standard_fhd", True),
    ((640, 360), 25.0, "standard_fhd", True),
])
def test_geometry_matches_oracle(gpu, size, fps, display, resize):
    cs = abi.srgb8(*size)
    with api.CVVDP(cs, fps=fps, model=display, resize_to_display=resize) as h:
        bands, ring = h.geometry()
        dims = h.distmap_resolution()
    o = oracle.CVVDP(size[0], size[1], fps, display=display, resize_to_display=resize)
    assert (bands, ring, dims) == (o.levels, o.taps, tuple(o.resize))


def test_errors(gpu, tmp_path):
    cs = abi.srgb8(64, 48)
    with pytest.raises(api.VshipError) as e:
        api.CVVDP(cs, model="not_a_display")
    assert e.value.code == abi.BadDisplayModel
    with pytest.raises(api.VshipError) as e:
        api.CVVDP(cs, abi.srgb8(64, 40))
    assert e.value.code == abi.DifferingInputType
    with pytest.raises(api.VshipError) as e:
        api.CVVDP(abi.srgb8(3, 64))
    assert e.value.code == abi.BadErrorType
    case = dict(name="e", w=64, h=48, seed=1, fps=24.0, ops="c")
    (p1, ls1), (p2, ls2) = build_frame(case, 0)
    with api.CVVDP(colorspace_of(case)) as h:
        a1, k1 = api.planes_arg(p1)
        a2, k2 = api.planes_arg(p2)
        out = np.zeros((48, 64), np.float32)
        import ctypes
        score = ctypes.c_double()
        rc = h.L.Vship_ComputeCVVDP(h.h, ctypes.byref(score), out.ctypes.data, 63 * 4, a1, a2,
                                    abi.LineSizes(*ls1), abi.LineSizes(*ls2))
        assert rc == abi.BadPointer
        assert np.isfinite(h.compute(p1, p2, ls1, ls2))  # the handler stays usable
