"""GPU parity against the reference itself: the unmodified Vship library, built from its own
sources for sm_100a (oracle/_ref/libvship_ref.so), scores the same inputs in the same
process through the same C ABI.

SSIMULACRA2: the reference's score equals, bit for bit, the FP32 restatement of its own
arithmetic (oracle/ssimu2_f32.c with CUDA's powf / cbrtf / expf); ours is within 1e-3 of the
exact FP64 metric.  The two differ by the reference's float rounding (up to ~1 on frames of a
few pixels, ~1e-3 at full HD), which the restatement reproduces exactly.

Butteraugli: our norms within 1e-4 relative of the reference's on every colour path whose
colour conversion is well conditioned; on the two PQ paths the reference's float PQ / ICtCp
arithmetic moves its norms by up to 4e-4, and there the reference equals FP64 Butteraugli on
the restatement's float colour values (1e-5) while ours equals FP64 on exact colour (1e-4).
"""
import os

import numpy as np
import pytest

from tests.golden.cases import CASES, build_case
from vship_b200 import api

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libvship_ref.so")
PQ_PATHS = {"b_yuv444p16_2020ncl_pq", "b_ictcp_pq_half"}


@pytest.fixture(scope="module")
def ref_lib(gpu):
    if not os.path.exists(REF):
        pytest.skip("reference library not built (oracle/build_ref.sh needs the reference sources)")
    return api.load_library(REF)


@pytest.fixture(scope="module")
def cuda_math_oracle(gpu, oracle_lib):
    oracle_lib.use_cuda_math(True)
    yield oracle_lib
    oracle_lib.use_cuda_math(False)


@pytest.mark.parametrize("case", [c for c in CASES if c["w"] * c["h"] <= 2_100_000], ids=lambda c: c["name"])
def test_matches_reference_library(gpu, ref_lib, cuda_math_oracle, case):
    o = cuda_math_oracle
    (p1, ls1, cs1), (p2, ls2, cs2) = build_case(case)
    if case["metric"] == "ssimu2":
        with api.SSIMU2(cs1, cs2) as mine:
            a = mine.compute(p1, p2, ls1, ls2)
        ref = api.SSIMU2(cs1, cs2, lib=ref_lib)
        b = ref.compute(p1, p2, ls1, ls2)
        ref.close()
        assert b == o.ssimu2_reference_arith(p1, ls1, cs1, p2, ls2, cs2), (case["name"], b)
        _, exact, _ = o.ssimu2(o.convert(p1, ls1, cs1), o.convert(p2, ls2, cs2))
        if case.get("identical"):
            assert a == 100.0
        else:
            assert abs(a - exact) <= 1e-3, (a, exact)
    else:
        with api.Butteraugli(cs1, cs2, qnorm=case["qnorm"], intensity=case["intensity"]) as mine:
            a, _ = mine.compute(p1, p2, ls1, ls2)
        ref = api.Butteraugli(cs1, cs2, qnorm=case["qnorm"], intensity=case["intensity"], lib=ref_lib)
        b, _ = ref.compute(p1, p2, ls1, ls2)
        ref.close()
        if case["name"] not in PQ_PATHS:
            for k in range(3):
                assert abs(a[k] - b[k]) <= 1e-4 * max(abs(b[k]), 1e-12), (k, a, b)
            return
        f1 = o.convert_f32(p1, ls1, cs1).astype(np.float64)
        f2 = o.convert_f32(p2, ls2, cs2).astype(np.float64)
        on_ref_colour, _ = o.butteraugli(f1, f2, case["intensity"], case["qnorm"])
        exact, _ = o.butteraugli(o.convert(p1, ls1, cs1), o.convert(p2, ls2, cs2), case["intensity"], case["qnorm"])
        for k in range(3):
            assert abs(b[k] - on_ref_colour[k]) <= 1e-5 * abs(on_ref_colour[k]), (k, b, on_ref_colour)
            assert abs(a[k] - exact[k]) <= 1e-4 * abs(exact[k]), (k, a, exact)
