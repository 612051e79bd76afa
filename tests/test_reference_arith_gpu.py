"""The reference library's SSIMULACRA2 scores reproduced exactly by the FP32 restatement of
its arithmetic (oracle/ssimu2_f32.c) when the restatement takes its powf / cbrtf / expf values
from CUDA itself (oracle/cuda_math.cu on this GPU).

The committed golden scores (tests/golden/reference_vectors.json) come from the unmodified
reference built with nvcc for sm_100a.  They differ from the exact (FP64) metric by up to 0.96
on tiny frames and ~1e-3 at full HD, because the reference forms the SSIM map in float with
cancelling terms (src/ssimu2/score.hpp:232-274).  This test shows that difference is the
reference's float arithmetic and nothing else: same operations, same roundings, same fused
multiply-adds, same transcendental results give the same score, to the last bit of the float
the reference returns, on every colour path, size and resize of the golden set.
"""
import json
import os

import pytest

from tests.golden.cases import build_case

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.json")


@pytest.fixture(scope="module")
def cuda_math_oracle(gpu, oracle_lib):
    oracle_lib.use_cuda_math(True)
    yield oracle_lib
    oracle_lib.use_cuda_math(False)


def _cases():
    with open(GOLDEN) as f:
        return [c for c in json.load(f)["cases"] if c["metric"] == "ssimu2"]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_fp32_restatement_reproduces_reference_score(cuda_math_oracle, case):
    (p1, ls1, cs1), (p2, ls2, cs2) = build_case(case)
    got = cuda_math_oracle.ssimu2_reference_arith(p1, ls1, cs1, p2, ls2, cs2)
    assert got == case["score"], (case["name"], got, case["score"])
