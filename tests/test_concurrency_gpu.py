"""Concurrent use of the C ABI, and CVVDP / SSIMULACRA2 edge cases, on the GPU.

* Handlers of all three metrics driven from several host threads at once (each handler by one
  thread, as the ABI requires) give exactly the results of the same calls made one after
  another: engines share no state, and every handler's work stays on its own stream.
* CVVDP at the frame rates that give the shortest rings (1 and 3 frames) matches the FP64 oracle.
* A 3840x2160 SSIMULACRA2 pair matches the FP64 oracle within the metric's tolerance.
"""
import threading

import numpy as np
import pytest

import oracle
from tests.golden.cases import colorspace_of
from tests.golden.cvvdp_cases import build_frame, run_library, run_oracle
from vship_b200 import abi, api, synth

pytestmark = pytest.mark.gpu


def _ssimu2_job(frames, cs):
    def run():
        with api.SSIMU2(cs) as h:
            return [h.compute(a, b, ls) for a, b, ls in frames]
    return run


def _butter_job(frames, cs):
    def run():
        with api.Butteraugli(cs, qnorm=5, intensity=203.0) as h:
            return [h.compute(a, b, ls, distmap=True)[0] for a, b, ls in frames]
    return run


def _cvvdp_job(case):
    cs = colorspace_of(case)

    def run():
        with api.CVVDP(cs, fps=case["fps"], model="standard_fhd") as h:
            out = []
            for t in range(6):
                (p1, ls1), (p2, ls2) = build_frame(case, t)
                out.append(h.compute(p1, p2, ls1, ls2))
            return out
    return run


def test_concurrent_handlers_match_sequential(gpu):
    w, h = 640, 360
    cs = abi.srgb8(w, h)
    frames = [(a, b, ls) for a, b, ls in synth.make_pairs(6, w, h, fmt="rgb8", seed=5, unique=6)]
    cv = [dict(name="cc%d" % k, w=160, h=120, seed=300 + k, fps=24.0, ops="c" * 6, step=14.0) for k in range(2)]
    jobs = [_ssimu2_job(frames, cs), _ssimu2_job(frames[::-1], cs), _butter_job(frames[:3], cs),
            _butter_job(frames[3:], cs), _cvvdp_job(cv[0]), _cvvdp_job(cv[1])]
    sequential = [job() for job in jobs]
    results = [None] * len(jobs)
    errors = []

    def runner(i):
        try:
            for _ in range(3):  # repeat so that the threads' calls interleave
                r = jobs[i]()
                if results[i] is None:
                    results[i] = r
                elif r != results[i]:
                    errors.append((i, "repeat differs"))
        except Exception as e:  # reported below, on the main thread
            errors.append((i, repr(e)))

    threads = [threading.Thread(target=runner, args=(i,)) for i in range(len(jobs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for i, (got, want) in enumerate(zip(results, sequential)):
        assert got == want, (i, got, want)


@pytest.mark.parametrize("fps,taps", [(0.0, 1), (8.0, 3)])
def test_cvvdp_short_rings_match_oracle(gpu, tmp_path, fps, taps):
    case = dict(name="ring%d" % taps, w=112, h=72, seed=140 + taps, fps=fps, ops="ccccc", step=16.0)
    got = run_library(case, directory=str(tmp_path))
    want = run_oracle(case)
    with api.CVVDP(colorspace_of(case), fps=fps) as h:
        assert h.geometry()[1] == taps
    for g, w in zip(got, want):
        assert abs(g["score"] - w["score"]) <= 1e-4, (g, w)


def test_ssimu2_4k_matches_oracle(gpu, oracle_lib):
    p1, p2, ls = synth.make_pairs(1, 3840, 2160, fmt="rgb8", seed=41, unique=1)[0]
    cs = abi.srgb8(3840, 2160)
    with api.SSIMU2(cs) as h:
        score = h.compute(p1, p2, ls)
    _, exact, _ = oracle_lib.ssimu2(oracle_lib.convert(p1, ls, cs), oracle_lib.convert(p2, ls, cs))
    assert abs(score - exact) <= 1e-3, (score, exact)
