"""Generates cvvdp_vectors.json: the CVVDP results the reference Vship library computes for
every sequence case of cvvdp_cases.py (one entry per operation: JOD scores, and distortion-map
statistics where the case asks for the map).

Runs only where the reference library built from its own sources (oracle/_ref/libvship_ref.so,
made by oracle/build_ref.sh) can execute, i.e. on a machine with a CUDA GPU:

    python -m tests.golden.make_golden_cvvdp [output.json]

The library is driven through its public C API (Vship_CVVDPInit3, Vship_ComputeCVVDP,
Vship_LoadTemporalCVVDP, Vship_ResetCVVDP, Vship_ResetScoreCVVDP).
"""
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.cvvdp_cases import CVVDP_CASES, run_library  # noqa: E402
from vship_b200 import api  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libvship_ref.so")


def main(out_path):
    L = api.load_library(REF_LIB)
    results = {}
    t0 = time.time()
    with tempfile.TemporaryDirectory() as d:
        for case in CVVDP_CASES:
            results[case["name"]] = run_library(case, lib=L, directory=d)
    with open(out_path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden_cvvdp.py", "library": "oracle/_ref/libvship_ref.so",
                   "cases": results}, f, indent=1)
    print("wrote %s (%d cases, %.1f s)" % (out_path, len(results), time.time() - t0))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "cvvdp_vectors.json"))
