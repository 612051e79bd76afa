"""Generates reference_vectors.json: the scores the reference Vship library computes for every
case of cases.py.

Runs only where the reference library built from its own sources (oracle/_ref/libvship_ref.so,
made by oracle/build_ref.sh) can execute, i.e. on a machine with a CUDA GPU:

    python -m tests.golden.make_golden [output.json]

The library is driven through its public C API (Vship_SSIMU2Init2 / Vship_ComputeSSIMU2 /
Vship_ButteraugliInit2 / Vship_ComputeButteraugli).  For Butteraugli a fixed sample of the
distortion map is stored as well.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.cases import CASES, build_case  # noqa: E402
from vship_b200 import api  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libvship_ref.so")


def main(out_path):
    L = api.load_library(REF_LIB)
    results = []
    t0 = time.time()
    for case in CASES:
        (p1, ls1, cs1), (p2, ls2, cs2) = build_case(case)
        entry = dict(case)
        if case["metric"] == "ssimu2":
            h = api.SSIMU2(cs1, cs2, gpu_id=0, lib=L)
            entry["score"] = h.compute(p1, p2, ls1, ls2)
            h.close()
        else:
            h = api.Butteraugli(cs1, cs2, qnorm=case["qnorm"], intensity=case["intensity"], gpu_id=0, lib=L)
            norms, dmap = h.compute(p1, p2, ls1, ls2, distmap=True)
            h.close()
            entry["norms"] = list(norms)
            flat = dmap.reshape(-1)
            idx = np.random.default_rng(case["seed"]).choice(flat.size, size=min(64, flat.size), replace=False)
            idx.sort()
            entry["distmap_sample"] = {"index": idx.tolist(), "value": [float(v) for v in flat[idx]]}
        results.append(entry)
        print(case["name"], entry.get("score", entry.get("norms")), flush=True)
    doc = {
        "generator": "tests/golden/make_golden.py",
        "library": "Vship 4.1.0 reference, built by oracle/build_ref.sh (nvcc, sm_100a)",
        "seconds": round(time.time() - t0, 2),
        "cases": results,
    }
    with open(out_path, "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote", out_path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_vectors.json"))
