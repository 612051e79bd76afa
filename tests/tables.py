"""Reads the metric constant tables from vship_b200/csrc/metric_tables.h for the tests."""
import os
import re

import numpy as np

_HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "vship_b200", "csrc", "metric_tables.h")


def weights():
    text = open(_HDR).read()
    body = text[text.index("#define VSHIP_SSIMU2_WEIGHT_LIST"):text.index("static const double kSsimu2Weights")]
    vals = [float(v) for v in re.findall(r"-?\d+\.\d+(?:e-?\d+)?", body)]
    assert len(vals) == 108
    return np.array(vals)
