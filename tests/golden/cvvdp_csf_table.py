"""Writes cvvdp_csf_table.h: the contrast-sensitivity table CVVDP is defined with.

The table is sampled data of the castleCSF model as the reference ships it
(src/cvvdp/csf_lut_weber.hpp: background luminances L_bkg[32] in cd/m^2, spatial frequencies
rho[32] in cycles/degree, and log10 sensitivities D2LUT[4 channels][32 luminances][32
frequencies]).  It cannot be recomputed bit for bit from the model's formulas, so the values
are carried over as data: each decimal literal is rounded the way the reference's compiler
rounds it (to double, then to the float array element) and written as an exact hexadecimal
float literal.

Test tooling: it reads the reference's sources and writes the library's header
vship_b200/csrc/cvvdp_csf_table.h; nothing in the library runs it.

Usage: python -m tests.golden.cvvdp_csf_table [path/to/csf_lut_weber.hpp]
(default: $VSHIP_REFERENCE_ROOT/src/cvvdp/csf_lut_weber.hpp, VSHIP_REFERENCE_ROOT defaulting
to /root/reference).  tests/test_cvvdp_oracle.py regenerates the header from the same file,
when it is present, and checks that the committed one is identical.
"""
import os
import re
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(ROOT, "vship_b200", "csrc", "cvvdp_csf_table.h")


def default_source():
    root = os.environ.get("VSHIP_REFERENCE_ROOT", "/root/reference")
    return os.path.join(root, "src", "cvvdp", "csf_lut_weber.hpp")


def _numbers(text):
    return [float(t) for t in re.findall(r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?", text)]


def parse(path):
    """Returns (lum[32], rho[32], logs[4*32*32]) as Python floats rounded to float32."""
    src = open(path).read()
    out = {}
    for name, count in (("L_bkg", 32), ("rho", 32), ("D2LUT", 4 * 32 * 32)):
        m = re.search(r"\b%s\s*(\[[^=]*)=\s*\{" % name, src)
        if m is None:
            raise ValueError("array %s not found in %s" % (name, path))
        body, depth, i = [], 0, m.end() - 1
        while True:
            ch = src[i]
            depth += ch == "{"
            depth -= ch == "}"
            body.append(ch)
            i += 1
            if depth == 0:
                break
        vals = _numbers("".join(body))
        if len(vals) != count:
            raise ValueError("%s: %d values, expected %d" % (name, len(vals), count))
        out[name] = [struct.unpack("<f", struct.pack("<f", v))[0] for v in vals]
    return out["L_bkg"], out["rho"], out["D2LUT"]


def hexf(v):
    mant, exp = float(v).hex().split("p")
    mant = mant.rstrip("0").rstrip(".") if "." in mant else mant
    return "%sp%sf" % (mant, exp)


def render(lum, rho, logs):
    lines = [
        "// Generated by cvvdp_csf_table.py: castleCSF table of CVVDP, exact float values of",
        "// src/cvvdp/csf_lut_weber.hpp.  Do not edit by hand.",
        "// Plain C arrays (C99 hexadecimal literals) so that C and C++ code can both include it.",
        "#pragma once",
        "",
        "#ifdef __cplusplus",
        "namespace vship {",
        "namespace cvvdp_tables {",
        "#endif",
        "",
        "// Background luminance axis (cd/m^2), 32 log-spaced samples.",
        "static const float kCsfLum[32] = {",
    ]
    lines += ["    %s," % hexf(v) for v in lum]
    lines += ["};", "", "// Spatial frequency axis (cycles/degree), 32 log-spaced samples.", "static const float kCsfRho[32] = {"]
    lines += ["    %s," % hexf(v) for v in rho]
    lines += ["};", "",
              "// log10 sensitivity [channel: Y sustained, RG, YV, Y transient][luminance][frequency].",
              "static const float kCsfLogS[4][32][32] = {"]
    for c in range(4):
        lines.append("    {")
        for i in range(32):
            row = logs[(c * 32 + i) * 32:(c * 32 + i + 1) * 32]
            lines.append("        {" + ", ".join(hexf(v) for v in row) + "},")
        lines.append("    },")
    lines += ["};", "", "#ifdef __cplusplus", "}  // namespace cvvdp_tables", "}  // namespace vship", "#endif", ""]
    return "\n".join(lines)


def main(argv):
    src = argv[1] if len(argv) > 1 else default_source()
    text = render(*parse(src))
    with open(OUT, "w") as f:
        f.write(text)
    print("wrote", OUT)


if __name__ == "__main__":
    main(sys.argv)
