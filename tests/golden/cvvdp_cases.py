"""Seeded CVVDP sequence cases shared by the golden-vector generator and the parity tests.

A case is a small dict: clip size and colourspace (the fields of cases.colorspace_of), frame
rate, display model (built-in name, or a custom display written to a JSON file), whether
frames are resized to the display, and a list of operations on one handler:
  "c"  Vship_ComputeCVVDP (a score is recorded)
  "d"  Vship_ComputeCVVDP with the distortion map (score and map statistics recorded)
  "l"  Vship_LoadTemporalCVVDP
  "r"  Vship_ResetCVVDP
  "s"  Vship_ResetScoreCVVDP
Frames move (the content field slides by a few pixels per frame) and the distortion varies
over time, so the temporal channels carry signal.  build_frame() regenerates the exact bytes.
"""
import json
import os

import numpy as np

from tests.golden.cases import _encode, _plane_field, colorspace_of
from vship_b200 import abi, synth

YUV = dict(family=abi.ColorYUV)


def _field(seed, pw, ph, extra):
    rng = np.random.default_rng(seed)
    return _plane_field(rng, pw + extra, ph + extra)


def build_frame(case, t):
    """Frame t of the case -> ((planes1, line_sizes1), (planes2, line_sizes2)) raw bytes."""
    cs = colorspace_of(case)
    speed = case.get("speed", 2)
    extra = speed * 64 + 8
    step = case.get("step", 16.0) * (1.0 + 0.35 * np.sin(0.9 * t + case["seed"]))
    ref, dist = [], []
    for c, (pw, ph) in enumerate(cs.plane_dims()):
        f = _field(case["seed"] * 10 + c, pw, ph, extra)
        off = (speed * t) % (extra - 4)
        f = f[off // 2: off // 2 + ph, off: off + pw]
        if case.get("identical"):
            d = f
        else:
            d = synth.dct_quantize(f[None] * 255.0, step)[0] / 255.0
            if case.get("flicker") and t % 2:
                d = np.clip(d * 0.97 + 0.01, 0.0, 1.0)
        ref.append(_encode(f, cs, c != 0))
        dist.append(_encode(d, cs, c != 0))
    out = []
    for planes in (ref, dist):
        ls = [p.shape[1] * p.itemsize for p in planes]
        out.append(([np.ascontiguousarray(p).view(np.uint8).reshape(p.shape[0], -1) for p in planes], ls))
    return out[0], out[1]


def display_json(case, directory):
    """Writes the case's custom display (if any) to a JSON file; returns (model key, path or None)."""
    disp = case.get("display", "standard_fhd")
    if isinstance(disp, str):
        return disp, None
    path = os.path.join(directory, case["name"] + "_display.json")
    with open(path, "w") as f:
        json.dump({"other_display": {"resolution": [640, 480]}, "custom": disp}, f)
    return "custom", path


def oracle_model(case):
    """The display as the oracle's model vector (see oracle.CVVDP_DISPLAYS)."""
    import oracle
    disp = case.get("display", "standard_fhd")
    if isinstance(disp, str):
        return oracle.CVVDP_DISPLAYS[disp]
    hdr = 1 if disp["colorspace"] in ("HDR", "BT.2020-PQ", "BT.2020-HLG") else 0
    return (disp["resolution"][0], disp["resolution"][1], hdr, disp["viewing_distance_meters"],
            disp["diagonal_size_inches"], disp["max_luminance"], disp["contrast"], disp["E_ambient"],
            disp.get("k_refl", 0.005), disp.get("exposure", 1.0))


SMALL_SDR = dict(name="small", colorspace="sRGB", resolution=[160, 90], viewing_distance_meters=0.5,
                 diagonal_size_inches=10.0, max_luminance=250.0, contrast=800.0, E_ambient=100.0)

CVVDP_CASES = [
    dict(name="c_rgb8_srgb_128x96", w=128, h=96, seed=101, fps=24.0, ops="cccccccc", step=14.0),
    dict(name="c_yuv420p10_bt709_160x90", w=160, h=90, seed=102, fps=30.0, ops="cccccc", step=16.0,
         sample=abi.SampleUINT10, range=abi.RangeLimited, subw=1, subh=1, loc=abi.ChromaLoc_Left,
         matrix=abi.MATRIX_BT709, trc=abi.TRC_BT709, display="standard_4k", **YUV),
    dict(name="c_rgb16_pq_2020_hdr", w=120, h=72, seed=103, fps=24.0, ops="ccccc", step=12.0,
         sample=abi.SampleUINT16, trc=abi.TRC_PQ, prim=abi.PRIMARIES_BT2020, display="standard_hdr_pq"),
    dict(name="c_float_linear_hdr", w=96, h=64, seed=104, fps=24.0, ops="cccc", step=12.0,
         sample=abi.SampleFLOAT, trc=abi.TRC_Linear, display="standard_hdr_linear", flicker=True),
    dict(name="c_rgb8_flicker_60fps", w=96, h=72, seed=105, fps=60.0, ops="cccccccccc", step=10.0, flicker=True),
    dict(name="c_ops_reset", w=96, h=64, seed=106, fps=24.0, ops="cclccscclrcc", step=18.0),
    dict(name="c_distmap", w=112, h=80, seed=107, fps=24.0, ops="cdcd", step=16.0),
    dict(name="c_identical", w=96, h=64, seed=108, fps=24.0, ops="ccc", identical=True),
    dict(name="c_crop", w=140, h=100, seed=109, fps=24.0, ops="ccc", step=16.0, crop=[4, 6, 2, 10]),
    dict(name="c_resize_down", w=320, h=180, seed=110, fps=24.0, ops="ccc", step=16.0, display=SMALL_SDR,
         resize=True),
    dict(name="c_resize_up", w=80, h=45, seed=111, fps=24.0, ops="cccd", step=16.0, display=SMALL_SDR,
         resize=True),
    dict(name="c_yuv420p10_crop_resize_down", w=352, h=208, seed=112, fps=25.0, ops="cccd", step=16.0,
         sample=abi.SampleUINT10, range=abi.RangeLimited, subw=1, subh=1, loc=abi.ChromaLoc_Left,
         matrix=abi.MATRIX_BT709, trc=abi.TRC_BT709, crop=[6, 6, 16, 16], display=SMALL_SDR, resize=True, **YUV),
    dict(name="c_yuv444p12_hlg_2020", w=128, h=80, seed=113, fps=30.0, ops="cccc", step=14.0,
         sample=abi.SampleUINT12, range=abi.RangeLimited, matrix=abi.MATRIX_BT2020_NCL, trc=abi.TRC_HLG,
         prim=abi.PRIMARIES_BT2020, display="standard_hdr_hlg", **YUV),
]


def frame_count(case):
    return sum(1 for o in case["ops"] if o in "cdl")


def _dmap_summary(dmap):
    h, w = dmap.shape
    rng = np.random.default_rng(w * 7919 + h)
    pts = [(int(rng.integers(0, w)), int(rng.integers(0, h))) for _ in range(16)]
    return {"mean": float(np.mean(dmap)), "max": float(np.max(dmap)),
            "samples": [[x, y, float(dmap[y, x])] for x, y in pts]}


def run_library(case, lib=None, directory=None, gpu_id=0, keep_maps=False):
    """Runs the case's operations through a Vship-ABI library (this one, or the reference's
    when `lib` is its handle).  Returns one entry per operation."""
    import tempfile
    from vship_b200 import api
    directory = directory or tempfile.mkdtemp(prefix="cvvdp_case_")
    key, path = display_json(case, directory)
    cs = colorspace_of(case)
    h = api.CVVDP(cs, cs, fps=case["fps"], resize_to_display=case.get("resize", False), model=key,
                  model_config_json=path, gpu_id=gpu_id, lib=lib)
    out, t = [], 0
    try:
        for op in case["ops"]:
            if op in "cdl":
                (p1, ls1), (p2, ls2) = build_frame(case, t)
                t += 1
            if op == "c":
                out.append({"op": op, "score": h.compute(p1, p2, ls1, ls2)})
            elif op == "d":
                score, dmap = h.compute(p1, p2, ls1, ls2, distmap=True)
                e = {"op": op, "score": score, "dmap": _dmap_summary(dmap)}
                if keep_maps:
                    e["map"] = dmap
                out.append(e)
            elif op == "l":
                h.load_temporal(p1, p2, ls1, ls2)
                out.append({"op": op})
            elif op == "r":
                h.reset()
                out.append({"op": op})
            elif op == "s":
                h.reset_score()
                out.append({"op": op})
    finally:
        h.close()
    return out


def run_oracle(case, keep_maps=False):
    """The same operations through the FP64 oracle (oracle/cvvdp.c)."""
    import oracle
    cs = colorspace_of(case)
    ow, oh = cs.out_dims()
    o = oracle.CVVDP(ow, oh, case["fps"], display=oracle_model(case), resize_to_display=case.get("resize", False),
                     trc=(cs.transferFunction, cs.transferFunction), primaries=(cs.primaries, cs.primaries))
    out, t = [], 0
    try:
        for op in case["ops"]:
            if op in "cdl":
                (p1, ls1), (p2, ls2) = build_frame(case, t)
                t += 1
                lin1 = oracle.convert_native(p1, ls1, cs)
                lin2 = oracle.convert_native(p2, ls2, cs)
            if op == "c":
                out.append({"op": op, "score": o.frame(lin1, lin2)})
            elif op == "d":
                score, dmap = o.frame(lin1, lin2, distmap=True)
                e = {"op": op, "score": score, "dmap": _dmap_summary(dmap)}
                if keep_maps:
                    e["map"] = dmap
                out.append(e)
            elif op == "l":
                o.frame(lin1, lin2, compute=False)
                out.append({"op": op})
            elif op == "r":
                o.reset()
                out.append({"op": op})
            elif op == "s":
                o.reset(only_score=True)
                out.append({"op": op})
    finally:
        o.close()
    return out
