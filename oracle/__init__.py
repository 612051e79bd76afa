"""FP64 CPU oracle of the SSIMULACRA2 / Butteraugli path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and reference legs may
import this package; the product (vship_b200) never does.  The C restatement lives in
oracle.c (each function cites the reference file:line it follows) and is compiled with gcc
into liboracle.so by build().
"""
import ctypes
import os
import subprocess

import numpy as np

from vship_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libvship_ref.so")
_lib = None


def build(force=False):
    """Compile oracle.c (gcc, OpenMP).  Needs only gcc; runs here and on the GPU box."""
    src = os.path.join(HERE, "oracle.c")
    hdr = os.path.join(os.path.dirname(HERE), "vship_b200", "csrc", "metric_tables.h")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return LIB_PATH
    tmp = LIB_PATH + ".tmp"
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-std=c11",
                           "-fvisibility=hidden", "-o", tmp, src, "-lm"])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def build_reference():
    """Compile the reference library from its own sources (only where they are mounted)."""
    script = os.path.join(HERE, "build_ref.sh")
    subprocess.check_call(["bash", script])
    return REF_LIB_PATH if os.path.exists(REF_LIB_PATH) else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_convert.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(abi.Colorspace), dp]
        L.oracle_convert.restype = ctypes.c_int
        L.oracle_ssimu2.argtypes = [dp, dp, ctypes.c_int64, ctypes.c_int64, dp, dp, dp]
        L.oracle_ssimu2_final.argtypes = [dp, ctypes.c_int]
        L.oracle_ssimu2_final.restype = ctypes.c_double
        L.oracle_butteraugli.argtypes = [dp, dp, ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                         ctypes.c_int, dp, dp]
        L.oracle_blur.argtypes = [dp, dp, ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_int]
        L.oracle_downsample.argtypes = [dp, ctypes.c_int64, ctypes.c_int64, dp]
        L.oracle_positive_xyb.argtypes = [dp, ctypes.c_int64]
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def convert(planes, line_sizes, cs):
    """Raw planes (bytes-like / uint8 arrays) -> planar linear BT.709 RGB, float64 (3, H, W)."""
    ow, oh = cs.out_dims()
    out = np.empty((3, oh, ow), dtype=np.float64)
    bufs = [np.ascontiguousarray(np.frombuffer(memoryview(p), dtype=np.uint8)) for p in planes]
    ptrs = (ctypes.c_void_p * 3)(*[b.ctypes.data for b in bufs])
    ls = (ctypes.c_int64 * 3)(*line_sizes)
    rc = lib().oracle_convert(ptrs, ls, ctypes.byref(cs), _dp(out))
    if rc != 0:
        raise ValueError("unsupported chroma subsampling")
    return out


def ssimu2(rgb1, rgb2):
    """Returns (score as the reference computes it, score in pure FP64, 108 features)."""
    rgb1 = np.ascontiguousarray(rgb1, dtype=np.float64)
    rgb2 = np.ascontiguousarray(rgb2, dtype=np.float64)
    _, h, w = rgb1.shape
    feats = np.zeros(108, dtype=np.float64)
    q = ctypes.c_double()
    d = ctypes.c_double()
    lib().oracle_ssimu2(_dp(rgb1), _dp(rgb2), w, h, _dp(feats), ctypes.byref(q), ctypes.byref(d))
    return q.value, d.value, feats


def ssimu2_final(features, quirk=True):
    f = np.ascontiguousarray(features, dtype=np.float64)
    return lib().oracle_ssimu2_final(_dp(f), 1 if quirk else 0)


def butteraugli(rgb1, rgb2, intensity=203.0, qnorm=2):
    """Returns ((normQ, norm3, norminf), distortion map float64 (H, W))."""
    rgb1 = np.ascontiguousarray(rgb1, dtype=np.float64)
    rgb2 = np.ascontiguousarray(rgb2, dtype=np.float64)
    _, h, w = rgb1.shape
    dmap = np.empty((h, w), dtype=np.float64)
    norms = np.zeros(3, dtype=np.float64)
    lib().oracle_butteraugli(_dp(rgb1), _dp(rgb2), w, h, float(intensity), int(qnorm), _dp(dmap), _dp(norms))
    return tuple(norms), dmap


def blur(plane, sigma, radius):
    plane = np.ascontiguousarray(plane, dtype=np.float64)
    out = np.empty_like(plane)
    h, w = plane.shape
    lib().oracle_blur(_dp(plane), _dp(out), w, h, float(sigma), int(radius))
    return out


def downsample(plane):
    plane = np.ascontiguousarray(plane, dtype=np.float64)
    h, w = plane.shape
    out = np.empty(((h - 1) // 2 + 1, (w - 1) // 2 + 1), dtype=np.float64)
    lib().oracle_downsample(_dp(plane), w, h, _dp(out))
    return out


def positive_xyb(rgb):
    """Planar linear RGB (3, H, W) -> positive XYB (3, H, W), float64 (makeXYB.hpp:6-47)."""
    out = np.array(rgb, dtype=np.float64, order="C", copy=True)
    lib().oracle_positive_xyb(_dp(out), out.shape[1] * out.shape[2])
    return out


def pyramid_level(rgb, level):
    """Linear RGB (3, H, W) -> positive XYB of pyramid level `level` (2x box downsamples of the
    linear RGB, src/ssimu2/downsample.hpp:3-19, then XYB)."""
    planes = [np.asarray(rgb[c], dtype=np.float64) for c in range(3)]
    for _ in range(level):
        planes = [downsample(p) for p in planes]
    return positive_xyb(np.stack(planes))


def num_threads():
    return lib().oracle_num_threads()
