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
    srcs = [os.path.join(HERE, "oracle.c"), os.path.join(HERE, "cvvdp.c"), os.path.join(HERE, "ssimu2_f32.c")]
    csrc = os.path.join(os.path.dirname(HERE), "vship_b200", "csrc")
    deps = srcs + [os.path.join(csrc, "metric_tables.h"), os.path.join(csrc, "cvvdp_csf_table.h")]
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(d) for d in deps)):
        return LIB_PATH
    tmp = LIB_PATH + ".tmp"
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-shared", "-fPIC", "-std=c11",
                           "-fvisibility=hidden", "-o", tmp] + srcs + ["-lm"])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


CUDA_MATH_PATH = os.path.join(HERE, "libcudamath.so")
_cuda_math = None


def build_cuda_math(force=False):
    """Compile cuda_math.cu (CUDA's own powf/cbrtf/expf over arrays) with nvcc's default math
    flags, as the reference library is built.  Test infrastructure only."""
    src = os.path.join(HERE, "cuda_math.cu")
    if not force and os.path.exists(CUDA_MATH_PATH) and os.path.getmtime(CUDA_MATH_PATH) >= os.path.getmtime(src):
        return CUDA_MATH_PATH
    tmp = CUDA_MATH_PATH + ".tmp"
    subprocess.check_call(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                           "-Xcompiler", "-fPIC", "-o", tmp, src])
    os.replace(tmp, CUDA_MATH_PATH)
    return CUDA_MATH_PATH


_MATH_FN = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_float,
                            ctypes.POINTER(ctypes.c_float), ctypes.c_int64)


def use_cuda_math(enable=True):
    """Make the FP32 restatement take powf/cbrtf/expf from CUDA on the current GPU (True) or
    from the correctly rounded CPU evaluation (False)."""
    global _cuda_math
    L = lib()
    if not enable:
        L.oracle_f32_set_math(ctypes.cast(None, _MATH_FN))
        _cuda_math = None
        return
    cm = ctypes.CDLL(build_cuda_math())
    cm.cm_eval.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_float,
                           ctypes.POINTER(ctypes.c_float), ctypes.c_int64]
    cm.cm_eval.restype = ctypes.c_int

    def _eval(op, x, y, out, n):
        rc = cm.cm_eval(op, x, y, out, n)
        if rc != 0:
            raise RuntimeError("cm_eval failed with CUDA error %d" % rc)

    _cuda_math = (cm, _MATH_FN(_eval))   # keep the callback alive
    L.oracle_f32_set_math(_cuda_math[1])


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
        fp = ctypes.POINTER(ctypes.c_float)
        L.oracle_f32_convert.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(abi.Colorspace), fp]
        L.oracle_f32_convert.restype = ctypes.c_int
        L.oracle_f32_ssimu2.argtypes = [fp, fp, ctypes.c_int64, ctypes.c_int64, fp]
        L.oracle_f32_ssimu2.restype = ctypes.c_double
        L.oracle_f32_set_math.argtypes = [_MATH_FN]
        L.oracle_convert_native.argtypes = L.oracle_convert.argtypes
        L.oracle_convert_native.restype = ctypes.c_int
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        L.oracle_cvvdp_new.restype = vp
        L.oracle_cvvdp_new.argtypes = [i64, i64, ctypes.c_double, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int]
        L.oracle_cvvdp_free.argtypes = [vp]
        L.oracle_cvvdp_info.argtypes = [vp, ctypes.POINTER(i64)]
        L.oracle_cvvdp_filters.argtypes = [vp, dp]
        L.oracle_cvvdp_reset.argtypes = [vp, ctypes.c_int]
        L.oracle_cvvdp_frame.argtypes = [vp, dp, dp, ctypes.c_int, dp, dp]
        L.oracle_cvvdp_bands.argtypes = [vp, dp]
        L.oracle_cvvdp_bands.restype = ctypes.c_double
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


def convert_native(planes, line_sizes, cs):
    """Like convert() but in the clip's own primaries (CVVDP's input, src/cvvdp/main.hpp:188)."""
    ow, oh = cs.out_dims()
    out = np.empty((3, oh, ow), dtype=np.float64)
    bufs = [np.ascontiguousarray(np.frombuffer(memoryview(p), dtype=np.uint8)) for p in planes]
    ptrs = (ctypes.c_void_p * 3)(*[b.ctypes.data for b in bufs])
    ls = (ctypes.c_int64 * 3)(*line_sizes)
    rc = lib().oracle_convert_native(ptrs, ls, ctypes.byref(cs), _dp(out))
    if rc != 0:
        raise ValueError("unsupported chroma subsampling")
    return out


# Built-in CVVDP displays (src/cvvdp/display_models.hpp:40-106) as oracle_cvvdp_new's model
# vector: res_x, res_y, hdr, viewing distance (m), diagonal (in), peak luminance, contrast,
# ambient illuminance (lux), k_refl, exposure.
CVVDP_DISPLAYS = {
    "standard_4k": (3840, 2160, 0, 0.7472, 30, 200, 1000, 250, 0.005, 1),
    "standard_hdr_pq": (3840, 2160, 1, 0.7472, 30, 1500, 1000000, 10, 0.005, 1),
    "standard_hdr_hlg": (3840, 2160, 1, 0.7472, 30, 1500, 1000000, 10, 0.005, 1),
    "standard_hdr_linear": (3840, 2160, 1, 0.7472, 30, 1500, 1000000, 10, 0.005, 1),
    "standard_hdr_dark": (3840, 2160, 1, 0.7472, 30, 1500, 1000000, 0, 0.005, 1),
    "standard_hdr_linear_zoom": (3840, 2160, 1, 0.25, 30, 10000, 1000000, 10, 0.005, 1),
    "standard_fhd": (1920, 1080, 0, 0.6, 24, 200, 1000, 250, 0.005, 1),
}


class CVVDP:
    """FP64 CVVDP of one clip pair with the reference's temporal state (cvvdp.c)."""

    def __init__(self, width, height, fps, display="standard_fhd", resize_to_display=False,
                 trc=(abi.TRC_BT709, abi.TRC_BT709), primaries=(abi.PRIMARIES_BT709, abi.PRIMARIES_BT709)):
        model = display if not isinstance(display, str) else CVVDP_DISPLAYS[display]
        m = np.ascontiguousarray(model, dtype=np.float64)
        self.h = lib().oracle_cvvdp_new(width, height, float(fps), 1 if resize_to_display else 0, _dp(m),
                                        trc[0], primaries[0], trc[1], primaries[1])
        if not self.h:
            raise ValueError("frame too small for CVVDP")
        info = (ctypes.c_int64 * 6)()
        lib().oracle_cvvdp_info(self.h, info)
        self.resize = (info[0], info[1])
        self.levels, self.taps = info[2], info[3]

    def frame(self, lin1, lin2, compute=True, distmap=False):
        """lin1/lin2: (3, H, W) linear RGB in the clip primaries.  Returns the JOD score (and the
        distortion map when asked) after adding the frame; None when compute is False."""
        a = np.ascontiguousarray(lin1, dtype=np.float64)
        b = np.ascontiguousarray(lin2, dtype=np.float64)
        score = ctypes.c_double(0.0)
        dmap = np.zeros((self.resize[1], self.resize[0]), dtype=np.float64) if distmap else None
        lib().oracle_cvvdp_frame(self.h, _dp(a), _dp(b), 1 if compute else 0, ctypes.byref(score),
                                 _dp(dmap) if distmap else None)
        if not compute:
            return None
        return (score.value, dmap) if distmap else score.value

    def bands(self):
        vals = np.zeros(4 * self.levels, dtype=np.float64)
        q = lib().oracle_cvvdp_bands(self.h, _dp(vals))
        return vals.reshape(self.levels, 4), q

    def filters(self):
        out = np.zeros(4 * self.taps, dtype=np.float64)
        lib().oracle_cvvdp_filters(self.h, _dp(out))
        return out.reshape(4, self.taps)

    def reset(self, only_score=False):
        lib().oracle_cvvdp_reset(self.h, 1 if only_score else 0)

    def close(self):
        if self.h:
            lib().oracle_cvvdp_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


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


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def convert_f32(planes, line_sizes, cs):
    """Raw planes -> planar linear BT.709 RGB in the reference's own float arithmetic
    (ssimu2_f32.c), float32 (3, H, W)."""
    ow, oh = cs.out_dims()
    out = np.empty((3, oh, ow), dtype=np.float32)
    bufs = [np.ascontiguousarray(np.frombuffer(memoryview(p), dtype=np.uint8)) for p in planes]
    ptrs = (ctypes.c_void_p * 3)(*[b.ctypes.data for b in bufs])
    ls = (ctypes.c_int64 * 3)(*line_sizes)
    if lib().oracle_f32_convert(ptrs, ls, ctypes.byref(cs), _fp(out)) != 0:
        raise ValueError("unsupported chroma subsampling")
    return out


def ssimu2_f32(rgb1, rgb2):
    """SSIMULACRA2 of two float32 (3, H, W) linear RGB images with the reference's float
    arithmetic (ssimu2_f32.c).  Returns (score, 108 float features)."""
    rgb1 = np.ascontiguousarray(rgb1, dtype=np.float32)
    rgb2 = np.ascontiguousarray(rgb2, dtype=np.float32)
    _, h, w = rgb1.shape
    feats = np.zeros(108, dtype=np.float32)
    score = lib().oracle_f32_ssimu2(_fp(rgb1), _fp(rgb2), w, h, _fp(feats))
    return score, feats


def ssimu2_reference_arith(p1, ls1, cs1, p2, ls2, cs2):
    """Score of a raw frame pair as the reference library's float pipeline forms it."""
    return ssimu2_f32(convert_f32(p1, ls1, cs1), convert_f32(p2, ls2, cs2))[0]


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
