"""Python binding of libvship.so (the B200 engine behind Vship's C ABI).

Loads the in-tree library with ctypes and mirrors the reference's API surface
(src/VshipAPI.h): handler objects for SSIMULACRA2 and Butteraugli with the same argument
meaning and the same error codes, raised here as VshipError carrying the library's detailed
message.  It refuses to run without the compiled library: there is no Python or CPU fallback.
"""
import ctypes
import os
import threading

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvship.so")

_lib = None
_lock = threading.Lock()


class VshipError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code
        self.name = abi.EXCEPTIONS.get(code, "BadErrorType")


def _declare(L):
    c = ctypes
    H2, HB = abi.SSIMU2Handler, abi.ButteraugliHandler
    u8pp = c.POINTER(c.POINTER(c.c_uint8))
    i64p = c.POINTER(c.c_int64)
    L.Vship_GetVersion.restype = abi.Version
    L.Vship_GetVersion.argtypes = []
    L.Vship_GetDeviceCount.argtypes = [c.POINTER(c.c_int)]
    L.Vship_SetDevice.argtypes = [c.c_int]
    L.Vship_GetDeviceInfo.argtypes = [c.POINTER(abi.DeviceInfo), c.c_int]
    L.Vship_GPUFullCheck.argtypes = [c.c_int]
    L.Vship_GetErrorMessage.argtypes = [c.c_int, c.c_char_p, c.c_int]
    L.Vship_GetErrorMessage.restype = c.c_int
    L.Vship_GetDetailedLastError.argtypes = [c.c_char_p, c.c_int]
    L.Vship_GetDetailedLastError.restype = c.c_int
    L.Vship_PinnedMalloc.argtypes = [c.POINTER(c.c_void_p), c.c_uint64]
    L.Vship_PinnedFree.argtypes = [c.c_void_p]
    L.Vship_SSIMU2Init.argtypes = [c.POINTER(H2), abi.Colorspace, abi.Colorspace]
    L.Vship_SSIMU2Init2.argtypes = [c.POINTER(H2), abi.Colorspace, abi.Colorspace, c.c_int]
    L.Vship_SSIMU2Free.argtypes = [H2]
    L.Vship_ComputeSSIMU2.argtypes = [H2, c.POINTER(c.c_double), u8pp, u8pp, i64p, i64p]
    L.Vship_SSIMU2GetDetailedLastError.argtypes = [H2, c.c_char_p, c.c_int]
    L.Vship_SSIMU2GetDetailedLastError.restype = c.c_int
    L.Vship_ButteraugliInit.argtypes = [c.POINTER(HB), abi.Colorspace, abi.Colorspace, c.c_int, c.c_float]
    L.Vship_ButteraugliInit2.argtypes = [c.POINTER(HB), abi.Colorspace, abi.Colorspace, c.c_int, c.c_float, c.c_int]
    L.Vship_ButteraugliFree.argtypes = [HB]
    L.Vship_ComputeButteraugli.argtypes = [HB, c.POINTER(abi.ButteraugliScore), c.c_void_p, c.c_int64, u8pp, u8pp, i64p, i64p]
    L.Vship_ButteraugliGetDetailedLastError.argtypes = [HB, c.c_char_p, c.c_int]
    L.Vship_ButteraugliGetDetailedLastError.restype = c.c_int
    HC = abi.CVVDPHandler
    L.Vship_CVVDPInit.argtypes = [c.POINTER(HC), abi.Colorspace, abi.Colorspace, c.c_float, c.c_bool, c.c_char_p]
    L.Vship_CVVDPInit2.argtypes = [c.POINTER(HC), abi.Colorspace, abi.Colorspace, c.c_float, c.c_bool, c.c_char_p,
                                   c.c_char_p]
    L.Vship_CVVDPInit3.argtypes = [c.POINTER(HC), abi.Colorspace, abi.Colorspace, c.c_float, c.c_bool, c.c_char_p,
                                   c.c_char_p, c.c_int]
    L.Vship_CVVDPFree.argtypes = [HC]
    L.Vship_CVVDPGetDistmapResolution.argtypes = [HC, i64p, i64p]
    L.Vship_ResetCVVDP.argtypes = [HC]
    L.Vship_ResetScoreCVVDP.argtypes = [HC]
    L.Vship_LoadTemporalCVVDP.argtypes = [HC, u8pp, u8pp, i64p, i64p]
    L.Vship_ComputeCVVDP.argtypes = [HC, c.POINTER(c.c_double), c.c_void_p, c.c_int64, u8pp, u8pp, i64p, i64p]
    L.Vship_CVVDPGetDetailedLastError.argtypes = [HC, c.c_char_p, c.c_int]
    L.Vship_CVVDPGetDetailedLastError.restype = c.c_int
    # extensions (absent from the reference library)
    if not hasattr(L, "VshipExt_ComputeSSIMU2Device"):
        return L
    vpp = c.POINTER(c.c_void_p)
    L.VshipExt_ComputeSSIMU2Device.argtypes = [H2, c.c_int, c.c_void_p, c.c_void_p, vpp, vpp, i64p, i64p, c.c_void_p]
    L.VshipExt_SSIMU2LastFeatures.argtypes = [H2, c.POINTER(c.c_float)]
    L.VshipExt_ComputeButteraugliDevice.argtypes = [HB, c.c_void_p, c.c_void_p, c.c_int64, vpp, vpp, i64p, i64p, c.c_void_p]
    L.VshipExt_SSIMU2KernelTiming.argtypes = [H2, c.c_int]
    L.VshipExt_SSIMU2KernelTimes.argtypes = [H2, c.c_void_p, c.c_int, c.c_int]
    L.VshipExt_SSIMU2KernelTimes.restype = c.c_int
    L.VshipExt_ButteraugliKernelTiming.argtypes = [HB, c.c_int]
    L.VshipExt_ButteraugliKernelTimes.argtypes = [HB, c.c_void_p, c.c_int, c.c_int]
    L.VshipExt_ButteraugliKernelTimes.restype = c.c_int
    L.VshipExt_SSIMU2Resolution.argtypes = [H2, i64p, i64p]
    L.VshipExt_ComputeSSIMU2NoAlloc.argtypes = [abi.Colorspace, abi.Colorspace, c.c_void_p, c.c_void_p, vpp, vpp,
                                                i64p, i64p, c.c_void_p]
    L.VshipExt_ButteraugliResolution.argtypes = [HB, i64p, i64p]
    L.VshipExt_ButteraugliTestTmaTimeout.argtypes = [HB]
    HBt = abi.SSIMU2BatchHandler
    FPp = c.POINTER(abi.FramePair)
    L.VshipExt_SSIMU2BatchInit.argtypes = [c.POINTER(HBt), c.c_int]
    L.VshipExt_SSIMU2BatchFree.argtypes = [HBt]
    L.VshipExt_SSIMU2BatchGetDetailedLastError.argtypes = [HBt, c.c_char_p, c.c_int]
    L.VshipExt_SSIMU2BatchGetDetailedLastError.restype = c.c_int
    L.VshipExt_ComputeSSIMU2BatchDevice.argtypes = [HBt, c.c_int, FPp, c.c_void_p, c.c_void_p, c.c_void_p]
    L.VshipExt_ComputeSSIMU2Batch.argtypes = [HBt, c.c_int, FPp, c.POINTER(c.c_double), c.c_void_p]
    L.VshipExt_SSIMU2BatchSetTileRows.argtypes = [HBt, c.c_int]
    L.VshipExt_SSIMU2BatchTileRows.argtypes = [HBt, c.POINTER(c.c_int)]
    L.VshipExt_SSIMU2BatchTestHoldFrontTile.argtypes = [HBt]
    L.VshipExt_SSIMU2BatchKernelTiming.argtypes = [HBt, c.c_int]
    L.VshipExt_SSIMU2BatchKernelTimes.argtypes = [HBt, c.c_void_p, c.c_int, c.c_int]
    L.VshipExt_SSIMU2BatchKernelTimes.restype = c.c_int
    HS = abi.SurrogateHandler
    L.VshipExt_SurrogateInit.argtypes = [c.POINTER(HS), abi.Colorspace, abi.Colorspace, c.c_int]
    L.VshipExt_SurrogateFree.argtypes = [HS]
    L.VshipExt_SurrogateGetDetailedLastError.argtypes = [HS, c.c_char_p, c.c_int]
    L.VshipExt_SurrogateGetDetailedLastError.restype = c.c_int
    L.VshipExt_SurrogateInputSize.argtypes = [HS, i64p]
    L.VshipExt_SurrogateInputs.argtypes = [HS, c.c_int, vpp, vpp, i64p, i64p, c.c_void_p, c.c_void_p]
    L.VshipExt_SurrogatePredictInputs.argtypes = [HS, c.c_int, c.c_void_p, c.c_void_p, c.c_void_p]
    L.VshipExt_SurrogatePredict.argtypes = [HS, c.c_int, vpp, vpp, i64p, i64p, c.c_void_p, c.c_void_p]
    L.VshipExt_SurrogateReferenceSize.argtypes = [HS, i64p]
    L.VshipExt_SurrogateReferences.argtypes = [HS, c.c_int, vpp, i64p, c.c_void_p, c.c_void_p]
    L.VshipExt_SurrogatePredictAgainst.argtypes = [HS, c.c_int, c.c_void_p, vpp, i64p, c.c_void_p, c.c_void_p]
    L.VshipExt_SurrogateTrain.argtypes = [HS, c.c_int, c.c_void_p, c.c_void_p, c.c_int, c.c_int, c.c_float, c.c_uint,
                                          c.c_void_p]
    L.VshipExt_SurrogateGradients.argtypes = [HS, c.c_int, c.c_void_p, c.c_void_p, c.c_void_p,
                                              c.POINTER(c.c_double)]
    L.VshipExt_SurrogateModel.argtypes = [HS, c.c_void_p, c.c_int]
    L.VshipExt_SurrogateModel.restype = c.c_int
    L.VshipExt_SurrogateSetModel.argtypes = [HS, c.c_void_p, c.c_int]
    L.VshipExt_SurrogateKernelTiming.argtypes = [HS, c.c_int]
    L.VshipExt_SurrogateKernelTimes.argtypes = [HS, c.c_void_p, c.c_int, c.c_int]
    L.VshipExt_SurrogateKernelTimes.restype = c.c_int
    L.VshipExt_CVVDPDisplayModel.argtypes = [c.c_char_p, c.c_char_p, c.POINTER(abi.CVVDPDisplay)]
    L.VshipExt_CVVDPGeometry.argtypes = [HC, c.POINTER(c.c_int), c.POINTER(c.c_int)]
    L.VshipExt_CVVDPKernelTiming.argtypes = [HC, c.c_int]
    L.VshipExt_CVVDPKernelTimes.argtypes = [HC, c.c_void_p, c.c_int, c.c_int]
    L.VshipExt_CVVDPKernelTimes.restype = c.c_int
    return L


class KernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_int), ("total_ms", ctypes.c_double)]


def load(path=None):
    """Loads (once) and returns the ctypes handle of libvship.so; raises if it is missing."""
    global _lib
    with _lock:
        if _lib is None or path is not None:
            p = path or LIB_PATH
            if not os.path.exists(p):
                raise RuntimeError("libvship.so is not built (run `python -m vship_b200.build`): %s" % p)
            _lib = _declare(ctypes.CDLL(p))
        return _lib


def load_library(path):
    """A separate handle on any library exporting the Vship ABI (e.g. the reference build)."""
    return _declare(ctypes.CDLL(path))


def _message(L, fn=None, handler=None):
    if fn is None:
        n = L.Vship_GetDetailedLastError(None, 0)
        buf = ctypes.create_string_buffer(n)
        L.Vship_GetDetailedLastError(buf, n)
    else:
        n = fn(handler, None, 0)
        if n <= 0:
            return _message(L)
        buf = ctypes.create_string_buffer(n)
        fn(handler, buf, n)
    return buf.value.decode(errors="replace")


def check(L, rc, fn=None, handler=None):
    if rc != 0:
        raise VshipError(rc, _message(L, fn, handler))


def planes_arg(planes):
    """Three buffers (bytes / numpy / ctypes addresses) -> uint8_t*[3] and keep-alive list."""
    keep = []
    arr = abi.PlanePtrs()
    for i, p in enumerate(planes):
        if isinstance(p, int):
            arr[i] = ctypes.cast(ctypes.c_void_p(p), ctypes.POINTER(ctypes.c_uint8))
            continue
        if hasattr(p, "ctypes"):
            addr = p.ctypes.data
            keep.append(p)
        else:
            buf = (ctypes.c_uint8 * len(p)).from_buffer_copy(p)
            keep.append(buf)
            addr = ctypes.addressof(buf)
        arr[i] = ctypes.cast(ctypes.c_void_p(addr), ctypes.POINTER(ctypes.c_uint8))
    return arr, keep


def version(lib=None):
    v = (lib or load()).Vship_GetVersion()
    return (v.major, v.minor, v.minorMinor, v.backend)


def device_count(lib=None):
    L = lib or load()
    n = ctypes.c_int(0)
    check(L, L.Vship_GetDeviceCount(ctypes.byref(n)))
    return n.value


def error_message(code, lib=None):
    L = lib or load()
    n = L.Vship_GetErrorMessage(code, None, 0)
    buf = ctypes.create_string_buffer(n)
    L.Vship_GetErrorMessage(code, buf, n)
    return buf.value.decode()


class SSIMU2:
    """An SSIMULACRA2 handler (Vship_SSIMU2Init2 .. Vship_SSIMU2Free)."""

    def __init__(self, src_cs, dis_cs=None, gpu_id=0, lib=None):
        self.L = lib or load()
        self.h = abi.SSIMU2Handler()
        self.src_cs, self.dis_cs = src_cs, dis_cs or src_cs
        rc = self.L.Vship_SSIMU2Init2(ctypes.byref(self.h), self.src_cs, self.dis_cs, gpu_id)
        self.alive = True
        if rc != 0:
            msg = _message(self.L, self.L.Vship_SSIMU2GetDetailedLastError, self.h)
            self.close()
            raise VshipError(rc, msg)

    def compute(self, planes1, planes2, line_sizes1, line_sizes2=None):
        a1, k1 = planes_arg(planes1)
        a2, k2 = planes_arg(planes2)
        ls1 = abi.LineSizes(*line_sizes1)
        ls2 = abi.LineSizes(*(line_sizes2 or line_sizes1))
        score = ctypes.c_double()
        rc = self.L.Vship_ComputeSSIMU2(self.h, ctypes.byref(score), a1, a2, ls1, ls2)
        check(self.L, rc, self.L.Vship_SSIMU2GetDetailedLastError, self.h)
        return score.value

    def last_features(self):
        import numpy as np
        out = (ctypes.c_float * 108)()
        check(self.L, self.L.VshipExt_SSIMU2LastFeatures(self.h, out))
        return np.frombuffer(out, dtype=np.float32).copy()

    def compute_device(self, n, ptrs1, ptrs2, line_sizes1, line_sizes2, d_scores, d_features=0, stream=0):
        """ptrs1/ptrs2: 3*n device plane addresses; d_scores/d_features: device addresses."""
        a1 = (ctypes.c_void_p * (3 * n))(*ptrs1)
        a2 = (ctypes.c_void_p * (3 * n))(*ptrs2)
        rc = self.L.VshipExt_ComputeSSIMU2Device(self.h, n, d_scores, d_features or None, a1, a2,
                                                 abi.LineSizes(*line_sizes1), abi.LineSizes(*line_sizes2), stream or None)
        check(self.L, rc, self.L.Vship_SSIMU2GetDetailedLastError, self.h)

    def kernel_timing(self, enable=True):
        check(self.L, self.L.VshipExt_SSIMU2KernelTiming(self.h, 1 if enable else 0))

    def kernel_times(self, reset=False):
        out = (KernelTime * 8)()
        n = self.L.VshipExt_SSIMU2KernelTimes(self.h, out, 8, 1 if reset else 0)
        if n < 0:
            check(self.L, abi.BadHandler)
        return {out[i].name.decode(): (out[i].launches, out[i].total_ms) for i in range(n)}

    def close(self):
        if getattr(self, "alive", False):
            self.alive = False
            self.L.Vship_SSIMU2Free(self.h)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Butteraugli:
    """A Butteraugli handler (Vship_ButteraugliInit2 .. Vship_ButteraugliFree)."""

    def __init__(self, src_cs, dis_cs=None, qnorm=2, intensity=203.0, gpu_id=0, lib=None):
        self.L = lib or load()
        self.h = abi.ButteraugliHandler()
        self.src_cs, self.dis_cs = src_cs, dis_cs or src_cs
        rc = self.L.Vship_ButteraugliInit2(ctypes.byref(self.h), self.src_cs, self.dis_cs, int(qnorm), float(intensity), gpu_id)
        self.alive = True
        if rc != 0:
            msg = _message(self.L, self.L.Vship_ButteraugliGetDetailedLastError, self.h)
            self.close()
            raise VshipError(rc, msg)

    def compute(self, planes1, planes2, line_sizes1, line_sizes2=None, distmap=False):
        """Returns ((normQ, norm3, norminf), distmap float32 (H, W) or None)."""
        import numpy as np
        a1, k1 = planes_arg(planes1)
        a2, k2 = planes_arg(planes2)
        ls1 = abi.LineSizes(*line_sizes1)
        ls2 = abi.LineSizes(*(line_sizes2 or line_sizes1))
        score = abi.ButteraugliScore()
        dm = None
        dst, stride = None, 0
        if distmap:
            w, h = self.src_cs.out_dims()
            dm = np.zeros((h, w), dtype=np.float32)
            dst, stride = dm.ctypes.data, w * 4
        rc = self.L.Vship_ComputeButteraugli(self.h, ctypes.byref(score), dst, stride, a1, a2, ls1, ls2)
        check(self.L, rc, self.L.Vship_ButteraugliGetDetailedLastError, self.h)
        return (score.normQ, score.norm3, score.norminf), dm

    def compute_device(self, ptrs1, ptrs2, line_sizes1, line_sizes2, d_norms, d_distmap=0, dststride=0, stream=0):
        a1 = (ctypes.c_void_p * 3)(*ptrs1)
        a2 = (ctypes.c_void_p * 3)(*ptrs2)
        rc = self.L.VshipExt_ComputeButteraugliDevice(self.h, d_norms, d_distmap or None, dststride, a1, a2,
                                                      abi.LineSizes(*line_sizes1), abi.LineSizes(*line_sizes2), stream or None)
        check(self.L, rc, self.L.Vship_ButteraugliGetDetailedLastError, self.h)

    def kernel_timing(self, enable=True):
        check(self.L, self.L.VshipExt_ButteraugliKernelTiming(self.h, 1 if enable else 0))

    def test_tma_timeout(self):
        """Arms the next call's test of the column pass's bounded tensor-map waits."""
        check(self.L, self.L.VshipExt_ButteraugliTestTmaTimeout(self.h), self.L.Vship_ButteraugliGetDetailedLastError, self.h)

    def kernel_times(self, reset=False):
        out = (KernelTime * 8)()
        n = self.L.VshipExt_ButteraugliKernelTimes(self.h, out, 8, 1 if reset else 0)
        if n < 0:
            check(self.L, abi.BadHandler)
        return {out[i].name.decode(): (out[i].launches, out[i].total_ms) for i in range(n)}

    def close(self):
        if getattr(self, "alive", False):
            self.alive = False
            self.L.Vship_ButteraugliFree(self.h)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CVVDP:
    """A CVVDP handler (Vship_CVVDPInit3 .. Vship_CVVDPFree): frames are fed in order; each
    compute() returns the JOD of the sequence so far."""

    def __init__(self, src_cs, dis_cs=None, fps=24.0, resize_to_display=False, model="standard_fhd",
                 model_config_json=None, gpu_id=0, lib=None):
        self.L = lib or load()
        self.h = abi.CVVDPHandler()
        self.src_cs, self.dis_cs = src_cs, dis_cs or src_cs
        js = model_config_json.encode() if model_config_json else None
        rc = self.L.Vship_CVVDPInit3(ctypes.byref(self.h), self.src_cs, self.dis_cs, float(fps), bool(resize_to_display),
                                     model.encode(), js, gpu_id)
        self.alive = True
        if rc != 0:
            msg = _message(self.L, self.L.Vship_CVVDPGetDetailedLastError, self.h)
            self.close()
            raise VshipError(rc, msg)

    def _check(self, rc):
        check(self.L, rc, self.L.Vship_CVVDPGetDetailedLastError, self.h)

    def distmap_resolution(self):
        w, h = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.L.Vship_CVVDPGetDistmapResolution(self.h, ctypes.byref(w), ctypes.byref(h)))
        return w.value, h.value

    def geometry(self):
        """(pyramid bands, ring frames) -- extension."""
        b, r = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.VshipExt_CVVDPGeometry(self.h, ctypes.byref(b), ctypes.byref(r)))
        return b.value, r.value

    def compute(self, planes1, planes2, line_sizes1, line_sizes2=None, distmap=False):
        """Returns the JOD score, or (score, distortion map float32 (H, W)) with distmap."""
        import numpy as np
        a1, k1 = planes_arg(planes1)
        a2, k2 = planes_arg(planes2)
        ls1 = abi.LineSizes(*line_sizes1)
        ls2 = abi.LineSizes(*(line_sizes2 or line_sizes1))
        score = ctypes.c_double()
        dm, dst, stride = None, None, 0
        if distmap:
            w, h = self.distmap_resolution()
            dm = np.zeros((h, w), dtype=np.float32)
            dst, stride = dm.ctypes.data, w * 4
        self._check(self.L.Vship_ComputeCVVDP(self.h, ctypes.byref(score), dst, stride, a1, a2, ls1, ls2))
        return (score.value, dm) if distmap else score.value

    def load_temporal(self, planes1, planes2, line_sizes1, line_sizes2=None):
        a1, k1 = planes_arg(planes1)
        a2, k2 = planes_arg(planes2)
        ls1 = abi.LineSizes(*line_sizes1)
        ls2 = abi.LineSizes(*(line_sizes2 or line_sizes1))
        self._check(self.L.Vship_LoadTemporalCVVDP(self.h, a1, a2, ls1, ls2))

    def reset(self):
        self._check(self.L.Vship_ResetCVVDP(self.h))

    def reset_score(self):
        self._check(self.L.Vship_ResetScoreCVVDP(self.h))

    def kernel_timing(self, enable=True):
        self._check(self.L.VshipExt_CVVDPKernelTiming(self.h, 1 if enable else 0))

    def kernel_times(self, reset=False):
        out = (KernelTime * 8)()
        n = self.L.VshipExt_CVVDPKernelTimes(self.h, out, 8, 1 if reset else 0)
        if n < 0:
            check(self.L, abi.BadHandler)
        return {out[i].name.decode(): (out[i].launches, out[i].total_ms) for i in range(n)}

    def close(self):
        if getattr(self, "alive", False):
            self.alive = False
            self.L.Vship_CVVDPFree(self.h)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cvvdp_display(model="standard_fhd", model_config_json=None, lib=None):
    """The display a CVVDP handler would use (VshipExt_CVVDPDisplayModel), as a dict; host only."""
    L = lib or load()
    out = abi.CVVDPDisplay()
    js = model_config_json.encode() if model_config_json else None
    rc = L.VshipExt_CVVDPDisplayModel(model.encode(), js, ctypes.byref(out))
    check(L, rc)
    return {f: getattr(out, f) for f, _ in abi.CVVDPDisplay._fields_}


def frame_pairs(items):
    """FramePair array from (src_cs, dis_cs, planes1, planes2, line_sizes1, line_sizes2) tuples.

    Planes are integer addresses (device or host) or numpy arrays (host); the returned
    keep-alive list holds the arrays for as long as the pairs are used."""
    arr = (abi.FramePair * len(items))()
    keep = []
    for i, (cs1, cs2, p1, p2, ls1, ls2) in enumerate(items):
        fp = arr[i]
        fp.src_colorspace, fp.dis_colorspace = cs1, cs2
        for dst, planes in ((fp.srcp1, p1), (fp.srcp2, p2)):
            for j, p in enumerate(planes):
                if isinstance(p, int):
                    dst[j] = p
                else:
                    keep.append(p)
                    dst[j] = p.ctypes.data
        for j in range(3):
            fp.lineSize[j], fp.lineSize2[j] = ls1[j], ls2[j]
    return arr, keep


class SSIMU2Batch:
    """Uneven SSIMULACRA2 batches (VshipExt_SSIMU2BatchInit .. VshipExt_SSIMU2BatchFree):
    pairs of any resolutions and formats scored in one persistent launch."""

    def __init__(self, gpu_id=0, lib=None):
        self.L = lib or load()
        self.h = abi.SSIMU2BatchHandler()
        rc = self.L.VshipExt_SSIMU2BatchInit(ctypes.byref(self.h), gpu_id)
        self.alive = True
        if rc != 0:
            msg = _message(self.L, self.L.VshipExt_SSIMU2BatchGetDetailedLastError, self.h)
            self.close()
            raise VshipError(rc, msg)

    def _check(self, rc):
        check(self.L, rc, self.L.VshipExt_SSIMU2BatchGetDetailedLastError, self.h)

    def compute(self, pairs, features=False):
        """Host-resident pairs (see frame_pairs); returns scores (and features (n, 108))."""
        import numpy as np
        arr, keep = frame_pairs(pairs)
        n = len(pairs)
        scores = np.zeros(n, dtype=np.float64)
        feats = np.zeros((n, 108), dtype=np.float32) if features else None
        self._check(self.L.VshipExt_ComputeSSIMU2Batch(
            self.h, n, arr, scores.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            feats.ctypes.data if features else None))
        return (scores, feats) if features else scores

    def compute_device(self, pairs, d_scores, d_features=0, stream=0):
        """Device-resident pairs (plane addresses are device pointers); asynchronous."""
        arr, keep = frame_pairs(pairs)
        self._check(self.L.VshipExt_ComputeSSIMU2BatchDevice(self.h, len(pairs), arr, d_scores,
                                                              d_features or None, stream or None))

    def compute_device_array(self, arr, n, d_scores, d_features=0, stream=0):
        """As compute_device, with a prepared FramePair array (no per-call conversion)."""
        self._check(self.L.VshipExt_ComputeSSIMU2BatchDevice(self.h, n, arr, d_scores, d_features or None,
                                                              stream or None))

    def set_tile_rows(self, rows):
        self._check(self.L.VshipExt_SSIMU2BatchSetTileRows(self.h, int(rows)))

    def tile_rows(self):
        r = ctypes.c_int(0)
        self._check(self.L.VshipExt_SSIMU2BatchTileRows(self.h, ctypes.byref(r)))
        return r.value

    def hold_front_tile(self):
        """Test hook: the next launch leaves its last front tile out, so that its bounded
        dependency wait runs out and the call reports Vship_HIPError."""
        self._check(self.L.VshipExt_SSIMU2BatchTestHoldFrontTile(self.h))

    def kernel_timing(self, enable=True):
        self._check(self.L.VshipExt_SSIMU2BatchKernelTiming(self.h, 1 if enable else 0))

    def kernel_times(self, reset=False):
        out = (KernelTime * 8)()
        n = self.L.VshipExt_SSIMU2BatchKernelTimes(self.h, out, 8, 1 if reset else 0)
        if n < 0:
            check(self.L, abi.BadHandler)
        return {out[i].name.decode(): (out[i].launches, out[i].total_ms) for i in range(n)}

    def close(self):
        if getattr(self, "alive", False):
            self.alive = False
            self.L.VshipExt_SSIMU2BatchFree(self.h)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Surrogate:
    """The learned SSIMULACRA2 surrogate of one colourspace pair (VshipExt_Surrogate*).

    Device arrays are passed as integer addresses (e.g. torch `data_ptr()`)."""

    def __init__(self, src_cs, dis_cs=None, gpu_id=0, lib=None):
        self.L = lib or load()
        self.h = abi.SurrogateHandler()
        rc = self.L.VshipExt_SurrogateInit(ctypes.byref(self.h), src_cs, dis_cs or src_cs, gpu_id)
        self.alive = True
        if rc != 0:
            msg = _message(self.L, self.L.VshipExt_SurrogateGetDetailedLastError, self.h)
            self.close()
            raise VshipError(rc, msg)

    def _check(self, rc):
        check(self.L, rc, self.L.VshipExt_SurrogateGetDetailedLastError, self.h)

    def input_elems(self):
        n = ctypes.c_int64(0)
        self._check(self.L.VshipExt_SurrogateInputSize(self.h, ctypes.byref(n)))
        return n.value

    def inputs(self, n, ptrs1, ptrs2, line_sizes1, line_sizes2, d_inputs, stream=0):
        a1 = (ctypes.c_void_p * (3 * n))(*ptrs1)
        a2 = (ctypes.c_void_p * (3 * n))(*ptrs2)
        self._check(self.L.VshipExt_SurrogateInputs(self.h, n, a1, a2, abi.LineSizes(*line_sizes1),
                                                    abi.LineSizes(*line_sizes2), d_inputs, stream or None))

    def predict(self, n, ptrs1, ptrs2, line_sizes1, line_sizes2, d_pred, stream=0):
        a1 = (ctypes.c_void_p * (3 * n))(*ptrs1)
        a2 = (ctypes.c_void_p * (3 * n))(*ptrs2)
        self._check(self.L.VshipExt_SurrogatePredict(self.h, n, a1, a2, abi.LineSizes(*line_sizes1),
                                                     abi.LineSizes(*line_sizes2), d_pred, stream or None))

    def reference_floats(self):
        n = ctypes.c_int64(0)
        self._check(self.L.VshipExt_SurrogateReferenceSize(self.h, ctypes.byref(n)))
        return n.value

    def references(self, n, ptrs1, line_sizes1, d_refs, stream=0):
        a1 = (ctypes.c_void_p * (3 * n))(*ptrs1)
        self._check(self.L.VshipExt_SurrogateReferences(self.h, n, a1, abi.LineSizes(*line_sizes1), d_refs,
                                                        stream or None))

    def predict_against(self, n, d_refs, ptrs2, line_sizes2, d_pred, stream=0):
        a2 = (ctypes.c_void_p * (3 * n))(*ptrs2)
        self._check(self.L.VshipExt_SurrogatePredictAgainst(self.h, n, d_refs, a2, abi.LineSizes(*line_sizes2),
                                                            d_pred, stream or None))

    def predict_inputs(self, n, d_inputs, d_pred, stream=0):
        self._check(self.L.VshipExt_SurrogatePredictInputs(self.h, n, d_inputs, d_pred, stream or None))

    def train(self, n, d_inputs, d_targets, epochs=8, batch=256, lr=3e-3, seed=1):
        import numpy as np
        hist = np.zeros(epochs, dtype=np.float32)
        self._check(self.L.VshipExt_SurrogateTrain(self.h, n, d_inputs, d_targets, epochs, batch, lr, seed,
                                                   hist.ctypes.data))
        return hist

    def kernel_timing(self, enable=True):
        self._check(self.L.VshipExt_SurrogateKernelTiming(self.h, 1 if enable else 0))

    def kernel_times(self, reset=False):
        out = (KernelTime * 8)()
        n = self.L.VshipExt_SurrogateKernelTimes(self.h, out, 8, 1 if reset else 0)
        if n < 0:
            check(self.L, abi.BadHandler)
        return {out[i].name.decode(): (out[i].launches, out[i].total_ms) for i in range(n)}

    def gradients(self, n, d_inputs, d_targets):
        import numpy as np
        g = np.zeros(self.num_params(), dtype=np.float32)
        loss = ctypes.c_double()
        self._check(self.L.VshipExt_SurrogateGradients(self.h, n, d_inputs, d_targets, g.ctypes.data,
                                                       ctypes.byref(loss)))
        return loss.value, g

    def model(self):
        import numpy as np
        n = self.L.VshipExt_SurrogateModel(self.h, None, 0)
        if n < 0:
            self._check(abi.BadHandler)
        out = np.zeros(n, dtype=np.float32)
        self.L.VshipExt_SurrogateModel(self.h, out.ctypes.data, n)
        return out

    def num_params(self):
        return self.L.VshipExt_SurrogateModel(self.h, None, 0) - 12

    def set_model(self, model):
        import numpy as np
        m = np.ascontiguousarray(model, dtype=np.float32)
        self._check(self.L.VshipExt_SurrogateSetModel(self.h, m.ctypes.data, len(m)))

    def close(self):
        if getattr(self, "alive", False):
            self.alive = False
            self.L.VshipExt_SurrogateFree(self.h)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PinnedBuffer:
    """Page-locked host memory from Vship_PinnedMalloc, exposed as a numpy uint8 array."""

    def __init__(self, nbytes, lib=None):
        import numpy as np
        self.L = lib or load()
        self.ptr = ctypes.c_void_p()
        check(self.L, self.L.Vship_PinnedMalloc(ctypes.byref(self.ptr), nbytes))
        self.nbytes = nbytes
        self.array = np.ctypeslib.as_array((ctypes.c_uint8 * nbytes).from_address(self.ptr.value))

    def free(self):
        if self.ptr:
            self.L.Vship_PinnedFree(self.ptr)
            self.ptr = ctypes.c_void_p()
