"""CPU tests of the C-ABI library: it loads, exports every function include/*.h declares
(and every Vship_* symbol of the reference build when that is present), and the calls that
need no GPU behave like the reference's (version, error texts and size convention, device
errors without a GPU, invalid handlers)."""
import ctypes
import os
import re
import subprocess

import pytest

from vship_b200 import abi, api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in ("VshipAPI.h", "VshipAPI_ext.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"EXPORTPREPROCESS\s+[\w\s\*]+?\b(\w+)\s*\(", text)
    return sorted(set(names))


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if " T " in l}


def test_exports_every_declared_symbol(vship_lib):
    names = declared_functions()
    assert len(names) >= 38
    syms = exported(api.LIB_PATH)
    missing = [n for n in names if n not in syms]
    assert not missing, missing
    for n in names:
        getattr(vship_lib, n)


def test_exports_cover_reference_build():
    ref = os.path.join(ROOT, "oracle", "_ref", "libvship_ref.so")
    if not os.path.exists(ref):
        pytest.skip("reference build not present")
    ref_syms = {s for s in exported(ref) if s.startswith("Vship_")}
    assert len(ref_syms) == 29
    assert ref_syms <= exported(api.LIB_PATH)


def test_version(vship_lib):
    assert api.version() == (4, 1, 0, 1)


def test_error_messages(vship_lib):
    L = vship_lib
    for code, name in abi.EXCEPTIONS.items():
        msg = api.error_message(code)
        expect = "InternalError" if name == "HIPError" else name
        assert msg.startswith(expect + ":"), (code, msg)
    n = L.Vship_GetErrorMessage(abi.BadHandler, None, 0)
    full = api.error_message(abi.BadHandler)
    assert n == len(full) + 1
    buf = ctypes.create_string_buffer(11)
    assert L.Vship_GetErrorMessage(abi.BadHandler, buf, 11) == n
    assert buf.value.decode() == full[:10]
    assert api.error_message(99).startswith("BadErrorType:")


def test_no_gpu_device_errors(vship_lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    L = vship_lib
    n = ctypes.c_int(-1)
    rc = L.Vship_GetDeviceCount(ctypes.byref(n))
    assert rc in (abi.DeviceCountError, abi.NoDeviceDetected)
    assert L.Vship_GPUFullCheck(0) == rc
    size = L.Vship_GetDetailedLastError(None, 0)
    buf = ctypes.create_string_buffer(size)
    L.Vship_GetDetailedLastError(buf, size)
    text = buf.value.decode()
    assert text.startswith("VshipException\n")
    assert " - At line " in text


def test_invalid_handlers(vship_lib):
    L = vship_lib
    h = abi.SSIMU2Handler(123456)
    score = ctypes.c_double()
    p = abi.PlanePtrs()
    ls = abi.LineSizes(1, 1, 1)
    assert L.Vship_ComputeSSIMU2(h, ctypes.byref(score), p, p, ls, ls) == abi.BadHandler
    assert L.Vship_SSIMU2Free(h) == abi.BadHandler
    assert L.Vship_SSIMU2GetDetailedLastError(h, None, 0) == 0
    hb = abi.ButteraugliHandler(77)
    sc = abi.ButteraugliScore()
    assert L.Vship_ComputeButteraugli(hb, ctypes.byref(sc), None, 0, p, p, ls, ls) == abi.BadHandler
    assert L.Vship_ButteraugliFree(hb) == abi.BadHandler
    size = L.Vship_GetDetailedLastError(None, 0)
    buf = ctypes.create_string_buffer(size)
    L.Vship_GetDetailedLastError(buf, size)
    assert "BadHandler" in buf.value.decode()


def test_cvvdp_host_errors(vship_lib):
    """CVVDP entry points that fail before touching a device: NULL arguments and unknown ids."""
    L = vship_lib
    h = abi.CVVDPHandler()
    cs = abi.srgb8(8, 8)
    L.Vship_CVVDPInit.argtypes = [ctypes.POINTER(abi.CVVDPHandler), abi.Colorspace, abi.Colorspace,
                                  ctypes.c_float, ctypes.c_bool, ctypes.c_char_p]
    assert L.Vship_CVVDPInit(ctypes.byref(h), cs, cs, 24.0, False, None) == abi.BadPointer
    assert L.Vship_CVVDPInit(None, cs, cs, 24.0, False, b"standard_fhd") == abi.BadPointer
    L.Vship_ResetCVVDP.argtypes = [abi.CVVDPHandler]
    assert L.Vship_ResetCVVDP(abi.CVVDPHandler(12345)) == abi.BadHandler
    L.Vship_CVVDPFree.argtypes = [abi.CVVDPHandler]
    assert L.Vship_CVVDPFree(abi.CVVDPHandler(12345)) == abi.BadHandler


def test_struct_layouts_match_c():
    # sizes of the ABI structs as a C compiler lays them out
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "VshipAPI.h"
#include "VshipAPI_ext.h"
int main(void){
 printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(Vship_Colorspace_t), offsetof(Vship_Colorspace_t, sample),
        offsetof(Vship_Colorspace_t, crop), sizeof(Vship_DeviceInfo), sizeof(Vship_ButteraugliScore), sizeof(Vship_Version),
        sizeof(VshipExt_FramePair), offsetof(VshipExt_FramePair, srcp1), offsetof(VshipExt_FramePair, lineSize2));
 return 0;}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert vals == [ctypes.sizeof(abi.Colorspace), abi.Colorspace.sample.offset, abi.Colorspace.crop.offset,
                    ctypes.sizeof(abi.DeviceInfo), ctypes.sizeof(abi.ButteraugliScore), ctypes.sizeof(abi.Version),
                    ctypes.sizeof(abi.FramePair), abi.FramePair.srcp1.offset, abi.FramePair.lineSize2.offset]


def test_ssimu2_weights_match_reference_source():
    """The 108 SSIMULACRA2 weights the engine, the oracle and the tests share
    (vship_b200/csrc/metric_tables.h) are the reference's own float array
    (src/ssimu2/score.hpp:5-113), compared value for value after rounding both to float."""
    import numpy as np
    from tests import tables
    src = os.path.join(os.environ.get("VSHIP_REFERENCE_ROOT", "/root/reference"), "src", "ssimu2", "score.hpp")
    if not os.path.exists(src):
        pytest.skip("reference sources not present")
    text = open(src).read()
    body = text[text.index("weights[108]"):]
    body = body[body.index("{") + 1:body.index("}")]
    ref = np.array([float(v) for v in re.findall(r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?", body)], dtype=np.float32)
    assert ref.size == 108
    np.testing.assert_array_equal(tables.weights().astype(np.float32), ref)
    prune = float(re.search(r"weight_pruning\s*=\s*([0-9.]+)f", text).group(1))
    assert np.float32(prune) == np.float32(0.01)
