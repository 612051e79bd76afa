"""The VapourSynth plugin entry (VapourSynthPluginInit2) driven by a fake VapourSynth host.

tests/vsfake/vsfake.c stands in for a VapourSynth core: it implements the API slots the plugin
calls, registers the plugin's functions, builds clips from numpy frames and requests frames the
way VapourSynth does (arInitial, then arAllFramesReady).  Registration, argument checking and
the error paths run on the CPU; frame scoring runs on the GPU and must give exactly what the
library's C ABI gives for the same planes (the plugin scores through that ABI).

The registered names and argument strings are the reference's (src/VshipLib.cpp:63-67); the
frame properties are the reference's (src/ssimu2/vapoursynth.hpp, src/butter/vapoursynth.hpp).
"""
import ctypes
import json
import os
import subprocess
import threading

import numpy as np
import pytest

from vship_b200 import abi, api

HERE = os.path.dirname(os.path.abspath(__file__))
VS_ABI = os.path.join(os.path.dirname(HERE), "vship_b200", "csrc", "vs_abi.h")

CF_GRAY, CF_RGB, CF_YUV = 1, 2, 3
ST_INT, ST_FLOAT = 0, 1

REGISTERED = [
    ("SSIMULACRA2", "reference:vnode;distorted:vnode;numStream:int:opt;gpu_id:int:opt;", "clip:vnode;"),
    ("BUTTERAUGLI", "reference:vnode;distorted:vnode;qnorm:int:opt;intensity_multiplier:float:opt;"
                    "distmap:int:opt;numStream:int:opt;gpu_id:int:opt;", "clip:vnode;"),
    ("CVVDP", "reference:vnode;distorted:vnode;model_name:data:opt;model_config_json:data:opt;"
              "resizeToDisplay:int:opt;distmap:int:opt;gpu_id:int:opt;", "clip:vnode;"),
    ("GpuInfo", "gpu_id:int:opt;", "gpu_human_data:data;"),
]


@pytest.fixture(scope="module")
def host(vship_lib, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("vsfake") / "libvsfake.so")
    subprocess.run(["gcc", "-O1", "-shared", "-fPIC", "-o", out, os.path.join(HERE, "vsfake", "vsfake.c"), "-ldl"],
                   check=True)
    L = ctypes.CDLL(out)
    vp, cp, ip = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int
    L.vsfake_load.argtypes = [cp]
    L.vsfake_registered.argtypes = [ip, cp, cp, cp]
    L.vsfake_plugin.argtypes = [cp, cp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.vsfake_source.restype = vp
    L.vsfake_source.argtypes = [ip, ip, ip, ip, ip, ip, vp]
    L.vsfake_call.restype = vp
    L.vsfake_call.argtypes = [cp, vp, vp, cp, cp, cp, cp]
    L.vsfake_frame.argtypes = [vp, ip, cp, ctypes.POINTER(ctypes.c_double), vp, cp]
    L.vsfake_free_node.argtypes = [vp]
    from vship_b200 import build
    n = L.vsfake_load(build.OUT.encode())
    assert n == len(REGISTERED), n
    return L


def source(L, frames, cf=CF_RGB, st=ST_FLOAT, bits=32):
    """frames: array [n][3 or 1][h][w] of the sample type."""
    frames = np.ascontiguousarray(frames)
    n, _, h, w = frames.shape
    node = L.vsfake_source(w, h, n, cf, st, bits, frames.ctypes.data)
    source.keep.append(frames)
    return node


source.keep = []


def call(L, name, ref, dis, ints="", floats="", datas=""):
    """ints / floats / datas: "key=value" lists separated by ';'."""
    err = ctypes.create_string_buffer(4096)
    node = L.vsfake_call(name.encode(), ref, dis, ints.encode(), floats.encode(), datas.encode(), err)
    return node, err.value.decode()


def frame(L, node, n, prop, plane0=None):
    v = ctypes.c_double()
    err = ctypes.create_string_buffer(4096)
    rc = L.vsfake_frame(node, n, prop.encode(), ctypes.byref(v), plane0.ctypes.data if plane0 is not None else None,
                        err)
    assert rc == 0, err.value.decode()
    return v.value


def rgbs_clip(n, w, h, seed):
    rng = np.random.default_rng(seed)
    base = rng.random((n, 3, h, w), dtype=np.float32)
    k = np.ones(5, np.float32) / 5
    smooth = np.apply_along_axis(lambda r: np.convolve(r, k, mode="same"), 3, base)
    return smooth.astype(np.float32)


# ---------------------------------------------------------------------------------------- CPU


def _vs4_header():
    root = os.environ.get("VSHIP_REFERENCE_ROOT", "/root/reference")
    p = os.path.join(root, "include", "VapourSynth4.h")
    return p if os.path.exists(p) else None


def test_abi_layout_matches_vapoursynth4_header(tmp_path):
    """Every slot and structure field the plugin uses sits where the public VapourSynth 4 header
    puts it (checked at compile time by offsetof)."""
    hdr = _vs4_header()
    if hdr is None:
        pytest.skip("VapourSynth4.h not available")
    slots = ["createVideoFilter", "freeNode", "getVideoInfo", "newVideoFrame", "freeFrame", "copyFrame",
             "getFramePropertiesRW", "getStride", "getReadPtr", "getWritePtr", "getFrameWidth", "getFrameHeight",
             "queryVideoFormat", "getFrameFilter", "requestFrameFilter", "setFilterError", "createMap", "freeMap",
             "mapSetError", "mapGetError", "mapGetInt", "mapSetInt", "mapGetFloat", "mapSetFloat", "mapGetData",
             "mapSetData",
             "mapGetNode", "mapConsumeNode", "getPluginByID", "invoke", "getCoreInfo"]
    structs = {
        ("VsAbiVideoFormat", "VSVideoFormat"): ["colorFamily", "sampleType", "bitsPerSample", "bytesPerSample",
                                                "subSamplingW", "subSamplingH", "numPlanes"],
        ("VsAbiVideoInfo", "VSVideoInfo"): ["format", "fpsNum", "fpsDen", "width", "height", "numFrames"],
        ("VsAbiCoreInfo", "VSCoreInfo"): ["versionString", "core", "api", "numThreads", "maxFramebufferSize",
                                          "usedFramebufferSize"],
        ("VsAbiFilterDependency", "VSFilterDependency"): ["source", "requestPattern"],
        ("VsAbiPluginApi", "VSPLUGINAPI"): ["getAPIVersion", "configPlugin", "registerFunction"],
    }
    enums = [("vsCfGray", "cfGray"), ("vsCfRGB", "cfRGB"), ("vsCfYUV", "cfYUV"), ("vsStInteger", "stInteger"),
             ("vsStFloat", "stFloat"), ("vsArInitial", "arInitial"), ("vsArAllFramesReady", "arAllFramesReady"),
             ("vsFmParallel", "fmParallel"), ("vsFmParallelRequests", "fmParallelRequests"),
             ("vsRpStrictSpatial", "rpStrictSpatial"), ("vsMaReplace", "maReplace"),
             ("vsPeSuccess", "peSuccess"), ("vsDtUtf8", "dtUtf8"), ("VS_ABI_API_VERSION", "VAPOURSYNTH_API_VERSION"),
             ("VS_ABI_MAKE_VIDEO_ID(vsCfRGB, vsStFloat, 32, 0, 0)", "pfRGBS")]
    lines = ['#include "%s"' % hdr, '#include "%s"' % VS_ABI,
             "_Static_assert(sizeof(VsAbiApi) == offsetof(VSAPI, getCoreInfo) + sizeof(void*), \"slot count\");"]
    for s in slots:
        lines.append('_Static_assert(offsetof(VsAbiApi, %s) == offsetof(VSAPI, %s), "%s");' % (s, s, s))
    for (mine, theirs), fields in structs.items():
        lines.append('_Static_assert(sizeof(%s) == sizeof(%s), "%s");' % (mine, theirs, mine))
        for f in fields:
            lines.append('_Static_assert(offsetof(%s, %s) == offsetof(%s, %s), "%s.%s");' % (mine, f, theirs, f,
                                                                                           mine, f))
    for mine, theirs in enums:
        lines.append('_Static_assert((%s) == (%s), "%s");' % (mine, theirs, mine))
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_registration(host):
    name, args, ret = (ctypes.create_string_buffer(512) for _ in range(3))
    got = []
    for i in range(len(REGISTERED)):
        assert host.vsfake_registered(i, name, args, ret) == 0
        got.append((name.value.decode(), args.value.decode(), ret.value.decode()))
    assert got == REGISTERED
    pid, ns = ctypes.create_string_buffer(128), ctypes.create_string_buffer(64)
    ver, apiv = ctypes.c_int(), ctypes.c_int()
    host.vsfake_plugin(pid, ns, ctypes.byref(ver), ctypes.byref(apiv))
    assert (pid.value, ns.value, ver.value, apiv.value) == (b"com.lumen.vship", b"vship", (4 << 16) | 1, 4 << 16)


@pytest.mark.gpu
def test_cvvdp_bad_display(gpu, host):
    a = source(host, rgbs_clip(1, 64, 48, 1))
    node, err = call(host, "CVVDP", a, a, datas="model_name=no_such_display")
    assert node is None and "BadDisplayModel" in err, err


def test_non_rgbs_without_resize_plugin(host):
    """A YUV clip needs the resize plugin (src/util/torgbs.hpp); the fake core has none."""
    yuv = source(host, np.zeros((1, 3, 48, 64), np.uint8), cf=CF_YUV, st=ST_INT, bits=8)
    rgb = source(host, rgbs_clip(1, 64, 48, 2))
    for fn in ("SSIMULACRA2", "BUTTERAUGLI", "CVVDP"):
        node, err = call(host, fn, yuv, rgb)
        assert node is None and "com.vapoursynth.resize" in err, err


def test_differing_clips_rejected(host):
    a = source(host, rgbs_clip(1, 64, 48, 3))
    b = source(host, rgbs_clip(1, 64, 40, 4))
    for fn in ("SSIMULACRA2", "BUTTERAUGLI", "CVVDP"):
        node, err = call(host, fn, a, b)
        assert node is None
        assert api.error_message(4) in err, err


# ---------------------------------------------------------------------------------------- GPU


def _rgbs_cs(w, h):
    return abi.colorspace(w, h, sample=abi.SampleFLOAT, transfer=abi.TRC_BT709)


def _planes(frames, k):
    return [np.ascontiguousarray(frames[k, c]) for c in range(3)], [frames.shape[3] * 4] * 3


@pytest.mark.gpu
def test_ssimulacra2_frames_match_c_abi(gpu, host):
    n, w, h = 4, 300, 200  # 1200-byte rows, padded to 1216 by the host
    ref, dis = rgbs_clip(n, w, h, 10), rgbs_clip(n, w, h, 10)
    dis += np.float32(0.03) * rgbs_clip(n, w, h, 11)
    node, err = call(host, "SSIMULACRA2", source(host, ref), source(host, dis), ints="numStream=2")
    assert node is not None, err
    want = []
    with api.SSIMU2(_rgbs_cs(w, h)) as s:
        for k in range(n):
            p1, ls = _planes(ref, k)
            p2, _ = _planes(dis, k)
            want.append(s.compute(p1, p2, ls))
    # frames requested from four threads share the filter's two handlers
    got = [None] * n
    threads = [threading.Thread(target=lambda k=k: got.__setitem__(k, frame(host, node, k, "_SSIMULACRA2")))
               for k in range(n)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert got == want
    assert all(10.0 < v < 100.0 for v in got), got
    host.vsfake_free_node(node)


@pytest.mark.gpu
def test_butteraugli_frames_and_distmap_match_c_abi(gpu, host):
    n, w, h = 2, 256, 160
    ref, dis = rgbs_clip(n, w, h, 20), rgbs_clip(n, w, h, 20)
    dis[:, :, 40:80, 60:120] *= np.float32(0.8)
    node, err = call(host, "BUTTERAUGLI", source(host, ref), source(host, dis), ints="qnorm=3;distmap=1",
                      floats="intensity_multiplier=250")
    assert node is not None, err
    with api.Butteraugli(_rgbs_cs(w, h), qnorm=3, intensity=250.0) as b:
        for k in range(n):
            p1, ls = _planes(ref, k)
            p2, _ = _planes(dis, k)
            norms, dmap = b.compute(p1, p2, ls, distmap=True)
            got = np.zeros((h, w), np.float32)
            q = frame(host, node, k, "_BUTTERAUGLI_QNorm", got)
            assert q == norms[0]
            assert frame(host, node, k, "_BUTTERAUGLI_3Norm") == norms[1]
            assert frame(host, node, k, "_BUTTERAUGLI_INFNorm") == norms[2]
            np.testing.assert_array_equal(got, dmap)
    host.vsfake_free_node(node)


@pytest.mark.gpu
def test_cvvdp_frames_match_c_abi(gpu, host, tmp_path):
    """A CVVDP clip scores its frames in order through one handler: the _CVVDP property of
    frame n is the JOD of frames 0..n, as the C ABI gives it; distmap=1 returns the map at the
    display size (resizeToDisplay with a custom display from model_config_json)."""
    n, w, h = 5, 192, 108
    ref, dis = rgbs_clip(n, w, h, 30), rgbs_clip(n, w, h, 30)
    dis += np.float32(0.02) * rgbs_clip(n, w, h, 31)
    node, err = call(host, "CVVDP", source(host, ref), source(host, dis), datas="model_name=standard_4k")
    assert node is not None, err
    got = [frame(host, node, k, "_CVVDP") for k in range(n)]
    host.vsfake_free_node(node)
    with api.CVVDP(_rgbs_cs(w, h), fps=24.0, model="standard_4k") as c:
        want = []
        for k in range(n):
            p1, ls = _planes(ref, k)
            p2, _ = _planes(dis, k)
            want.append(c.compute(p1, p2, ls))
    assert got == want
    assert all(5.0 < v <= 10.0 for v in got), got
    disp = {"name": "t", "colorspace": "sRGB", "resolution": [96, 54], "viewing_distance_meters": 0.5,
            "diagonal_size_inches": 10.0, "max_luminance": 250.0, "contrast": 800.0, "E_ambient": 100.0}
    path = str(tmp_path / "d.json")
    json.dump({"tiny": disp}, open(path, "w"))
    node, err = call(host, "CVVDP", source(host, ref), source(host, dis), ints="resizeToDisplay=1;distmap=1",
                     datas="model_name=tiny;model_config_json=" + path)
    assert node is not None, err
    dmap = np.zeros((54, 96), np.float32)
    v0 = frame(host, node, 0, "_CVVDP", dmap)
    host.vsfake_free_node(node)
    with api.CVVDP(_rgbs_cs(w, h), fps=24.0, model="tiny", model_config_json=path, resize_to_display=True) as c:
        p1, ls = _planes(ref, 0)
        p2, _ = _planes(dis, 0)
        s0, m0 = c.compute(p1, p2, ls, distmap=True)
    assert v0 == s0
    np.testing.assert_array_equal(dmap, m0)


@pytest.mark.gpu
def test_gpu_info(gpu, host):
    node, text = call(host, "GpuInfo", None, None)
    assert node is None and text.startswith("GPU 0: ")
    node, text = call(host, "GpuInfo", None, None, ints="gpu_id=0")
    assert "MultiProcessorCount: " in text and "PassKernelCheck : 1" in text
