"""Builds libvship.so (the C-ABI drop-in) in-tree with nvcc for sm_100a.

    python -m vship_b200.build [--force]

Each .cu in csrc/ compiles to an object in parallel; they link into vship_b200/libvship.so
with the CUDA runtime linked statically, so the library has no dependency beyond the driver.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libvship.so")
BUILD_DIR = os.path.join(HERE, "_build")
# Bounds-check build (-DVSHIP_BOUNDS_CHECK): guard bands around every device buffer, checked
# after each API call; used by tests/test_bounds_check_gpu.py, never by the product path.
OUT_BC = os.path.join(HERE, "libvship_bc.so")
BUILD_DIR_BC = os.path.join(HERE, "_build_bc")
SOURCES = ["api.cu", "ssimu2.cu", "ssimu2_batch.cu", "surrogate.cu", "butter.cu", "cvvdp.cu", "vsplugin.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                     "-Xcudafe", "--diag_suppress=177", "--expt-relaxed-constexpr"]


def nvcc():
    exe = shutil.which("nvcc")
    if exe:
        return exe
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found")


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    inc = os.path.join(os.path.dirname(HERE), "include")
    files += [os.path.join(inc, f) for f in os.listdir(inc)]
    files.append(os.path.abspath(__file__))
    return max(os.path.getmtime(f) for f in files)


def build(force=False, verbose=False, bounds_check=False):
    out, build_dir = (OUT_BC, BUILD_DIR_BC) if bounds_check else (OUT, BUILD_DIR)
    if not force and os.path.exists(out) and os.path.getmtime(out) >= _deps():
        return out
    os.makedirs(build_dir, exist_ok=True)
    exe = nvcc()
    extra = ["-DVSHIP_BOUNDS_CHECK"] if bounds_check else []

    def compile_one(src):
        obj = os.path.join(build_dir, os.path.splitext(src)[0] + ".o")
        cmd = [exe] + NVCC_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = out + ".tmp"
    cmd = [exe] + ARCH + ["-shared", "-Xlinker", "-Bsymbolic", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, bounds_check="--bounds-check" in sys.argv))
