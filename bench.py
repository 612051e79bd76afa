"""Benchmark of the SSIMULACRA2 hot path: 1080p frame pairs per second on B200.

Workload (the configuration the headline metric is quoted on): batches of 64 frame pairs,
1920x1080 Y'CbCr 4:2:0, 10-bit limited range, BT.709 matrix/transfer/primaries, seeded
synthetic content (sinusoid sums + noise, distorted by 8x8 DCT quantisation with per-frame
steps in [4, 48] and the 4:2:0 chroma round trip).  One step scores one batch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm prints one JSON line with
  value       device-resident throughput (inputs already in HBM, VshipExt_ComputeSSIMU2Device
              on 64 pairs per call), CUDA events on the launching stream, max over ranks;
  e2e         the same metric through Vship_ComputeSSIMU2 with pinned host buffers
              (host->device copies and the score read-back inside the timed region);
  roofline    achieved HBM bandwidth of the dominant kernel (algorithmic bytes per launch /
              its average CUDA-event launch duration) against MEASURED_PEAKS.json;
  cpu_baseline  the FP64 oracle on all host cores, on a bounded sample of the same workload.
The reference arm runs the unmodified Vship library built from its own sources
(oracle/_ref/libvship_ref.so) through its own C API, with pinned host buffers and the
best of several handler/thread counts, on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, BATCH = 1920, 1080, 64
WORKLOAD = "ssimu2_1080p_yuv420p10_bt709_batch64"
METRIC = "1080p SSIMU2 frame-pairs/s"
UNIT = "frame-pairs/s"

# Algorithmic bytes per 1080p pair: the front kernel reads the
# raw 10-bit 4:2:0 planes of both frames and writes the XYB planes the maps read; the maps
# kernel reads those planes once.
RAW_BYTES_PER_IMAGE = 1920 * 1080 * 2 + 2 * 960 * 540 * 2
XYB_FLOATS_PER_IMAGE = 1920 * 1080 + 2 * 960 * 540 + 2 * 480 * 270 + 3 * 240 * 135 + 3 * 120 * 68
ALGO_BYTES = {
    "ssimu2_front": 2 * (RAW_BYTES_PER_IMAGE + 4 * XYB_FLOATS_PER_IMAGE),
    "ssimu2_maps": 2 * 4 * XYB_FLOATS_PER_IMAGE,
    "ssimu2_final": 0,
}


def maps_flop_per_pair(w, h):
    """FP32 arithmetic of the maps kernel for one pair: every unpruned (plane, level) is cut into
    32 x 32 output tiles, and each output position costs ~370 FLOP (the horizontal 17-tap pass
    over 1.5x the rows for four moment inputs, 204; the vertical pass, 136; the maps, ~30)."""
    planes = [1, 2, 2, 3, 3]  # Y at level 0; X, Y at 1-2; X, Y, B at 3-4; level 5 pruned
    tiles = 0
    for n in planes:
        tiles += n * (-(-w // 32)) * (-(-h // 32))
        w, h = (w - 1) // 2 + 1, (h - 1) // 2 + 1
    return tiles * 1024 * 370


B200_SMS = 148
FP32_LANES_PER_SM = 128


def fp32_peak_tflops(clocks):
    """FP32 SIMT peak at the SM clock sampled during the timed region: SMs x FP32 lanes x 2
    FLOP per FMA x clock.  Falls back to the maximum SM clock (1965 MHz) without samples."""
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz") or 1965.0
    return round(B200_SMS * FP32_LANES_PER_SM * 2 * mhz * 1e6 / 1e12, 2), \
        "%d SMs x %d FP32 lanes x 2 x %.0f MHz (sampled SM clock)" % (B200_SMS, FP32_LANES_PER_SM, mhz)


def traffic_of(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/traffic.json),
    with its provenance, or (None, None)."""
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(tp):
        return None, None
    with open(tp) as f:
        tr = json.load(f).get(kernel)
    return (tr.get("bytes_per_launch"), tr.get("source")) if tr else (None, None)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = open(os.devnull, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=self.out, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            text, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            text = ""
        rows = [l.split(",") for l in text.strip().splitlines() if l.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_workload(seed):
    from vship_b200 import synth
    t = time.time()
    pairs = synth.make_pairs(BATCH, W, H, fmt="yuv420p10", seed=seed, unique=8, steps=(4.0, 48.0))
    log("generated %d pairs in %.1fs" % (len(pairs), time.time() - t))
    return pairs


def pinned_frames(pairs, api, lib=None):
    """Each frame in one page-locked buffer with its planes back to back, the layout FFVship
    (the reference's own client) gives Vship_ComputeSSIMU2 (src/ffvship_utility/ffmpegmain.hpp:630-637)."""
    pinned, host_pairs = [], []
    for p1, p2, _ in pairs:
        frames = []
        for planes in (p1, p2):
            nbytes = sum(p.nbytes for p in planes)
            pb = api.PinnedBuffer(nbytes, lib=lib)
            off, ptrs = 0, []
            for p in planes:
                pb.array[off:off + p.nbytes] = p.view(np.uint8).reshape(-1)
                ptrs.append(pb.ptr.value + off)
                off += p.nbytes
            pinned.append(pb)
            frames.append(ptrs)
        host_pairs.append((frames[0], frames[1]))
    return pinned, host_pairs


def input_bytes(pairs):
    return sum(p.nbytes for pr in pairs for p in pr[0] + pr[1])


def run_ours(args, world, rank, local):
    import torch
    from vship_b200 import abi, api
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    cs = abi.yuv420_10bit_bt709(W, H)
    pairs = make_workload(seed=1234 + rank)
    ls = pairs[0][2]

    # ---------------- device-resident throughput (value) ----------------
    dev = []
    for p1, p2, _ in pairs:
        dev.append(([torch.from_numpy(p.view(np.uint8)).cuda() for p in p1],
                    [torch.from_numpy(p.view(np.uint8)).cuda() for p in p2]))
    ptr1 = [t.data_ptr() for d in dev for t in d[0]]
    ptr2 = [t.data_ptr() for d in dev for t in d[1]]
    scores = torch.zeros(BATCH, dtype=torch.float64, device="cuda")
    h = api.SSIMU2(cs, gpu_id=local)
    stream = torch.cuda.current_stream()

    def step():
        h.compute_device(BATCH, ptr1, ptr2, ls, ls, scores.data_ptr(), 0, stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = t.item()
    ms_per_step = ms / args.steps
    value = BATCH * world * args.steps / (ms / 1e3)
    dev_scores = scores.cpu().numpy()

    # ---------------- per-kernel timing for the roofline ----------------
    h.kernel_timing(True)
    h.kernel_times(reset=True)
    for _ in range(max(3, args.steps // 2)):
        step()
    torch.cuda.synchronize()
    ktimes = h.kernel_times(reset=True)
    h.kernel_timing(False)
    top = max(ktimes.items(), key=lambda kv: kv[1][1])
    top_name, (launches, total_ms) = top
    avg_ms = total_ms / launches
    peak, peak_kind = measured_peaks()
    achieved = ALGO_BYTES[top_name] * BATCH / (avg_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": top_name, "achieved": round(achieved, 1), "peak": peak,
                "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": None, "algorithmic_bytes_per_launch": ALGO_BYTES[top_name] * BATCH,
                "avg_launch_ms": round(avg_ms, 4),
                "kernels_ms_per_launch": {k: round(v[1] / v[0], 4) for k, v in ktimes.items()}}
    if top_name == "ssimu2_maps":
        # The maps kernel is arithmetic-bound (47 FLOP per algorithmic byte, far right of the
        # FP32 ridge): its compute fraction is the descriptive figure.
        flop = maps_flop_per_pair(W, H) * BATCH
        tf = flop / (avg_ms / 1e3) / 1e12
        pk = fp32_peak_tflops(clocks)
        roofline["compute"] = {"flop_per_launch": flop, "achieved_tflops": round(tf, 2),
                               "peak_tflops": pk[0], "peak_source": pk[1], "frac": round(tf / pk[0], 4)}
    roofline["traffic"], src = traffic_of(top_name)
    if src:
        roofline["traffic_source"] = src

    # ---------------- end to end through the C ABI (e2e) ----------------
    nthreads = args.e2e_threads
    pinned, host_pairs = pinned_frames(pairs, api)
    handlers = [api.SSIMU2(cs, gpu_id=local) for _ in range(nthreads)]
    e2e_scores = np.zeros(BATCH)

    def worker(k):
        torch.cuda.set_device(local)
        for i in range(k, BATCH, nthreads):
            e2e_scores[i] = handlers[k].compute(host_pairs[i][0], host_pairs[i][1], ls, ls)

    def e2e_step():
        ths = [threading.Thread(target=worker, args=(k,)) for k in range(nthreads)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = t.item()
    e2e_value = BATCH * world * args.steps / e2e_s
    max_dev = float(np.max(np.abs(e2e_scores - dev_scores)))
    for hh in handlers:
        hh.close()
    h.close()
    for pb in pinned:
        pb.free()

    # ---------------- CPU baseline: FP64 oracle on a bounded sample ----------------
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(pairs, cs, budget_s=args.cpu_seconds)
        cpu["max_abs_dscore_vs_fp64"] = cpu.pop("_maxd", None)
        # accuracy of our scores on the same sample against FP64
        cpu_err = float(np.max(np.abs(np.array(cpu.pop("_scores")) - dev_scores[:cpu["_n"]])))
        cpu.pop("_n")
        cpu["max_abs_dscore_gpu_vs_fp64"] = cpu_err

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "pairs_per_step": BATCH, "width": W, "height": H,
                   "format": "YUV420 10-bit limited BT.709", "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs (%.0f MB per step) larger than L2" % (input_bytes(pairs) / 1e6)},
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT,
                "api": "Vship_ComputeSSIMU2, each frame in one pinned buffer (FFVship layout)",
                "threads_handlers": nthreads, "timer": "wall clock, synchronised",
                "h2d_bytes_per_step": input_bytes(pairs), "d2h_bytes_per_step": BATCH * (8 + 108 * 4),
                "max_abs_score_diff_vs_device_path": max_dev},
        "gpu_launches": 3 * args.steps,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_baseline(pairs, cs, budget_s=12.0):
    import oracle
    oracle.build()
    n, t0, scores, maxd = 0, time.perf_counter(), [], 0.0
    while n < len(pairs) and (time.perf_counter() - t0) < budget_s:
        p1, p2, ls = pairs[n]
        q, d, _ = oracle.ssimu2(oracle.convert(p1, ls, cs), oracle.convert(p2, ls, cs))
        scores.append(d)
        maxd = max(maxd, abs(q - d))
        n += 1
    dt = time.perf_counter() - t0
    return {"value": round(n / dt, 3), "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
            "sample": "%d of the workload's 1080p pairs, colour conversion + SSIMU2 in FP64 (%.1f s)" % (n, dt),
            "_scores": scores, "_n": n, "_maxd": maxd}


def run_reference(args, world, rank, local):
    if rank != 0:
        return
    from vship_b200 import abi, api
    ref = os.path.join(ROOT, "oracle", "_ref", "libvship_ref.so")
    if not os.path.exists(ref):
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libvship_ref.so was not built"}))
        return
    import torch
    torch.cuda.set_device(local)
    L = api.load_library(ref)
    cs = abi.yuv420_10bit_bt709(W, H)
    pairs = make_workload(seed=1234)
    ls = pairs[0][2]
    pinned, host_pairs = pinned_frames(pairs, api, lib=L)
    best = None
    for nthreads in args.ref_threads:
        handlers = [api.SSIMU2(cs, gpu_id=local, lib=L) for _ in range(nthreads)]
        out = np.zeros(BATCH)

        def worker(k):
            torch.cuda.set_device(local)
            for i in range(k, BATCH, nthreads):
                out[i] = handlers[k].compute(host_pairs[i][0], host_pairs[i][1], ls, ls)

        def step():
            ths = [threading.Thread(target=worker, args=(k,)) for k in range(nthreads)]
            for t in ths:
                t.start()
            for t in ths:
                t.join()

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        v = BATCH * args.steps / dt
        log("reference: %d handlers/threads -> %.1f pairs/s" % (nthreads, v))
        if best is None or v > best[0]:
            best = (v, nthreads, dt)
        for hh in handlers:
            hh.close()
    for pb in pinned:
        pb.free()
    v, nthreads, dt = best
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "pairs_per_step": BATCH, "width": W, "height": H,
                   "format": "YUV420 10-bit limited BT.709",
                   "library": "Vship 4.1.0 built from its sources with nvcc for sm_100a (oracle/build_ref.sh)",
                   "api": "Vship_ComputeSSIMU2, each frame in one pinned buffer (FFVship layout)",
                   "threads_handlers": nthreads,
                   "threads_swept": args.ref_threads},
        "e2e": {"value": round(v, 2), "unit": UNIT, "h2d_bytes_per_step": input_bytes(pairs),
                "d2h_bytes_per_step": BATCH * 4 * 108},
        "cpu_baseline": {"value": round(v, 2), "unit": UNIT, "kind": "reference", "cores": nthreads,
                         "sample": "%d steps of %d pairs; the reference has no CPU implementation, so its own CUDA "
                                   "build runs on the B200, driven by %d host threads" % (args.steps, BATCH, nthreads)},
    }
    print(json.dumps(line), flush=True)


PWORKLOAD = "ssimu2_1080p_srgb8_single_pair"
SCOPIES = 16  # distinct copies of the pair cycled through, 199 MB of input: larger than L2
RGB8_BYTES_PER_IMAGE = 3 * W * H


def single_pair(rank):
    """One 1080p 8-bit sRGB pair (full range, BT.709 primaries) as the single-pair
    configuration describes it: sinusoid-sum content + N(0, 3) noise, distorted by 8x8 DCT
    quantisation with step 16."""
    from vship_b200 import synth
    return synth.make_pairs(1, W, H, fmt="rgb8", seed=4321 + rank, steps=16.0)[0]


def streams_rate(streams, enqueue, calls, warmup):
    """Device time of `calls` asynchronous calls dealt round-robin over `streams` (call i on
    stream i % len(streams)), all enqueued from this thread: CUDA events on the current stream,
    which every stream waits for before its first call and which waits for every stream after
    its last.  Returns calls per second."""
    import torch
    main = torch.cuda.current_stream()

    def run(n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        for s_ in streams:
            s_.wait_event(e0)
        for i in range(n):
            enqueue(i, streams[i % len(streams)])
        for s_ in streams:
            ev = torch.cuda.Event()
            ev.record(s_)
            main.wait_event(ev)
        e1.record(main)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    run(warmup)
    return calls / (run(calls) / 1e3)


def single_e2e(api, cs, host_pairs, ls, local, threads_list, calls, warmup, lib=None):
    """Through Vship_ComputeSSIMU2 (host frames): latency of one thread's sequential calls and
    the best throughput over T threads with a handler each, every call scoring one pair of the
    cycled copies.  Returns (latency_ms, best pairs/s, its thread count, {T: pairs/s})."""
    import torch
    sweep = {}
    lat = None
    for nthreads in threads_list:
        handlers = [api.SSIMU2(cs, gpu_id=local, lib=lib) for _ in range(nthreads)]

        def worker(k, n):
            torch.cuda.set_device(local)
            for i in range(n):
                fr = host_pairs[(k * 7 + i) % len(host_pairs)]
                handlers[k].compute(fr[0], fr[1], ls, ls)

        def run(n):
            ths = [threading.Thread(target=worker, args=(k, n)) for k in range(nthreads)]
            for t in ths:
                t.start()
            for t in ths:
                t.join()

        run(warmup)
        t0 = time.perf_counter()
        run(calls)
        dt = time.perf_counter() - t0
        sweep[nthreads] = round(nthreads * calls / dt, 2)
        if nthreads == 1:
            lat = dt / calls * 1e3
        for hh in handlers:
            hh.close()
    best_t = max(sweep, key=sweep.get)
    return lat, sweep[best_t], best_t, sweep


def run_single(args, rank, local, reference=False):
    """Single-pair configuration: one 1080p 8-bit sRGB pair per call.  The reference's own
    benchmark separates latency (sequential calls) from throughput (several threads and
    handlers, test/apibenchmark.cpp:110-117); both are reported, for the device-resident entry
    (ours only) and end to end through Vship_ComputeSSIMU2 with pinned host frames."""
    import torch
    from vship_b200 import abi, api
    torch.cuda.set_device(local)
    lib = None
    if reference:
        ref = os.path.join(ROOT, "oracle", "_ref", "libvship_ref.so")
        if not os.path.exists(ref):
            print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libvship_ref.so was not built"}))
            return
        lib = api.load_library(ref)
    cs = abi.srgb8(W, H)
    p1, p2, ls = single_pair(rank)
    pairs = [(p1, p2, ls)] * SCOPIES
    pinned, host_pairs = pinned_frames(pairs, api, lib=lib)
    calls = max(args.steps, 1) * SCOPIES
    threads = [1, 2, 3, 4, 8]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    lat, e2e, e2e_t, sweep = single_e2e(api, cs, host_pairs, ls, local, threads, calls, args.warmup * SCOPIES, lib=lib)
    if reference:
        clocks = sampler.stop()
    for pb in pinned:
        pb.free()
    config = {"workload": PWORKLOAD, "pairs_per_call": 1, "width": W, "height": H, "format": "RGB 8-bit full range sRGB",
              "distortion": "8x8 DCT quantisation, step 16",
              "l2": "%d copies of the pair cycled (%.0f MB of input, larger than L2)" % (SCOPIES, SCOPIES * 2 * RGB8_BYTES_PER_IMAGE / 1e6)}
    common = {"metric": "1080p SSIMU2 frame-pairs/s, single pair per call", "unit": UNIT, "n_gpus": 1,
              "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
              "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    e2e_obj = {"value": round(e2e, 2), "unit": UNIT, "api": "Vship_ComputeSSIMU2, each frame in one pinned buffer",
               "threads_handlers": e2e_t, "threads_swept": sweep, "latency_ms": round(lat, 4),
               "timer": "wall clock", "h2d_bytes_per_step": calls * 2 * RGB8_BYTES_PER_IMAGE,
               "d2h_bytes_per_step": calls * 8}
    if reference:
        line = dict(common, impl="reference", value=round(e2e, 2), ms_per_step=round(calls / e2e * 1e3, 3),
                    config=dict(config, library="Vship 4.1.0 built from its sources with nvcc for sm_100a "
                                "(oracle/build_ref.sh)", calls_per_step=calls),
                    e2e=e2e_obj, clocks=clocks,
                    cpu_baseline={"value": round(e2e, 2), "unit": UNIT, "kind": "reference", "cores": e2e_t,
                                  "sample": "%d calls per thread; the reference has no CPU implementation, so its "
                                            "own CUDA build runs on the B200" % calls})
        print(json.dumps(line), flush=True)
        return

    # device-resident: the pair copies in HBM, one pair per call on one stream
    dev = [([torch.from_numpy(p).cuda() for p in p1], [torch.from_numpy(p).cuda() for p in p2]) for _ in range(SCOPIES)]
    ptrs = [([t.data_ptr() for t in a], [t.data_ptr() for t in b]) for a, b in dev]
    score = torch.zeros(1, dtype=torch.float64, device="cuda")
    h = api.SSIMU2(cs, gpu_id=local)
    stream = torch.cuda.current_stream()

    def one(i):
        a, b = ptrs[i % SCOPIES]
        h.compute_device(1, a, b, ls, ls, score.data_ptr(), 0, stream.cuda_stream)

    for i in range(args.warmup * SCOPIES):
        one(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(calls):
        one(i)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    value = calls / (ms / 1e3)
    # per-call latency: host enqueue to completion of one call, calls one at a time
    lats = []
    for i in range(min(calls, 64)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        one(i)
        torch.cuda.synchronize()
        lats.append((time.perf_counter() - t0) * 1e3)
    h.kernel_timing(True)
    h.kernel_times(reset=True)
    for i in range(calls):
        one(i)
    torch.cuda.synchronize()
    ktimes = h.kernel_times(reset=True)
    h.kernel_timing(False)
    got = float(score.item())
    h.close()
    # throughput with several callers (the reference's own throughput method uses several
    # threads and handlers): k handlers, each on its own stream, one pair per call
    stream_sweep = {}
    for k in (1, 2, 4, 8):
        hs = [api.SSIMU2(cs, gpu_id=local) for _ in range(k)]
        outs = torch.zeros(k, dtype=torch.float64, device="cuda")
        streams = [torch.cuda.Stream() for _ in range(k)]

        def enq(i, st, hs=hs, outs=outs, k=k):
            a, b = ptrs[i % SCOPIES]
            hs[i % k].compute_device(1, a, b, ls, ls, outs[i % k:i % k + 1].data_ptr(), 0, st.cuda_stream)

        stream_sweep[k] = round(streams_rate(streams, enq, calls, args.warmup * SCOPIES), 2)
        if not np.all(outs.cpu().numpy() == got):
            raise SystemExit("concurrent handlers disagree with the single-handler score")
        for hh in hs:
            hh.close()
    clocks = sampler.stop()
    value = max(stream_sweep.values())
    top_name, (launches, total_ms) = max(ktimes.items(), key=lambda kv: kv[1][1])
    avg_ms = total_ms / launches
    peak, peak_kind = measured_peaks()
    algo = {"ssimu2_front": 2 * (RGB8_BYTES_PER_IMAGE + 4 * XYB_FLOATS_PER_IMAGE), "ssimu2_maps": 2 * 4 * XYB_FLOATS_PER_IMAGE,
            "ssimu2_final": 0}[top_name]
    achieved = algo / (avg_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": top_name, "achieved": round(achieved, 1), "peak": peak,
                "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                "algorithmic_bytes_per_launch": algo, "avg_launch_ms": round(avg_ms, 4),
                "kernels_ms_per_launch": {k: round(v[1] / v[0], 4) for k, v in ktimes.items()},
                "note": "one pair per launch: the pyramid (33 MB) stays in L2 between the front and maps kernels"}
    if top_name == "ssimu2_maps":
        flop = maps_flop_per_pair(W, H)
        tf = flop / (avg_ms / 1e3) / 1e12
        pk = fp32_peak_tflops(clocks)
        roofline["compute"] = {"flop_per_launch": flop, "achieved_tflops": round(tf, 2), "peak_tflops": pk[0],
                               "peak_source": pk[1], "frac": round(tf / pk[0], 4)}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        oracle.build()
        t0, n = time.perf_counter(), 0
        while n == 0 or (time.perf_counter() - t0) < min(args.cpu_seconds, 10.0):
            _, exact, _ = oracle.ssimu2(oracle.convert(p1, ls, cs), oracle.convert(p2, ls, cs))
            n += 1
        dt = time.perf_counter() - t0
        cpu = {"value": round(n / dt, 3), "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
               "sample": "the pair scored %d times by the FP64 oracle (colour conversion + SSIMU2, %.1f s)" % (n, dt),
               "max_abs_dscore_gpu_vs_fp64": abs(got - exact)}
    line = dict(common, value=round(value, 2), ms_per_step=round(calls / value * 1e3 / max(args.steps, 1), 4),
                config=dict(config, calls_per_step=SCOPIES, device_value="best over 1/2/4/8 handlers, each on "
                            "its own stream, one pair per call", handlers_swept=stream_sweep),
                latency_ms={"device_call_median": round(statistics.median(lats), 4),
                            "device_stream_per_pair": round(ms / calls, 4), "e2e_sequential": round(lat, 4)},
                e2e=e2e_obj, gpu_launches=3 * calls, roofline=roofline, cpu_baseline=cpu, clocks=clocks)
    print(json.dumps(line), flush=True)


BW, BH, BBATCH = 3840, 2160, 32
BWORKLOAD = "butteraugli_4k_srgb8_batch32_q5_i203_distmap"
BMETRIC = "4K Butteraugli frame-pairs/s"
# Algorithmic bytes per 4K Butteraugli pair (FP32 staged model: inputs, then per scale every
# opsin and band plane of both images written and read once, the accumulator and mask planes
# written and read, the per-scale diff map, and the final distortion map written).
B_ALGO_BYTES = 2_903_040_000
# Kernels per 8-bit sRGB pair call: 2 colour conversions, 6 downsamples, per scale 2 images x
# (opsin, lf row pass, lf column pass, mf, hf, mask) + 1 diff map, then combine + final norms.
B_LAUNCHES_PER_PAIR = 2 + 6 + 2 * (2 * 6 + 1) + 2


def run_butteraugli(args, world, rank, local):
    """Secondary line: Butteraugli on 4K 8-bit sRGB pairs (intensity 203, Q-norm 5, distortion
    map returned), device-resident and end to end through Vship_ComputeButteraugli."""
    import torch
    from vship_b200 import abi, api, synth
    torch.cuda.set_device(local)
    t = time.time()
    pairs = synth.make_pairs(BBATCH, BW, BH, fmt="rgb8", seed=77 + rank, unique=4, blur=(0.0, 1.5))
    log("generated %d 4K pairs in %.1fs" % (len(pairs), time.time() - t))
    cs = abi.srgb8(BW, BH)
    ls = pairs[0][2]
    dev = [([torch.from_numpy(p).cuda() for p in a], [torch.from_numpy(p).cuda() for p in b]) for a, b, _ in pairs]
    norms = torch.zeros(BBATCH, 3, dtype=torch.float64, device="cuda")
    dmap = torch.zeros(BH, BW, dtype=torch.float32, device="cuda")
    h = api.Butteraugli(cs, qnorm=5, intensity=203.0, gpu_id=local)
    stream = torch.cuda.current_stream()

    def step():
        for i, (d1, d2) in enumerate(dev):
            h.compute_device([x.data_ptr() for x in d1], [x.data_ptr() for x in d2], ls, ls,
                             norms[i].data_ptr(), dmap.data_ptr(), BW * 4, stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    dev_norms = norms.cpu().numpy().copy()
    # several callers: k handlers, each on its own stream and distortion map, pairs dealt round-robin
    stream_sweep = {1: round(BBATCH * args.steps / (ms / 1e3), 2)}
    for k in (2, 4):
        hs = [api.Butteraugli(cs, qnorm=5, intensity=203.0, gpu_id=local) for _ in range(k)]
        kn = torch.zeros(BBATCH, 3, dtype=torch.float64, device="cuda")
        dms = [torch.zeros(BH, BW, dtype=torch.float32, device="cuda") for _ in range(k)]
        streams = [torch.cuda.Stream() for _ in range(k)]

        def enq(i, st, hs=hs, kn=kn, dms=dms, k=k):
            d1, d2 = dev[i % BBATCH]
            hs[i % k].compute_device([x.data_ptr() for x in d1], [x.data_ptr() for x in d2], ls, ls,
                                     kn[i % BBATCH].data_ptr(), dms[i % k].data_ptr(), BW * 4, st.cuda_stream)

        stream_sweep[k] = round(streams_rate(streams, enq, BBATCH * args.steps, BBATCH * args.warmup), 2)
        if not np.array_equal(kn.cpu().numpy(), dev_norms):
            raise SystemExit("concurrent handlers disagree with the single-handler norms")
        for hh in hs:
            hh.close()
        del dms
    clocks = sampler.stop()
    value = max(stream_sweep.values())
    h.kernel_timing(True)
    h.kernel_times(reset=True)
    step()
    torch.cuda.synchronize()
    ktimes = h.kernel_times(reset=True)
    h.kernel_timing(False)
    per_pair_ms = {k: round(v[1] / BBATCH, 4) for k, v in ktimes.items()}
    h.close()
    e2e, e2e_threads, sweep = butter_e2e(args, pairs, cs, ls, local)
    peak, peak_kind = measured_peaks()
    achieved = B_ALGO_BYTES / (sum(v[1] for v in ktimes.values()) / BBATCH / 1e3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        import oracle
        oracle.build()
        k, t0, maxrel = 0, time.perf_counter(), 0.0
        while k < BBATCH and (k == 0 or time.perf_counter() - t0 < args.cpu_seconds):
            p1, p2, _ = pairs[k]
            on, _ = oracle.butteraugli(oracle.convert(p1, ls, cs), oracle.convert(p2, ls, cs), 203.0, 5)
            maxrel = max(maxrel, max(abs(dev_norms[k][j] - on[j]) / abs(on[j]) for j in range(3)))
            k += 1
        dt = time.perf_counter() - t0
        cpu = {"value": round(k / dt, 4), "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
               "sample": "first %d 4K pairs of the workload, colour conversion + Butteraugli in FP64 (%.1f s)" % (k, dt),
               "max_rel_dnorm_gpu_vs_fp64": maxrel}
    traffic, traffic_src = traffic_of("butteraugli_pair")
    line = {"metric": BMETRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(BBATCH / value * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": BWORKLOAD, "pairs_per_step": BBATCH, "width": BW, "height": BH,
                       "device_value": "best over 1/2/4 handlers, each on its own stream",
                       "handlers_swept": stream_sweep},
            "e2e": {"value": round(e2e, 2), "unit": UNIT,
                    "api": "Vship_ComputeButteraugli with distortion map, pinned frames",
                    "threads_handlers": e2e_threads, "threads_swept": sweep,
                    "h2d_bytes_per_step": BBATCH * 2 * 3 * BW * BH, "d2h_bytes_per_step": BBATCH * (BW * BH * 4 + 24)},
            "kernels_ms_per_pair": per_pair_ms,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                         "traffic_source": traffic_src, "algorithmic_bytes_per_pair": B_ALGO_BYTES,
                         "scope": "whole pipeline, per pair"},
            "gpu_launches": args.steps * BBATCH * B_LAUNCHES_PER_PAIR,
            "cpu_baseline": cpu, "clocks": clocks}
    print(json.dumps(line), flush=True)


CMETRIC = "1080p CVVDP frames/s"
CWORKLOAD = "cvvdp_1080p_yuv420p10_bt709_24fps_standard_fhd"
CFRAMES = 24  # frames per step and sequence: one second of 24 fps video


def run_cvvdp(args, rank, local, reference=False):
    """CVVDP over 1080p 10-bit 4:2:0 BT.709 sequences at 24 fps on the standard_fhd display,
    end to end through Vship_ComputeCVVDP with pinned host frames (the reference has no
    device-pointer entry); T concurrent sequences, each on its own handler and host thread,
    best of the swept T.  Both arms run the same frames; one step is CFRAMES frames of every
    sequence."""
    import threading
    import torch
    from vship_b200 import abi, api, synth
    torch.cuda.set_device(local)
    lib = None
    if reference:
        ref_path = os.path.join(ROOT, "oracle", "_ref", "libvship_ref.so")
        if not os.path.exists(ref_path):
            print(json.dumps({"impl": "reference", "unavailable": "reference library not built (oracle/build_ref.sh)"}))
            return
        lib = api.load_library(ref_path)
    t = time.time()
    pairs = synth.make_pairs(8, W, H, fmt="yuv420p10", seed=91 + rank, unique=8, steps=(4.0, 48.0))
    log("generated %d frame pairs in %.1fs" % (len(pairs), time.time() - t))
    cs = abi.yuv420_10bit_bt709(W, H)
    pinned, host_pairs = pinned_frames(pairs, api, lib=lib)
    ls = pairs[0][2]
    sweep = {}
    best = None
    for nthreads in args.cvvdp_threads:
        handlers = [api.CVVDP(cs, fps=24.0, model="standard_fhd", gpu_id=local, lib=lib) for _ in range(nthreads)]
        scores = [[] for _ in range(nthreads)]

        def worker(i, frames):
            h = handlers[i]
            for f in range(frames):
                a, b = host_pairs[(f + i) % len(host_pairs)]
                scores[i].append(h.compute(a, b, ls, ls))

        def run(frames):
            th = [threading.Thread(target=worker, args=(i, frames)) for i in range(nthreads)]
            for x in th:
                x.start()
            for x in th:
                x.join()

        run(CFRAMES * args.warmup)
        torch.cuda.synchronize()
        sampler = ClockSampler(local)
        sampler.start()
        t0 = time.perf_counter()
        run(CFRAMES * args.steps)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        clocks = sampler.stop()
        fps = nthreads * CFRAMES * args.steps / dt
        sweep[nthreads] = round(fps, 2)
        if best is None or fps > best[0]:
            best = (fps, nthreads, dt, clocks, scores[0][-1])
        ktimes = None
        if not reference and nthreads == args.cvvdp_threads[0]:
            h = handlers[0]
            h.kernel_timing(True)
            h.kernel_times(reset=True)
            for f in range(CFRAMES):
                a, b = host_pairs[f % len(host_pairs)]
                h.compute(a, b, ls, ls)
            kt = h.kernel_times(reset=True)
            h.kernel_timing(False)
            ktimes = {k: round(v[1] / CFRAMES, 4) for k, v in kt.items()}
            sweep["kernels_ms_per_frame"] = ktimes
            taps = h.geometry()[1]
        for h in handlers:
            h.close()
    for pb in pinned:
        pb.free()
    fps, nthreads, dt, clocks, last = best
    line = {"metric": CMETRIC, "value": round(fps, 2), "unit": "frames/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": CWORKLOAD, "frames_per_step_per_sequence": CFRAMES, "width": W, "height": H,
                       "display": "standard_fhd", "fps": 24.0, "sequences": nthreads, "threads_swept": sweep,
                       "timer": "wall clock, synchronised"},
            "e2e": {"value": round(fps, 2), "unit": "frames/s", "api": "Vship_ComputeCVVDP, pinned host frames",
                    "h2d_bytes_per_step": nthreads * CFRAMES * input_bytes(pairs[:1]),
                    "d2h_bytes_per_step": nthreads * CFRAMES * 8},
            "last_jod": round(last, 6), "clocks": clocks}
    if not reference and "kernels_ms_per_frame" in sweep:
        # Dominant HBM-bound kernel: the temporal filter reads the whole ring of both clips
        # (taps x 3 DKL planes) and writes 4 channel planes per clip.
        n = W * H
        algo = 2 * taps * 3 * n * 4 + 2 * 4 * n * 4
        ms = sweep["kernels_ms_per_frame"]["cvvdp_temporal"]
        peak, peak_kind = measured_peaks()
        ach = algo / (ms / 1e3) / 1e9
        line["roofline"] = {"bound": "hbm", "kernel": "cvvdp_temporal", "achieved": round(ach, 1), "peak": peak,
                            "peak_source": peak_kind, "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": None,
                            "algorithmic_bytes_per_launch": algo, "avg_launch_ms": ms, "ring_frames": taps}
    if reference:
        line["impl"] = "reference"
        line["cpu_baseline"] = {"value": round(fps, 2), "unit": "frames/s", "kind": "reference", "cores": nthreads,
                                "sample": "the reference has no CPU implementation: its own CUDA build on the B200"}
    print(json.dumps(line), flush=True)


def butter_e2e(args, pairs, cs, ls, local, lib=None):
    """Butteraugli end to end through Vship_ComputeButteraugli (distortion map returned) with
    pinned host frames: T host threads, each with its own handler, best of T in 1, 2, 4, 8.
    Returns (pairs/s, T, sweep)."""
    import threading
    import torch
    from vship_b200 import api
    pinned, host_pairs = pinned_frames(pairs, api, lib=lib)
    sweep, best = {}, None
    for nthreads in (1, 2, 4, 8):
        handlers = [api.Butteraugli(cs, qnorm=5, intensity=203.0, gpu_id=local, lib=lib) for _ in range(nthreads)]

        def worker(k, reps):
            for _ in range(reps):
                for i in range(k, len(host_pairs), nthreads):
                    handlers[k].compute(host_pairs[i][0], host_pairs[i][1], ls, ls, distmap=True)

        def run(reps):
            th = [threading.Thread(target=worker, args=(k, reps)) for k in range(nthreads)]
            for x in th:
                x.start()
            for x in th:
                x.join()

        run(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run(args.steps)
        dt = time.perf_counter() - t0
        v = len(host_pairs) * args.steps / dt
        sweep[nthreads] = round(v, 2)
        if best is None or v > best[0]:
            best = (v, nthreads)
        for h in handlers:
            h.close()
    for pb in pinned:
        pb.free()
    return best[0], best[1], sweep


def run_butteraugli_reference(args, rank, local):
    """Reference arm of the Butteraugli line: the reference library built from its own sources
    (oracle/_ref) on the same 4K pairs, end to end through its C API."""
    import torch
    from vship_b200 import abi, api, synth
    torch.cuda.set_device(local)
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libvship_ref.so")
    if not os.path.exists(ref_path):
        print(json.dumps({"impl": "reference", "unavailable": "reference library not built (oracle/build_ref.sh)"}))
        return
    L = api.load_library(ref_path)
    pairs = synth.make_pairs(BBATCH, BW, BH, fmt="rgb8", seed=77 + rank, unique=4, blur=(0.0, 1.5))
    cs = abi.srgb8(BW, BH)
    v, nthreads, sweep = butter_e2e(args, pairs, cs, pairs[0][2], local, lib=L)
    line = {"impl": "reference", "metric": BMETRIC, "value": round(v, 2), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": BWORKLOAD, "pairs_per_step": BBATCH, "width": BW, "height": BH,
                       "library": "Vship 4.1.0 built from its sources with nvcc for sm_100a (oracle/build_ref.sh)",
                       "api": "Vship_ComputeButteraugli with distortion map, pinned frames",
                       "threads_handlers": nthreads, "threads_swept": sweep},
            "e2e": {"value": round(v, 2), "unit": UNIT, "h2d_bytes_per_step": BBATCH * 2 * 3 * BW * BH,
                    "d2h_bytes_per_step": BBATCH * (BW * BH * 4 + 4)},
            "cpu_baseline": {"value": round(v, 2), "unit": UNIT, "kind": "reference", "cores": nthreads,
                             "sample": "the reference has no CPU implementation: its own CUDA build on the B200"}}
    print(json.dumps(line), flush=True)


UNEVEN_RES = [(640, 360), (1280, 720), (1920, 1080), (3840, 2160)]
UNEVEN_N = 256
UWORKLOAD = "ssimu2_uneven_256_srgb8_360p_720p_1080p_4k"
UMETRIC = "uneven-resolution SSIMU2 frame-pairs/s"


def xyb_floats(w, h):
    """Floats of the XYB planes some map reads, for a w x h image (Y at level 0; X, Y at
    levels 1-2; X, Y, B at levels 3-4)."""
    sizes = [(w, h)]
    for _ in range(5):
        pw, ph = sizes[-1]
        sizes.append(((pw - 1) // 2 + 1, (ph - 1) // 2 + 1))
    planes = [1, 2, 2, 3, 3, 0]
    return sum(n * sw * sh for n, (sw, sh) in zip(planes, sizes))


def make_uneven(seed):
    """256 pairs with resolutions drawn uniformly from UNEVEN_RES (seeded), 8-bit sRGB, content
    and DCT distortion as the headline workload; 8 distinct pairs per resolution are cycled."""
    from vship_b200 import synth
    rng = np.random.default_rng(seed)
    draw = rng.integers(0, len(UNEVEN_RES), UNEVEN_N)
    t = time.time()
    gen = {}
    for k, (w, h) in enumerate(UNEVEN_RES):
        gen[k] = synth.make_pairs(8, w, h, fmt="rgb8", seed=seed + 17 * k, unique=4, steps=(4.0, 48.0))
    pairs = []
    seen = {k: 0 for k in gen}
    for k in draw:
        p1, p2, ls = gen[int(k)][seen[int(k)] % 8]
        seen[int(k)] += 1
        pairs.append((UNEVEN_RES[int(k)], p1, p2, ls))
    log("generated %d uneven pairs in %.1fs (%s)" % (len(pairs), time.time() - t,
                                                     {"%dx%d" % UNEVEN_RES[k]: seen[k] for k in seen}))
    return pairs


def uneven_pinned(pairs, api, lib=None):
    """Each frame of the uneven workload in one pinned buffer (FFVship layout)."""
    pinned, host = [], []
    for (wh, p1, p2, ls) in pairs:
        frames = []
        for planes in (p1, p2):
            nbytes = sum(p.nbytes for p in planes)
            pb = api.PinnedBuffer(nbytes, lib=lib)
            off, ptrs = 0, []
            for p in planes:
                pb.array[off:off + p.nbytes] = p.reshape(-1)
                ptrs.append(pb.ptr.value + off)
                off += p.nbytes
            pinned.append(pb)
            frames.append(ptrs)
        host.append((wh, frames[0], frames[1], ls))
    return pinned, host


def run_uneven(args, world, rank, local):
    """Uneven batch: 256 pairs of mixed resolutions scored in one persistent launch replayed
    from a CUDA graph (VshipExt_ComputeSSIMU2BatchDevice), against per-frame launches and
    per-resolution batched launches of the per-handler path."""
    import torch
    from vship_b200 import abi, api
    torch.cuda.set_device(local)
    pairs = make_uneven(seed=4321 + rank)
    n = len(pairs)
    cs = {wh: abi.srgb8(*wh) for wh in UNEVEN_RES}
    dev = [(wh, [torch.from_numpy(p).cuda() for p in p1], [torch.from_numpy(p).cuda() for p in p2], ls)
           for wh, p1, p2, ls in pairs]
    items = [(cs[wh], cs[wh], [t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls) for wh, d1, d2, ls in dev]
    arr, keep = api.frame_pairs(items)
    scores = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    b = api.SSIMU2Batch(gpu_id=local)
    if args.tile_rows:
        b.set_tile_rows(args.tile_rows)

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def batch_step():
        b.compute_device_array(arr, n, scores.data_ptr(), 0, stream.cuda_stream)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ms = timed(batch_step, args.steps)
    clocks = sampler.stop()
    value = n * args.steps / (ms / 1e3)
    rows = b.tile_rows()
    batch_scores = scores.cpu().numpy().copy()
    # tile-height sweep (the autotuner's candidates), timed the same way
    sweep = {}
    for r in (16, 32, 64):
        b.set_tile_rows(r)
        sweep[r] = round(n * 3 / (timed(batch_step, 3) / 1e3), 1)
    b.set_tile_rows(args.tile_rows or 0)
    b.kernel_timing(True)
    b.kernel_times(reset=True)
    for _ in range(3):
        batch_step()
    torch.cuda.synchronize()
    kt = b.kernel_times(reset=True)
    b.kernel_timing(False)
    launches, total_ms = kt["ssimu2_batch"]
    avg_ms = total_ms / launches
    algo = sum(2 * (3 * w * h + 8 * xyb_floats(w, h)) for (w, h), _, _, _ in pairs)
    peak, peak_kind = measured_peaks()
    achieved = algo / (avg_ms / 1e3) / 1e9

    # per-frame launches: one handler per resolution, one pair per call
    handlers = {wh: api.SSIMU2(cs[wh], gpu_id=local) for wh in UNEVEN_RES}
    pf_scores = torch.zeros(n, dtype=torch.float64, device="cuda")
    pf_args = [(handlers[wh], [t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls) for wh, d1, d2, ls in dev]

    def per_frame_step():
        for i, (hh, a1, a2, ls) in enumerate(pf_args):
            hh.compute_device(1, a1, a2, ls, ls, pf_scores[i].data_ptr(), 0, stream.cuda_stream)

    pf_ms = timed(per_frame_step, max(1, args.steps // 2))
    per_frame = n * max(1, args.steps // 2) / (pf_ms / 1e3)
    max_diff = float(np.max(np.abs(pf_scores.cpu().numpy() - batch_scores)))

    # per-resolution batches: each handler scores all pairs of its resolution per call
    groups = {}
    for i, (wh, d1, d2, ls) in enumerate(dev):
        groups.setdefault(wh, []).append(i)
    grp_args = []
    for wh, idx in groups.items():
        a1 = [t.data_ptr() for i in idx for t in dev[i][1]]
        a2 = [t.data_ptr() for i in idx for t in dev[i][2]]
        out = torch.zeros(len(idx), dtype=torch.float64, device="cuda")
        grp_args.append((handlers[wh], len(idx), a1, a2, dev[idx[0]][3], out))

    def per_class_step():
        for hh, k, a1, a2, ls, out in grp_args:
            hh.compute_device(k, a1, a2, ls, ls, out.data_ptr(), 0, stream.cuda_stream)

    pc_ms = timed(per_class_step, max(1, args.steps // 2))
    per_class = n * max(1, args.steps // 2) / (pc_ms / 1e3)
    for hh in handlers.values():
        hh.close()

    # end to end: host API of the batch handler with each frame in one pinned buffer
    pinned, host = uneven_pinned(pairs, api)
    host_items = [(cs[wh], cs[wh], f1, f2, ls, ls) for wh, f1, f2, ls in host]
    harr, hkeep = api.frame_pairs(host_items)
    e2e_scores = np.zeros(n)
    import ctypes as _ct
    L = api.load()

    def e2e_step():
        rc = L.VshipExt_ComputeSSIMU2Batch(b.h, n, harr, e2e_scores.ctypes.data_as(_ct.POINTER(_ct.c_double)), None)
        if rc != 0:
            raise RuntimeError("VshipExt_ComputeSSIMU2Batch failed: %d" % rc)

    for _ in range(args.warmup):
        e2e_step()
    t0 = time.perf_counter()
    e2e_steps = max(1, args.steps // 2)
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    e2e_diff = float(np.max(np.abs(e2e_scores - batch_scores)))
    in_bytes = sum(p.nbytes for _, p1, p2, _ in pairs for p in p1 + p2)
    for pb in pinned:
        pb.free()
    b.close()

    cpu = None
    if not args.no_cpu_baseline:
        import oracle
        oracle.build()
        k, t0, maxd = 0, time.perf_counter(), 0.0
        while k < n and time.perf_counter() - t0 < args.cpu_seconds:
            wh, p1, p2, ls = pairs[k]
            q, d, _ = oracle.ssimu2(oracle.convert(p1, ls, cs[wh]), oracle.convert(p2, ls, cs[wh]))
            maxd = max(maxd, abs(batch_scores[k] - d))
            k += 1
        dt = time.perf_counter() - t0
        cpu = {"value": round(k / dt, 3), "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
               "sample": "first %d pairs of the uneven workload in FP64 (%.1f s)" % (k, dt),
               "max_abs_dscore_gpu_vs_fp64": maxd}
    line = {
        "metric": UMETRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": UWORKLOAD, "pairs_per_step": n, "resolutions": ["%dx%d" % r for r in UNEVEN_RES],
                   "format": "8-bit sRGB", "tile_rows": rows, "launch": "one persistent launch per step (CUDA graph)",
                   "l2": "inputs (%.0f MB per step) larger than L2" % (in_bytes / 1e6)},
        "per_frame_value": round(per_frame, 2), "per_class_value": round(per_class, 2),
        "tile_rows_sweep": sweep, "max_abs_score_diff_vs_per_frame": max_diff,
        "e2e": {"value": round(n * e2e_steps / e2e_s, 2), "unit": UNIT,
                "api": "VshipExt_ComputeSSIMU2Batch, each frame in one pinned buffer",
                "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": n * 8,
                "max_abs_score_diff_vs_device_path": e2e_diff},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "kernel": "ssimu2_batch", "achieved": round(achieved, 1), "peak": peak,
                     "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                     "algorithmic_bytes_per_launch": algo, "avg_launch_ms": round(avg_ms, 4),
                     "scope": "the whole graph launch (front, tile table, maps, final)"},
        "cpu_baseline": cpu, "clocks": clocks,
    }
    tr, src = traffic_of("ssimu2_batch")
    if tr:
        line["roofline"]["traffic"], line["roofline"]["traffic_source"] = tr, src
    print(json.dumps(line), flush=True)


def run_uneven_reference(args, world, rank, local):
    """Reference arm of the uneven workload: the reference library, one handler per resolution
    per host thread, one pair per call through Vship_ComputeSSIMU2 with pinned frames."""
    if rank != 0:
        return
    from vship_b200 import abi, api
    ref = os.path.join(ROOT, "oracle", "_ref", "libvship_ref.so")
    if not os.path.exists(ref):
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libvship_ref.so was not built"}))
        return
    import torch
    torch.cuda.set_device(local)
    L = api.load_library(ref)
    pairs = make_uneven(seed=4321)
    n = len(pairs)
    cs = {wh: abi.srgb8(*wh) for wh in UNEVEN_RES}
    pinned, host = uneven_pinned(pairs, api, lib=L)
    best = None
    for nthreads in args.ref_threads:
        handlers = [{wh: api.SSIMU2(cs[wh], gpu_id=local, lib=L) for wh in UNEVEN_RES} for _ in range(nthreads)]
        out = np.zeros(n)

        def worker(k):
            torch.cuda.set_device(local)
            for i in range(k, n, nthreads):
                wh, f1, f2, ls = host[i]
                out[i] = handlers[k][wh].compute(f1, f2, ls, ls)

        def step():
            ths = [threading.Thread(target=worker, args=(k,)) for k in range(nthreads)]
            for t in ths:
                t.start()
            for t in ths:
                t.join()

        for _ in range(args.warmup):
            step()
        t0 = time.perf_counter()
        steps = max(1, args.steps // 2)
        for _ in range(steps):
            step()
        dt = time.perf_counter() - t0
        v = n * steps / dt
        log("reference uneven: %d threads -> %.1f pairs/s" % (nthreads, v))
        if best is None or v > best[0]:
            best = (v, nthreads, dt / steps)
        for hs in handlers:
            for hh in hs.values():
                hh.close()
    for pb in pinned:
        pb.free()
    v, nthreads, dt = best
    print(json.dumps({
        "impl": "reference", "metric": UMETRIC, "value": round(v, 2), "unit": UNIT, "n_gpus": 1,
        "steps": max(1, args.steps // 2), "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": UWORKLOAD, "pairs_per_step": n, "threads_handlers": nthreads,
                   "api": "Vship_ComputeSSIMU2 per pair, one handler per resolution per thread"},
        "e2e": {"value": round(v, 2), "unit": UNIT,
                "h2d_bytes_per_step": sum(p.nbytes for _, a, b, _ in pairs for p in list(a) + list(b)),
                "d2h_bytes_per_step": n * 4 * 108},
        "cpu_baseline": {"value": round(v, 2), "unit": UNIT, "kind": "reference", "cores": nthreads,
                         "sample": "the reference's CUDA build on the B200 driven by %d host threads" % nthreads}}),
        flush=True)


SWORKLOAD = "surrogate_target_quality_train200k_512_eval1000_1080p_yuv420p10"
SMETRIC = "surrogate target-quality search: exact SSIMU2 calls saved"


def run_surrogate(args, world, rank, local):
    """Learned surrogate, end to end: a training set of seeded 512x512 10-bit 4:2:0 pairs (DCT
    steps uniform in [2, 64]) scored by the exact engine, training on the GPU with the
    library's own kernels, then bisection to SSIMULACRA2 = 80 over 1080p frames with the
    surrogate (exact fallback within +/-2) and without it."""
    import torch
    from vship_b200 import abi, api, target_quality as tq
    torch.cuda.set_device(local)
    out = {"metric": SMETRIC, "unit": "fraction of exact calls saved", "n_gpus": 1, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP16 weights)", "data": "synthetic"}
    cs512 = abi.yuv420_10bit_bt709(512, 512)
    sur = api.Surrogate(cs512)
    ex512 = api.SSIMU2(cs512)
    n, held = args.sur_train, 4096
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    X, T = tq.build_training_set(sur, ex512, n + held, 512, 512, seed=2024, chunk=1024)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    hist = sur.train(n, X.data_ptr(), T.data_ptr(), epochs=args.sur_epochs, batch=256, lr=3e-3, seed=11)
    t2 = time.perf_counter()
    pred = torch.zeros(held, dtype=torch.float32, device="cuda")
    sur.predict_inputs(held, X[n].data_ptr(), pred.data_ptr())
    torch.cuda.synchronize()
    tgt = T[n:].cpu().numpy()
    rmse512 = tq.rmse(pred.cpu().numpy(), tgt)
    model = sur.model()
    ex512.close()
    sur.close()
    del X, T
    torch.cuda.empty_cache()
    log("training set %d pairs in %.1fs, training %d epochs in %.1fs, held-out RMSE %.3f (std %.2f)"
        % (n + held, t1 - t0, args.sur_epochs, t2 - t1, rmse512, tgt.std()))

    # Bisection over 1080p frames.
    w, h, frames = 1920, 1080, args.sur_frames
    cs = abi.yuv420_10bit_bt709(w, h)
    sur = api.Surrogate(cs)
    sur.set_model(model)
    ex = api.SSIMU2(cs)
    gen = tq.GpuFrames()
    refs = torch.empty((frames, 3, h, w), dtype=torch.uint8, device="cuda")
    for i0 in range(0, frames, 32):
        i1 = min(frames, i0 + 32)
        refs[i0:i1] = gen.references(i1 - i0, w, h, seed=500 + i0).round().to(torch.uint8)
    ref_yuv = [torch.empty((frames, h, w), dtype=torch.int16, device="cuda"),
               torch.empty((frames, h // 2, w // 2), dtype=torch.int16, device="cuda"),
               torch.empty((frames, h // 2, w // 2), dtype=torch.int16, device="cuda")]
    for i0 in range(0, frames, 32):
        i1 = min(frames, i0 + 32)
        for dst, src in zip(ref_yuv, gen.yuv420p10(refs[i0:i1].float())):
            dst[i0:i1] = src

    def fy(i0, i1):
        return tuple(x[i0:i1] for x in ref_yuv)

    def dy(i0, i1, st):
        return gen.yuv420p10(gen.dct_quantize(refs[i0:i1].float(), st))

    torch.cuda.synchronize()
    t3 = time.perf_counter()
    base = tq.search(fy, dy, frames, ex, None)
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    guided = tq.search(fy, dy, frames, ex, sur)
    torch.cuda.synchronize()
    t5 = time.perf_counter()
    fa = tq.final_scores(fy, dy, frames, ex, base["step"])
    fb = tq.final_scores(fy, dy, frames, ex, guided["step"])

    # Cost of one prediction against one exact score (device-resident 1080p pairs, 64 per call).
    yb = dy(0, 64, np.full(64, 20.0))
    p1, ls = tq.planes_of(fy(0, 64))
    p2, _ = tq.planes_of(yb)
    pr = torch.zeros(64, dtype=torch.float32, device="cuda")
    sc = torch.zeros(64, dtype=torch.float64, device="cuda")

    def rate(fn, reps=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return 64 * reps / (e0.elapsed_time(e1) / 1e3)

    refs64 = torch.zeros((64, sur.reference_floats()), dtype=torch.float32, device="cuda")
    sur.references(64, p1, ls, refs64.data_ptr())
    sur_rate = rate(lambda: sur.predict(64, p1, p2, ls, ls, pr.data_ptr()))
    against_rate = rate(lambda: sur.predict_against(64, refs64.data_ptr(), p2, ls, pr.data_ptr()))
    ex_rate = rate(lambda: ex.compute_device(64, p1, p2, ls, ls, sc.data_ptr(), 0, 0))
    sur.close()
    ex.close()
    saved = 1.0 - guided["exact_calls"] / base["exact_calls"]
    errs = np.array(guided["surrogate_errors"])
    out.update({
        "value": round(saved, 4), "steps": 1, "warmup": 0,
        "config": {"workload": SWORKLOAD, "train_pairs": n, "train_size": "512x512", "held_out": held,
                   "eval_frames": frames, "eval_size": "1920x1080", "format": "YUV420 10-bit limited BT.709",
                   "target": 80.0, "margin": 2.0, "bisection": "7 halvings of step in [2, 64]",
                   "epochs": args.sur_epochs, "batch": 256},
        "exact_calls": {"with_surrogate": guided["exact_calls"], "without": base["exact_calls"],
                        "probes": guided["probes"]},
        "final_abs_error": {"with_surrogate": round(float(np.mean(np.abs(fb - 80))), 4),
                            "without": round(float(np.mean(np.abs(fa - 80))), 4),
                            "max_with_surrogate": round(float(np.max(np.abs(fb - 80))), 4)},
        "same_decision_fraction": round(float(np.mean(np.abs(base["step"] - guided["step"]) < 1e-9)), 4),
        "mean_abs_step_difference": round(float(np.mean(np.abs(base["step"] - guided["step"]))), 4),
        "surrogate_rmse": {"held_out_512": round(rmse512, 4), "held_out_std": round(float(tgt.std()), 3),
                           "near_threshold_1080p_mae": round(float(errs.mean()), 4) if len(errs) else None},
        "training": {"set_seconds": round(t1 - t0, 2), "train_seconds": round(t2 - t1, 2),
                     "samples_per_second": round(n * args.sur_epochs / (t2 - t1), 1),
                     "loss_per_epoch": [round(float(x), 5) for x in hist]},
        "search_seconds": {"without": round(t4 - t3, 2), "with_surrogate": round(t5 - t4, 2)},
        "pairs_per_second_1080p": {"surrogate_pair": round(sur_rate, 1),
                                   "surrogate_against_prepared_reference": round(against_rate, 1),
                                   "exact": round(ex_rate, 1)},
        "search_gpu_ms_estimate": {
            "without": round(base["exact_calls"] / ex_rate * 1e3, 1),
            "with_surrogate": round((guided["probes"] / against_rate + guided["exact_calls"] / ex_rate
                                     + frames / (2 * against_rate)) * 1e3, 1)},
    })
    print(json.dumps(out), flush=True)


def run_profile_case(args):
    """Small device-resident run for ncu captures: `--profile-pairs` 1080p pairs, `--steps`
    calls of VshipExt_ComputeSSIMU2Device, nothing else (no timing, no e2e, no CPU leg)."""
    import torch
    from vship_b200 import abi, api, synth
    n = args.profile_pairs
    pairs = synth.make_pairs(n, W, H, fmt="yuv420p10", seed=5, unique=2)
    cs = abi.yuv420_10bit_bt709(W, H)
    ls = pairs[0][2]
    dev = [([torch.from_numpy(p.view(np.uint8)).cuda() for p in a], [torch.from_numpy(p.view(np.uint8)).cuda() for p in b])
           for a, b, _ in pairs]
    ptr1 = [t.data_ptr() for d in dev for t in d[0]]
    ptr2 = [t.data_ptr() for d in dev for t in d[1]]
    scores = torch.zeros(n, dtype=torch.float64, device="cuda")
    h = api.SSIMU2(cs)
    for _ in range(args.steps):
        h.compute_device(n, ptr1, ptr2, ls, ls, scores.data_ptr(), 0, 0)
    torch.cuda.synchronize()
    h.close()
    log("profile case: %d pairs x %d calls, scores %s" % (n, args.steps, np.round(scores.cpu().numpy()[:4], 4)))


def run_profile_uneven(args):
    """Small uneven case for ncu captures: `--profile-uneven` pairs drawn like the uneven
    workload, scored `--steps` times by the batch graph (32-row tiles), then once per
    resolution by the per-handler path.  No timing."""
    import torch
    from vship_b200 import abi, api, synth
    rng = np.random.default_rng(4321)
    draw = rng.integers(0, len(UNEVEN_RES), args.profile_uneven)
    gen = {k: synth.make_pairs(2, w, h, fmt="rgb8", seed=5 + k, unique=1) for k, (w, h) in enumerate(UNEVEN_RES)}
    dev = []
    for i, k in enumerate(draw):
        p1, p2, ls = gen[int(k)][i % 2]
        dev.append((UNEVEN_RES[int(k)], [torch.from_numpy(p).cuda() for p in p1], [torch.from_numpy(p).cuda() for p in p2], ls))
    cs = {wh: abi.srgb8(*wh) for wh in UNEVEN_RES}
    items = [(cs[wh], cs[wh], [t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls) for wh, d1, d2, ls in dev]
    n = len(items)
    scores = torch.zeros(n, dtype=torch.float64, device="cuda")
    with api.SSIMU2Batch() as b:
        b.set_tile_rows(32)
        for _ in range(args.steps):
            b.compute_device(items, scores.data_ptr())
        torch.cuda.synchronize()
    batch = scores.cpu().numpy().copy()
    groups = {}
    for i, (wh, d1, d2, ls) in enumerate(dev):
        groups.setdefault(wh, []).append(i)
    for wh, idx in groups.items():
        with api.SSIMU2(cs[wh]) as h:
            out = torch.zeros(len(idx), dtype=torch.float64, device="cuda")
            h.compute_device(len(idx), [t.data_ptr() for i in idx for t in dev[i][1]],
                             [t.data_ptr() for i in idx for t in dev[i][2]], dev[idx[0]][3], dev[idx[0]][3],
                             out.data_ptr(), 0, 0)
            torch.cuda.synchronize()
            scores[idx] = out
    log("profile uneven: %d pairs, max |batch - per-class| = %.3g" %
        (n, float(np.max(np.abs(scores.cpu().numpy() - batch)))))


def run_profile_butter(args):
    """Small device-resident Butteraugli run for ncu captures: `--profile-butter` 4K 8-bit sRGB
    pairs (intensity 203, Q-norm 5, distortion map on), `--steps` calls each, nothing else."""
    import torch
    from vship_b200 import abi, api, synth
    n = args.profile_butter
    pairs = synth.make_pairs(n, BW, BH, fmt="rgb8", seed=77, unique=1, blur=(0.0, 1.5))
    cs = abi.srgb8(BW, BH)
    ls = pairs[0][2]
    dev = [([torch.from_numpy(p).cuda() for p in a], [torch.from_numpy(p).cuda() for p in b]) for a, b, _ in pairs]
    norms = torch.zeros(n, 3, dtype=torch.float64, device="cuda")
    dmap = torch.zeros(BH, BW, dtype=torch.float32, device="cuda")
    with api.Butteraugli(cs, qnorm=5, intensity=203.0) as h:
        for _ in range(args.steps):
            for i, (d1, d2) in enumerate(dev):
                h.compute_device([x.data_ptr() for x in d1], [x.data_ptr() for x in d2], ls, ls,
                                 norms[i].data_ptr(), dmap.data_ptr(), BW * 4, 0)
        torch.cuda.synchronize()
    log("profile butteraugli: %d pairs x %d calls, norms %s" % (n, args.steps, np.round(norms.cpu().numpy()[0], 4)))


def run_profile_cvvdp(args):
    """Only N 1080p frame pairs through one CVVDP handler (for ncu captures)."""
    from vship_b200 import abi, api, synth
    pairs = synth.make_pairs(4, W, H, fmt="yuv420p10", seed=91, unique=4, steps=(4.0, 48.0))
    cs = abi.yuv420_10bit_bt709(W, H)
    pinned, host_pairs = pinned_frames(pairs, api)
    ls = pairs[0][2]
    h = api.CVVDP(cs, fps=24.0, model="standard_fhd")
    for f in range(args.profile_cvvdp):
        a, b = host_pairs[f % len(host_pairs)]
        score = h.compute(a, b, ls, ls)
    h.close()
    for pb in pinned:
        pb.free()
    log("profile cvvdp: %d frames, last JOD %.6f" % (args.profile_cvvdp, score))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-threads", type=int, default=4)
    ap.add_argument("--ref-threads", type=int, nargs="+", default=[1, 3, 4, 8])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cvvdp-threads", type=int, nargs="+", default=[1, 2, 4],
                    help="cvvdp: concurrent sequences (handlers) swept")
    ap.add_argument("--metric", default="ssimu2",
                    choices=["ssimu2", "ssimu2-single", "butteraugli", "ssimu2-uneven", "surrogate", "cvvdp"],
                    help="ssimu2-single: one 1080p 8-bit sRGB pair per call (latency and throughput); "
                         "butteraugli: secondary 4K Butteraugli line; ssimu2-uneven: 256 pairs of mixed "
                         "resolutions in one persistent launch, instead of the headline metric")
    ap.add_argument("--tile-rows", type=int, default=0, help="ssimu2-uneven: fixed map tile rows (0: autotune)")
    ap.add_argument("--sur-train", type=int, default=200000, help="surrogate: training pairs")
    ap.add_argument("--sur-epochs", type=int, default=8, help="surrogate: training epochs")
    ap.add_argument("--sur-frames", type=int, default=1000, help="surrogate: 1080p frames searched")
    ap.add_argument("--profile-pairs", type=int, default=0,
                    help="only run N device-resident pairs --steps times (for ncu captures)")
    ap.add_argument("--profile-butter", type=int, default=0,
                    help="only run N 4K Butteraugli pairs --steps times (for ncu captures)")
    ap.add_argument("--profile-uneven", type=int, default=0,
                    help="only run N uneven pairs through the batch graph --steps times and once per "
                         "resolution through handlers (for ncu captures)")
    ap.add_argument("--profile-cvvdp", type=int, default=0,
                    help="only run N 1080p frames through one CVVDP handler (for ncu captures)")
    args = ap.parse_args()
    if args.profile_cvvdp:
        run_profile_cvvdp(args)
        return
    if args.profile_pairs:
        run_profile_case(args)
        return
    if args.profile_uneven:
        run_profile_uneven(args)
        return
    if args.profile_butter:
        run_profile_butter(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_env()
    if args.metric == "butteraugli":
        if rank == 0:
            if args.impl == "ours":
                run_butteraugli(args, world, rank, local)
            else:
                run_butteraugli_reference(args, rank, local)
        return
    if args.metric == "cvvdp":
        if rank == 0:
            run_cvvdp(args, rank, local, reference=args.impl == "reference")
        return
    if args.metric == "ssimu2-single":
        if rank == 0:
            run_single(args, rank, local, reference=args.impl == "reference")
        return
    if args.metric == "surrogate":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no surrogate or "
                                  "target-quality search; its exact metric is measured by the other metrics"}))
        elif rank == 0:
            run_surrogate(args, world, rank, local)
        return
    if args.metric == "ssimu2-uneven":
        if args.impl == "reference":
            run_uneven_reference(args, world, rank, local)
        elif rank == 0:
            run_uneven(args, world, rank, local)
        return
    if args.impl == "reference":
        run_reference(args, world, rank, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
