"""Replicas on the GPU: one process per rank scores its shard of the pairs with the engine on
the device its gpu_id names (Vship_SSIMU2Init2's device argument), and the gathered scores
equal one process's bit for bit.  With one GPU both ranks share it: replicas are independent
processes whose kernels never wait on each other, so sharing a device is only slower.  Also
the device argument's error path: an id out of range is rejected."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from vship_b200 import abi, api, synth

pytestmark = pytest.mark.gpu

N, W, H = 6, 320, 180


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_q):
    import datetime
    import torch
    import torch.distributed as dist
    from vship_b200 import abi, api, replicas, synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    gpu = rank % torch.cuda.device_count()
    pairs = synth.make_pairs(N, W, H, fmt="yuv420p10", seed=5, unique=3)
    cs = abi.yuv420_10bit_bt709(W, H)
    with api.SSIMU2(cs, gpu_id=gpu) as h:
        scores = replicas.score_pairs(pairs, lambda pr: h.compute(pr[0], pr[1], pr[2]), rank, world)
    out_q.put((rank, gpu, scores.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replica_processes_match_one(gpu):
    pairs = synth.make_pairs(N, W, H, fmt="yuv420p10", seed=5, unique=3)
    cs = abi.yuv420_10bit_bt709(W, H)
    with api.SSIMU2(cs, gpu_id=0) as h:
        want = [h.compute(p1, p2, ls) for p1, p2, ls in pairs]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0, p.exitcode
    for rank, gpu_used, scores in res:
        assert scores == want, (rank, scores, want)


def test_device_argument_out_of_range_is_rejected(gpu):
    """As the reference: Init2 selects the device with a checked cudaSetDevice, so an id out of
    range fails with the CUDA error code (Vship_HIPError, src/VshipLib.cpp:209-216), and
    Vship_SetDevice rejects it with Vship_BadDeviceArgument (:176-186)."""
    import torch
    n = torch.cuda.device_count()
    cs = abi.srgb8(64, 48)
    L = api.load()
    for bad in (n, n + 3, -1):
        with pytest.raises(api.VshipError) as e:
            api.SSIMU2(cs, gpu_id=bad)
        assert e.value.code == abi.HIPError, (bad, e.value.code)
        with pytest.raises(api.VshipError) as e:
            api.Butteraugli(cs, gpu_id=bad)
        assert e.value.code == abi.HIPError, (bad, e.value.code)
        assert L.Vship_SetDevice(bad) == abi.BadDeviceArgument
    assert L.Vship_SetDevice(0) == abi.NoError
