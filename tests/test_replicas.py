"""Replica sharding across ranks, run as two gloo processes on the CPU (the multi-GPU path
has no device-side exchange, so the host logic is all there is to test)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_q):
    import torch.distributed as dist
    from vship_b200 import abi, replicas, synth
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    pairs = synth.make_pairs(5, 48, 32, fmt="rgb8", seed=3, unique=2)
    cs = abi.srgb8(48, 32)

    def score(pr):
        p1, p2, ls = pr
        return oracle.ssimu2(oracle.convert(p1, ls, cs), oracle.convert(p2, ls, cs))[1]

    scores = replicas.score_pairs(pairs, score, rank, world)
    t = replicas.max_over_ranks(1.0 + rank, world)
    out_q.put((rank, scores.tolist(), t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_match_single_process():
    import oracle
    from vship_b200 import abi, replicas, synth
    oracle.build()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0, p.exitcode
    pairs = synth.make_pairs(5, 48, 32, fmt="rgb8", seed=3, unique=2)
    cs = abi.srgb8(48, 32)
    want = [oracle.ssimu2(oracle.convert(a, ls, cs), oracle.convert(b, ls, cs))[1] for a, b, ls in pairs]
    # The oracle's OpenMP reductions combine per-thread partial sums in an unspecified order,
    # so two runs agree to rounding, not bit for bit.
    for rank, scores, t in res:
        np.testing.assert_allclose(np.array(scores), np.array(want), rtol=1e-12, atol=0)
        assert t == 2.0
    assert replicas.shard(5, 0, 2) == [0, 2, 4] and replicas.shard(5, 1, 2) == [1, 3]
