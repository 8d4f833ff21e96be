"""The multi-GPU path is replicas only: each rank advances its own channel, the ranks meet only
at the barrier and the timing reduction.  This runs that host logic on CPU with two gloo ranks,
each stepping an oracle replica of the same seeded channel."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import time

    import torch.distributed as dist
    from datetime import timedelta

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    os.environ["OMP_NUM_THREADS"] = "1"
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from oracle import pyoracle
        from polymer_dns_b200 import replicas
        from tests import kmm_cases as kc
        p = kc.cfg_small(16, 16, 12)
        o = pyoracle.Oracle(p)
        kc.load_initial(o, p, kc.initial_fields(p, amp=0.05, seed=0))
        assert o.initial() == 0
        dist.barrier()
        t0 = time.perf_counter()
        steps = 2
        for _ in range(steps):
            assert o.step() == 0
        local_ms = (time.perf_counter() - t0) * 1e3 + 50.0 * rank   # rank 1 made slower on purpose
        dist.barrier()
        ms, value = replicas.job_throughput(dist, local_ms, steps, world, "cpu")
        sums = replicas.checksum_all(dist, float(np.abs(o.get("V")).sum()), world, "cpu")
        out.put((rank, local_ms, ms, value, sums))
    finally:
        dist.destroy_process_group()


def test_replicas_two_gloo_ranks(oracle_mod):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    (r0, l0, m0, v0, s0), (r1, l1, m1, v1, s1) = res
    assert m0 == m1 == pytest.approx(max(l0, l1))          # the job time is the slowest rank's
    assert v0 == pytest.approx(2 * 2 / (max(l0, l1) / 1e3))  # every rank's steps count
    assert s0 == s1 and s0[0] == s0[1]                     # identical replicas, no exchange


def test_autotune_candidates_follow_the_configuration():
    """The tuner times only the variants that apply: TMA z tiles, blocked columns and graph replay
    on the fused step; the tensor-core y transforms on the mixed routine path; nothing else."""
    from polymer_dns_b200 import abi, autotune
    fused = abi.default_params(nx=64, ny=64, nz=64)
    c = autotune.candidates(fused)
    assert len(c) == 8 and {abi.OPT_ZTMA, abi.OPT_COLUMN_BLOCKED, abi.OPT_GRAPH} == set(c[0])
    assert len(autotune.candidates(abi.default_params(nx=64, ny=64, nz=64, precision=1))) == 4
    assert autotune.candidates(abi.default_params(nx=64, ny=64, nz=64, polymer_on=1)) == [{}]
    mixed_poly = autotune.candidates(abi.default_params(nx=64, ny=64, nz=64, polymer_on=1, precision=1))
    assert mixed_poly == [{abi.OPT_TC_DCT: 0}, {abi.OPT_TC_DCT: 1}]
    assert autotune.shape_key(fused) != autotune.shape_key(abi.default_params(nx=64, ny=64, nz=96))
    assert autotune.describe({abi.OPT_ZTMA: 1, abi.OPT_GRAPH: 0}) == "ztma=1,graph=0" or \
        autotune.describe({abi.OPT_ZTMA: 1, abi.OPT_GRAPH: 0}) == "graph=0,ztma=1"
