"""Multi-process plumbing on the CPU (gloo, world size 2, 127.0.0.1): the
ensemble's variants dealt to ranks, the max-over-ranks timing reduction and
the host-side gather the bench uses for N GPUs."""
import os
import socket

import numpy as np
import pytest


def test_lpt_assignment_is_a_balanced_partition():
    from hrdayapy_b200.sharding import lpt_assign
    sizes = [2210680, 2991686, 995887, 3008430, 2971943, 1576466, 1637594, 926419,
             2571145, 2024087, 1850409, 1899688, 1663052, 2048364, 1993857, 2173101]
    for n in (1, 2, 3, 4, 8):
        parts = lpt_assign(sizes, n)
        flat = sorted(v for p in parts for v in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[v] for v in p) for p in parts]
        # LPT bound: max load <= mean load + largest item
        assert max(loads) <= np.mean(loads) + max(sizes)
    assert lpt_assign([5, 1], 4)[2:] == [[], []]
    with pytest.raises(ValueError):
        lpt_assign([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from hrdayapy_b200.sharding import gather_to_all, lpt_assign, max_over_ranks
        parts = lpt_assign([3, 9, 4, 1, 7], world)
        mine = parts[rank]
        t = max_over_ranks(10.0 + rank)
        got = gather_to_all({"rank": rank, "variants": mine})
        dist.barrier()
        out.put((rank, t, got))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, got in res:
        assert t == 11.0                                   # max over ranks
        assert [g["rank"] for g in got] == [0, 1]
        assert sorted(v for g in got for v in g["variants"]) == [0, 1, 2, 3, 4]


def _variant_runs(indices):
    """FP64 oracle runs (3 ms) of small heart variants of uneven size, each
    with its own geometry, longitudinal conductivity and g_Ks / g_Kr."""
    from oracle import mono as orc
    from tests import cases
    out = []
    for v in indices:
        shape = (20 + 2 * v, 18 + v, 14 + v)
        args, fibre, kw = cases.ragged_aniso_case(seed=30 + v, shape=shape, T=3.0)
        kw = dict(kw, sigma_l=0.25 + 0.03 * v)
        nodes, el, act, S, phi = args
        r = orc.run(nodes, el, act, S, phi, fibre_dir=fibre, anisotropic=True, vm_save_dt=1.0,
                    gks_scale=0.7 + 0.2 * v, gkr_scale=1.3 - 0.2 * v, **kw)
        out.append(r["Vm"][-1])
    return out


def _shard_worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["ORACLE_THREADS"] = "2"
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from hrdayapy_b200.sharding import shard_run_gather
        sizes = [(20 + 2 * v) * (18 + v) * (14 + v) for v in range(4)]
        res = shard_run_gather(sizes, _variant_runs)
        dist.barrier()
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_sharded_variants_equal_the_single_rank_run():
    """Four variants dealt to two ranks (LPT), each rank running its share,
    gathered in variant order on both ranks: every variant's result equals
    that of one process running all four."""
    import torch.multiprocessing as mp
    from hrdayapy_b200.sharding import shard_run_gather
    ref = shard_run_gather([1, 1, 1, 1], _variant_runs)      # no process group: all here
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got in res:
        assert len(got) == 4
        for v in range(4):
            np.testing.assert_array_equal(got[v], ref[v])
