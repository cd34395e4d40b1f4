"""Slab split of one heart over ranks (hrdayapy_b200.slab), host side: the
partition, the local problems' renumbering and the ghost exchange over two
gloo ranks.  The GPU run against the single-device run is in
tests/test_slab_gpu.py."""
import os
import socket

import numpy as np
import pytest

from tests import cases


def _prob(brick=(4, 4, 8), T=2.0):
    from hrdayapy_b200 import monodomain as M
    args, fibre, kw = cases.ragged_aniso_case(T=T)
    nodes, el, act, S, phi = args
    prob, _ = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=True,
                        vm_save_dt=kw["dt"], brick=brick, **dict(kw, A_P=2.0 / kw["R_P"]))
    return prob


def _neighbour_slot(lay, slots, off):
    """Slot of the voxel at offset off from each slot (-1 where the brick is absent)."""
    bi, bj, bk = lay.brick
    bv = bi * bj * bk
    slots = np.asarray(slots, np.int64)
    b, q = slots // bv, slots % bv
    li, lj, lk = q // (bj * bk), (q // bk) % bj, q % bk
    c = np.stack([li + off[0], lj + off[1], lk + off[2]])
    ext = np.array([bi, bj, bk])[:, None]
    d = np.where(c < 0, -1, np.where(c >= ext, 1, 0))
    c = c - d * ext
    nb = np.asarray(lay.brick_nbr, np.int64)[b, (d[0] + 1) * 9 + (d[1] + 1) * 3 + (d[2] + 1)]
    return np.where(nb >= 0, nb * bv + (c[0] * bj + c[1]) * bk + c[2], -1)


@pytest.mark.parametrize("world", [2, 3])
def test_plan_and_local_problems(world):
    from hrdayapy_b200.layout import TAG_PMJ, TAG_SURF
    from hrdayapy_b200.slab import local_problem, plan_slabs
    prob = _prob()
    lay = prob.layout
    bv = lay.bv
    plan = plan_slabs(prob, world)
    assert plan.cuts[0] == 0 and plan.cuts[-1] == lay.n_bricks and np.all(np.diff(plan.cuts) > 0)
    tag = np.asarray(prob.tag, np.uint32)
    pmj_bricks = np.unique(np.where(tag & TAG_PMJ)[0] // bv)
    seen = np.zeros(prob.n_myo, int)
    offs = [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)
            if 0 < abs(a) + abs(b) + abs(c) <= 2]
    for r in range(world):
        loc, owned, gl = local_problem(prob, plan, r)
        seen[owned] += 1
        assert set(pmj_bricks) <= set(plan.local_bricks(r))
        # every owned node sits at the same voxel, with the same tag
        g_sl = np.asarray(lay.slot_of_node, np.int64)[owned]
        l_sl = np.asarray(loc.layout.slot_of_node, np.int64)[:len(owned)]
        assert np.array_equal(np.asarray(loc.tag)[l_sl], tag[g_sl])
        assert np.array_equal(loc.layout.vox_idx[:len(owned)], lay.vox_idx[owned])
        # every tissue slot of the local problem is a node (owned, then ghosts)
        all_sl = np.asarray(loc.layout.slot_of_node, np.int64)
        tissue = np.where(np.asarray(loc.tag) & 0x3)[0]
        assert np.array_equal(np.sort(all_sl), tissue)
        # neighbours through the local brick table are the global neighbours
        l2g = (plan.local_bricks(r)[:, None] * bv + np.arange(bv)).ravel()
        for off in offs:
            gn = _neighbour_slot(lay, g_sl, off)
            ln = _neighbour_slot(loc.layout, l_sl, off)
            ok = gn >= 0
            assert np.all(ln[ok] >= 0)
            assert np.array_equal(l2g[ln[ok]], gn[ok])
        # Purkinje edges point at the same voxels
        gi = np.asarray(prob.pk_idx, np.int64)
        li = np.asarray(loc.pk_idx, np.int64)
        m = gi < 0
        assert np.array_equal(gi[~m], li[~m])
        assert np.array_equal(l2g[-li[m] - 1], -gi[m] - 1)
        # ghosts report nothing
        ghost = ~np.isin(plan.local_bricks(r), plan.owned(r)).repeat(bv)
        assert not (np.asarray(loc.tag)[ghost] & TAG_SURF).any()
        assert (np.asarray(loc.surf_of_slot)[ghost] == -1).all()
    assert np.all(seen == 1)


def test_single_rank_plan_is_the_whole_problem():
    from hrdayapy_b200.slab import local_problem, plan_slabs
    prob = _prob()
    plan = plan_slabs(prob, 1)
    loc, owned, gl = local_problem(prob, plan, 0)
    assert len(plan.export) == 0 and np.array_equal(owned, np.arange(prob.n_myo))
    assert loc.n_myo == prob.n_myo
    assert np.array_equal(np.asarray(loc.tag), np.asarray(prob.tag))
    assert np.array_equal(np.asarray(loc.layout.brick_nbr), np.asarray(prob.layout.brick_nbr))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from hrdayapy_b200.slab import SlabExchange, local_problem, plan_slabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        prob = _prob()
        bv = prob.layout.bv
        plan = plan_slabs(prob, world)
        loc, owned, gl = local_problem(prob, plan, rank)
        ex = SlabExchange(plan, rank, gl, bv)
        rng = np.random.default_rng(1)
        Wg = rng.standard_normal(prob.layout.n_slots).astype(np.float32)
        l2g = (plan.local_bricks(rank)[:, None] * bv + np.arange(bv)).ravel()
        own_slot = np.isin(plan.local_bricks(rank), plan.owned(rank)).repeat(bv)
        W = np.where(own_slot, Wg[l2g], np.float32(-999.0))     # ghosts stale
        send = np.zeros(ex.width, np.float32)
        send[:len(ex.send_slots)] = W[ex.send_slots]
        parts = [torch.empty(ex.width) for _ in range(world)]
        dist.all_gather(parts, torch.from_numpy(send))
        out = torch.cat(parts).numpy()
        W[ex.recv_slots] = out[ex.recv_pos]
        q.put((rank, bool(np.array_equal(W, Wg[l2g]))))
    finally:
        dist.destroy_process_group()


def test_ghost_exchange_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_exchange_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=180) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    assert sorted(res) == [(0, True), (1, True)]
