"""One heart split into slabs over ranks (hrdayapy_b200.slab) against the
same heart on one device: the assembled Vm snapshots and activation /
deactivation events agree bit for bit.  The ranks are processes on the one
GPU of the test machine, exchanging the ghosts through host memory (gloo):
no kernel waits on another rank, so they may share a device."""
import os

import numpy as np
import pytest

from tests import cases
from tests.test_slab import _free_port

pytestmark = pytest.mark.gpu
T_MS = 6.0


def _prob():
    from hrdayapy_b200 import monodomain as M
    args, fibre, kw = cases.ragged_aniso_case(T=T_MS)
    nodes, el, act, S, phi = args
    prob, _ = M.prepare(nodes, el, act, S, S, phi, fibre_dir=fibre, anisotropic=True,
                        vm_save_dt=0.1, act_threshold=-20.0, deact_threshold=-20.0,
                        **dict(kw, A_P=2.0 / kw["R_P"]))
    return prob


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    from hrdayapy_b200.slab import SlabRun
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        prob = _prob()
        run = SlabRun(prob)
        run.run(prob.n_steps)
        vm = run.vm_frames()
        ev = run.events()
        run.close()
        if rank == 0:
            q.put((vm, ev[0], ev[1], ev[2], ev[3]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_split_equals_single_device(world):
    import multiprocessing as mp
    from hrdayapy_b200 import monodomain as M
    prob = _prob()
    sim = M.MonoHandle(prob)
    sim.run(prob.n_steps, graph_chunk=50)
    vm_ref = sim.vm_frames()
    ev_ref = sim.events()
    sim.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    import queue
    import time
    res, t0 = None, time.time()
    while res is None:
        try:
            res = q.get(timeout=2)
        except queue.Empty:
            # a worker that died fails the test at once
            if any(p.exitcode not in (None, 0) for p in ps) or time.time() - t0 > 300:
                for p in ps:
                    if p.is_alive():
                        p.terminate()
                pytest.fail(f"slab workers: exit codes {[p.exitcode for p in ps]}")
    vm, a, na, d, nd = res
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    np.testing.assert_array_equal(vm, vm_ref)
    np.testing.assert_array_equal(a, ev_ref[0])
    np.testing.assert_array_equal(na, ev_ref[1])
    np.testing.assert_array_equal(d, ev_ref[2])
    np.testing.assert_array_equal(nd, ev_ref[3])
    assert (na > 0).any()          # the wave reached voxels on every slab
