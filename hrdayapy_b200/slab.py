"""One heart split over several GPUs in slabs of bricks (one process per GPU,
torch.distributed for the exchange).

The reference advances one heart on one device (simulation/functions/
purkinje_myocardium_pipeline.py:1347-1420); here its brick layout is cut
into contiguous ranges of bricks.  Bricks are numbered with i slowest, so
each range is a slab along i, and the ranges are balanced by tissue count.
Each rank runs an ordinary monodomain handle (hp_mono_*) on a local problem
made of:
  * its own bricks;
  * ghost copies of the bricks next to its slab (the one-voxel halo of the
    stencil lies inside them, bricks being at least one voxel thick);
  * ghost copies of every brick that holds a junction voxel.  The Purkinje
    tree is small (2 % of the work) and every rank advances all of it, so
    it needs every junction voxel's potential.
After each step the owners' post-ionic potentials W of the exported bricks
(the union of all ranks' ghosts) are all-gathered and written over the
ghosts.  The next step then reads exactly the values a single-device run
reads, so every owned voxel and every Purkinje node follows the single-device
run bit for bit.  The ghosts' own updates are discarded: their W is
overwritten, and their snapshots, surface frames and events are not
reported (slot_of_node lists owned nodes only, ghost slots carry no surface
flag).

The exchange is the only collective on the data path: one all-gather of
(exported bricks x brick volume) floats per step.  With NCCL it runs on the
device, on the handle's stream; with gloo (tests on the CPU side of one
GPU) it goes through host memory.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import numpy as np

from .layout import TAG_PMJ, TAG_SURF, BrickLayout

PHENO_MASK = 0x3


@dataclass
class SlabPlan:
    """Partition of one problem's bricks over `world` ranks (the same on
    every rank: computed from the problem alone)."""
    world: int
    cuts: np.ndarray              # (world + 1,) owned brick ranges [cuts[r], cuts[r + 1])
    ghosts: list                  # per rank: sorted global brick ids held as ghosts
    export: np.ndarray            # sorted global ids of every ghost brick (the exchange set)
    export_owner: np.ndarray      # owner rank of each exported brick

    def owned(self, r):
        return np.arange(self.cuts[r], self.cuts[r + 1], dtype=np.int64)

    def local_bricks(self, r):
        return np.union1d(self.owned(r), self.ghosts[r]).astype(np.int64)


def plan_slabs(prob, world: int) -> SlabPlan:
    """Contiguous brick ranges balanced by tissue voxels, their ghosts and
    the exchange set."""
    if world < 1:
        raise ValueError("world must be >= 1")
    lay = prob.layout
    nb, bv = lay.n_bricks, lay.bv
    if prob.theta != 0.0:
        raise ValueError("the slab split runs the explicit step (theta = 0)")
    if lay.shape is None:
        raise ValueError("the slab split needs a single-heart problem")
    tag = np.asarray(prob.tag, np.uint32).reshape(nb, bv)
    tissue = ((tag & PHENO_MASK) != 0).sum(1)
    if nb < world:
        raise ValueError(f"{nb} bricks cannot be split over {world} ranks")
    cum = np.concatenate([[0], np.cumsum(tissue)])
    cuts = [0]
    for r in range(1, world):
        c = int(np.searchsorted(cum, cum[-1] * r / world))
        cuts.append(min(max(c, cuts[-1] + 1), nb - (world - r)))
    cuts.append(nb)
    cuts = np.asarray(cuts, np.int64)
    pmj = np.where(((tag & TAG_PMJ) != 0).any(1))[0]
    nbr = np.asarray(lay.brick_nbr, np.int64)
    ghosts = []
    for r in range(world):
        own = np.arange(cuts[r], cuts[r + 1])
        n = nbr[own].ravel()
        n = n[(n >= 0) & ((n < cuts[r]) | (n >= cuts[r + 1]))]
        g = np.union1d(n, pmj)
        g = g[(g < cuts[r]) | (g >= cuts[r + 1])]
        ghosts.append(g.astype(np.int64))
    export = np.unique(np.concatenate(ghosts)) if world > 1 else np.zeros(0, np.int64)
    owner = np.searchsorted(cuts, export, side="right") - 1
    return SlabPlan(world=world, cuts=cuts, ghosts=ghosts, export=export.astype(np.int64),
                    export_owner=owner.astype(np.int64))


def local_problem(prob, plan: SlabPlan, rank: int):
    """Rank `rank`'s problem: its own and ghost bricks, renumbered in global
    order.  Returns (problem, owned_nodes, local_of_global_brick).  The
    problem's first len(owned_nodes) nodes are the owned voxels, whose
    global (reference-order) ids owned_nodes lists; its remaining nodes are
    the ghost voxels."""
    lay = prob.layout
    nb, bv = lay.n_bricks, lay.bv
    L = plan.local_bricks(rank)
    gl = np.full(nb, -1, np.int64)
    gl[L] = np.arange(len(L))
    own = np.zeros(nb, bool)
    own[plan.cuts[rank]:plan.cuts[rank + 1]] = True
    sl = (L[:, None] * bv + np.arange(bv)[None, :]).ravel()       # local slot -> global slot
    ghost_slot = ~own[L].repeat(bv)
    tag = np.asarray(prob.tag, np.uint32)[sl].copy()
    tag[ghost_slot] &= ~np.uint32(TAG_SURF)
    surf_of_slot = np.asarray(prob.surf_of_slot, np.int32)[sl].copy()
    surf_of_slot[ghost_slot] = -1
    ns_g = lay.n_slots

    def comp3(a):
        return np.asarray(a).reshape(3, ns_g)[:, sl].reshape(-1)

    def loc_slot(gs):
        gs = np.asarray(gs, np.int64)
        return gl[gs // bv] * bv + gs % bv

    nbr = np.asarray(lay.brick_nbr, np.int64)[L]
    nbr = np.where(nbr >= 0, gl[np.maximum(nbr, 0)], -1).astype(np.int32)
    sos = np.asarray(lay.slot_of_node, np.int64)
    node_brick = sos // bv
    owned_nodes = np.where(own[node_brick])[0]
    # every tissue slot of the local problem is a node: the owned nodes
    # first (the reported columns), then the ghost voxels (never reported)
    ghost_nodes = np.where(~own[node_brick] & (gl[node_brick] >= 0))[0]
    local_nodes = np.concatenate([owned_nodes, ghost_nodes])
    new_sos = loc_slot(sos[local_nodes]).astype(np.int32)
    idx = np.asarray(prob.pk_idx, np.int64).copy()
    myo = idx < 0
    if myo.any():
        ls = loc_slot(-idx[myo] - 1)
        if (gl[(-idx[myo] - 1) // bv] < 0).any():
            raise RuntimeError("local_problem: a junction voxel is not local")
        idx[myo] = -ls - 1
    new_lay = BrickLayout(shape=lay.shape, brick=lay.brick, vox_idx=lay.vox_idx[local_nodes],
                          n_bricks=len(L), brick_coords=np.asarray(lay.brick_coords)[L],
                          brick_nbr=nbr, slot_of_node=new_sos,
                          nbr_bits=np.asarray(lay.nbr_bits)[local_nodes])
    bvar = None if prob.brick_variant is None else np.asarray(prob.brick_variant)[L]
    p = dataclasses.replace(
        prob, layout=new_lay, tag=tag,
        wface=comp3(prob.wface) if prob.anisotropic else None,
        doff=comp3(prob.doff) if prob.anisotropic else None,
        pk_idx=idx.astype(np.int32), pmj_row=np.asarray(prob.pmj_row, np.int32)[sl],
        surf_of_slot=surf_of_slot, brick_variant=bvar)
    return p, owned_nodes, gl


class SlabExchange:
    """Index sets of one rank's exchange.  The gathered buffer holds, for
    every rank in order, its exported bricks (ascending) padded to the
    largest count, brick volume floats each."""

    def __init__(self, plan: SlabPlan, rank: int, gl: np.ndarray, bv: int):
        world = plan.world
        exp, own = plan.export, plan.export_owner
        counts = np.bincount(own, minlength=world) if len(exp) else np.zeros(world, np.int64)
        self.max_cnt = int(counts.max()) if len(counts) else 0
        self.width = self.max_cnt * bv             # floats per rank in the gathered buffer
        first = np.concatenate([[0], np.cumsum(counts)])
        k_in_owner = np.arange(len(exp)) - first[own] if len(exp) else np.zeros(0, np.int64)
        mine = exp[own == rank]
        lane = np.arange(bv, dtype=np.int64)
        self.send_slots = (gl[mine][:, None] * bv + lane).ravel().astype(np.int32)
        g = plan.ghosts[rank]
        e = np.searchsorted(exp, g)
        if len(g) and not np.array_equal(exp[e], g):
            raise RuntimeError("SlabExchange: a ghost brick is missing from the exchange set")
        self.recv_slots = (gl[g][:, None] * bv + lane).ravel().astype(np.int32)
        self.recv_pos = ((own[e] * self.width + k_in_owner[e] * bv)[:, None] + lane).ravel()
        self.recv_pos = self.recv_pos.astype(np.int64)


class SlabRun:
    """One heart over the ranks of the default process group, one GPU each
    (the caller sets the device).  run(n) advances n steps with an exchange
    after each; vm_frames() / events() assemble the owned parts in the
    reference's node order on every rank."""

    def __init__(self, prob):
        import ctypes as C

        import torch
        import torch.distributed as dist

        from . import _lib
        from .monodomain import MonoHandle
        self._C = C
        self.rank = dist.get_rank() if dist.is_initialized() else 0
        self.world = dist.get_world_size() if dist.is_initialized() else 1
        self.prob = prob
        self.plan = plan_slabs(prob, self.world)
        local, self.owned_nodes, gl = local_problem(prob, self.plan, self.rank)
        self.local = local
        self.sim = MonoHandle(local)
        bv = prob.layout.bv
        self.ex = SlabExchange(self.plan, self.rank, gl, bv)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.on_device = dist.is_initialized() and dist.get_backend() == "nccl"
        self._stream = self.sim._torch_stream
        with torch.cuda.stream(self._stream):
            self.send_slots = torch.from_numpy(self.ex.send_slots).to(dev)
            self.recv_slots = torch.from_numpy(self.ex.recv_slots).to(dev)
            self.recv_pos = torch.from_numpy(self.ex.recv_pos).to(dev)
            self.send_buf = torch.zeros(max(self.ex.width, 1), dtype=torch.float32, device=dev)
        self._lib = _lib
        self.exchange()      # W_0 (already equal on every rank; exchanged for uniformity)

    def exchange(self):
        import torch
        import torch.distributed as dist
        if self.world == 1:
            return
        L = self._lib.lib()
        C = self._C
        sp = C.c_void_p(self._stream.cuda_stream)
        with torch.cuda.stream(self._stream):
            self._lib.check(L.hp_mono_w_gather(self.sim.h, C.c_void_p(self.send_slots.data_ptr()),
                                               len(self.ex.send_slots),
                                               C.c_void_p(self.send_buf.data_ptr()), sp),
                            "hp_mono_w_gather")
            w = self.ex.width
            if self.on_device:
                out = torch.empty(self.world * w, dtype=torch.float32, device=self.send_buf.device)
                dist.all_gather_into_tensor(out, self.send_buf[:w])
            else:
                host = self.send_buf[:w].cpu()
                parts = [torch.empty(w, dtype=torch.float32) for _ in range(self.world)]
                dist.all_gather(parts, host)
                out = torch.cat(parts).to(self.send_buf.device)
            recv = out.index_select(0, self.recv_pos).contiguous()
            self._lib.check(L.hp_mono_w_scatter(self.sim.h, C.c_void_p(self.recv_slots.data_ptr()),
                                                len(self.ex.recv_slots),
                                                C.c_void_p(recv.data_ptr()), sp),
                            "hp_mono_w_scatter")
            self._keep = recv      # alive until the scatter has run (the next sync)

    def run(self, n: int):
        for _ in range(int(n)):
            self.sim.run(1, graph_chunk=0)
            self.exchange()

    def _assemble(self, local_rows):
        """Owned per-node columns of every rank -> (..., N) in node order."""
        import torch.distributed as dist
        local_rows = np.ascontiguousarray(local_rows[..., :len(self.owned_nodes)])
        parts = [(self.owned_nodes, local_rows)]
        if self.world > 1:
            parts = [None] * self.world
            dist.all_gather_object(parts, (self.owned_nodes, local_rows))
        n = self.prob.n_myo
        out = np.empty(local_rows.shape[:-1] + (n,), local_rows.dtype)
        for nodes, rows in parts:
            out[..., nodes] = rows
        return out

    def vm_frames(self):
        return self._assemble(self.sim.vm_frames())

    def events(self):
        a, na, d, nd = self.sim.events()
        return self._assemble(a), self._assemble(na), self._assemble(d), self._assemble(nd)

    def close(self):
        self.sim.close()
