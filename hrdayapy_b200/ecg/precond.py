"""Learned flexible-CG preconditioner for the torso solve (libhrdaya_b200
hp_precond_* / hp_torso_*_fcg / hp_torso_train_precond).  No counterpart in
the reference, whose torso solver is Jacobi-PCG only."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib

LAYERS = ["e1a", "e1b", "e2a", "e2b", "e3a", "e3b", "d2a", "d2b", "d1a", "d1b", "out"]
LCIN = [16, 16, 16, 32, 32, 64, 96, 32, 48, 16, 16]
LCOUT = [16, 16, 32, 32, 64, 64, 32, 32, 16, 16, 1]


def param_offsets():
    """(w_offset, b_offset) of each layer in the flat parameter vector
    (w: [cout][cin][27], then b: [cout])."""
    o, out = 0, []
    for ci, co in zip(LCIN, LCOUT):
        ow = o
        o += co * ci * 27
        out.append((ow, o))
        o += co
    return out, o


def torso_arrays(solver):
    a = _lib.HpTorsoArrays()
    _lib.check(_lib.lib().hp_torso_arrays(solver.h, C.byref(a)), "hp_torso_arrays")
    return a


class LearnedPreconditioner:
    """M(r) = omega D^-1 r + Q A_c^-1 Q^T r + P(s CNN(...)) for the torso
    solve of ``solver`` (a TorsoSolver).  coarse_agg: 0 picks the aggregate
    size, > 0 fixes it, -1 leaves the coarse level out.  zero_output starts
    the network with a zero output layer, so that the untrained
    preconditioner is exactly the method without the network and training
    only adds corrections to it."""

    def __init__(self, solver, labels, n_materials, omega=0.6, seed=0, params=None,
                 coarse_agg=0, zero_output=True):
        _lib.require_cuda()
        arr = torso_arrays(solver)
        self.solver = solver
        self.arrays = arr
        lab = np.ascontiguousarray(labels, np.uint8)
        d = _lib.HpPrecondDesc()
        d.ni, d.nj, d.nk = lab.shape
        d.label = _lib.ptr(lab)
        d.n_materials = int(n_materials)
        d.pin_cell = int(arr.pin_cell)
        d.omega = float(omega)
        d.seed = int(seed)
        self._init = None if params is None else np.ascontiguousarray(params, np.float32)
        d.init_params = _lib.ptr(self._init)
        self._sigma = np.ascontiguousarray(solver.sigma_table, np.float64)
        d.sigma = _lib.ptr(self._sigma)
        d.h_m = float(solver.h_m)
        d.coarse_agg = int(coarse_agg)
        h = C.c_void_p()
        _lib.check(_lib.lib().hp_precond_create(C.byref(d), C.byref(h), solver.stream),
                   "hp_precond_create")
        self.h = h
        self.stream = solver.stream
        if zero_output and params is None:
            p, _ = self.params()
            ow, ob = param_offsets()[0][-1]
            p[ow:ob + LCOUT[-1]] = 0.0
            self.set_params(p)

    def coarse_info(self):
        """(aggregate edge length, coarse unknowns); (0, 0) without a coarse level."""
        ag, nc = C.c_int32(), C.c_int32()
        _lib.check(_lib.lib().hp_precond_coarse_info(self.h, C.byref(ag), C.byref(nc)),
                   "hp_precond_coarse_info")
        return int(ag.value), int(nc.value)

    def apply(self, r_ptr, z_ptr, use_net=True):
        """z = M(r) on the padded torso grid (device pointers)."""
        a = self.arrays
        _lib.check(_lib.lib().hp_precond_apply(self.h, C.c_void_p(a.label), C.c_void_p(a.invd),
                                               C.c_void_p(r_ptr), C.c_void_p(z_ptr),
                                               int(use_net), self.stream), "hp_precond_apply")

    def params(self):
        n = C.c_int64()
        _lib.check(_lib.lib().hp_precond_params(self.h, None, None, C.byref(n), 0, self.stream),
                   "hp_precond_params")
        p = np.empty(n.value, np.float32)
        g = np.empty(n.value, np.float32)
        _lib.check(_lib.lib().hp_precond_params(self.h, _lib.ptr(p), _lib.ptr(g), C.byref(n), 0,
                                                self.stream), "hp_precond_params")
        return p, g

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        n = C.c_int64()
        _lib.check(_lib.lib().hp_precond_params(self.h, _lib.ptr(p), None, C.byref(n), 1,
                                                self.stream), "hp_precond_params")

    def output(self):
        a = self.arrays
        y = np.empty((a.ni // 2) * (a.nj // 2) * (a.nk // 2), np.float32)
        sc = np.zeros(1, np.float32)
        err = np.zeros(1, np.int32)
        _lib.check(_lib.lib().hp_precond_output(self.h, _lib.ptr(y), _lib.ptr(sc), _lib.ptr(err),
                                                self.stream), "hp_precond_output")
        return y.reshape(a.ni // 2, a.nj // 2, a.nk // 2), float(sc[0]), int(err[0])

    def train_step(self, r_ptr, e_ptr, lr):
        loss = np.zeros(1, np.float32)
        _lib.check(_lib.lib().hp_precond_train_step(self.h, C.c_void_p(self.arrays.label),
                                                    C.c_void_p(self.arrays.invd), C.c_void_p(r_ptr),
                                                    C.c_void_p(e_ptr), float(lr), _lib.ptr(loss),
                                                    self.stream), "hp_precond_train_step")
        return float(loss[0])

    def train(self, vm_frames_dev, ks=(0, 2, 8, 32, 96), repeats=2, lr=1e-3, tol_exact=1e-8):
        """vm_frames_dev: CUDA tensor (n_frames, n_heart) float32 (mV)."""
        n_frames = int(vm_frames_dev.shape[0])
        ks = np.ascontiguousarray(np.sort(np.asarray(ks)), np.int32)
        hist = np.zeros(n_frames * len(ks) * repeats, np.float32)
        _lib.check(_lib.lib().hp_torso_train_precond(
            self.solver.h, self.h, C.c_void_p(vm_frames_dev.data_ptr()),
            int(vm_frames_dev.stride(0)), n_frames, _lib.ptr(ks), len(ks), int(repeats),
            float(lr), float(tol_exact), _lib.ptr(hist), self.stream), "hp_torso_train_precond")
        return hist

    def solve_frame(self, vm, tol=1e-6, max_iter=5000, fallback_iter=200, out=None,
                    use_net=True):
        """One frame by flexible CG with M (use_net=False: without the
        network; an integer k in {1, 2, 4}: the network term on every k-th
        iteration, True = 1); plain Jacobi-PCG finishes it past
        fallback_iter."""
        use_net = int(use_net)
        if use_net not in (0, 1, 2, 4):
            raise ValueError("use_net must be False, True or a period in {1, 2, 4}")
        s = self.solver
        st = _lib.HpSolveStats()
        on_dev = 0
        if hasattr(vm, "data_ptr"):
            vptr, on_dev = C.c_void_p(vm.data_ptr()), 1
        else:
            vm = np.ascontiguousarray(vm, np.float32)
            vptr = _lib.ptr(vm)
        if out is None:
            out = np.empty(s.n_read, np.float32)
        optr = C.c_void_p(out.data_ptr()) if hasattr(out, "data_ptr") else _lib.ptr(out)
        _lib.check(_lib.lib().hp_torso_solve_frame_fcg(s.h, self.h, vptr, on_dev, optr,
                                                       int(hasattr(out, "data_ptr")), float(tol),
                                                       int(max_iter), int(fallback_iter),
                                                       int(use_net), C.byref(st), s.stream),
                   "hp_torso_solve_frame_fcg")
        return out, st

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().hp_precond_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
