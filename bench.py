"""Benchmark: monodomain voxel-steps/s of the sm_100a time step, and torso
ECG solve ms/frame (plain PCG vs learned FCG at 1e-6).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                    [--impl ours|reference] [--no-torso] [--no-autotune]

One bench step = one Vm frame of simulated time (frame_steps time steps,
1 ms at dt = 0.02 ms) of the whole workload, inputs resident in HBM.  The
per-step working set (19 FP32 state arrays + coefficients, hundreds of MB)
is larger than the 126 MB L2, so no explicit flush is needed between
steps.  Prints ONE JSON line (rank 0); for the default workload it carries a
"torso" object with the ECG forward solve on frames the step simulated.

Workloads (seeded synthetic inputs, see hrdayapy_b200/synthetic.py):
  biv_shell  -- biventricular shell, ~2.5M voxels in 256^3 at 0.4 mm,
                helical fibres, endo/M/epi layers, fractal Purkinje tree
                (the configuration the headline metric is quoted on)
  slab64     -- 64x64x16 isotropic slab at 0.25 mm (the CPU-runnable case)
  ensemble16 -- 16 shell variants of uneven size in one launch per step
                against the same variants run one after another
  torso      -- the torso solve alone (--torso-shape) on seeded frames
  torso_learned -- the learned preconditioner at its stated size: 400 frames
                of the shell, training on 20,000 pairs from frames 0-199,
                test on frames 200-399

--impl reference times the CPU restatement of the reference method (FP64,
all host threads) on a bounded sample of the same workload.
Multi-GPU: each rank advances its own replica of the workload (the
monodomain step of one heart has no inter-rank exchange here), scaling weak.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples (every 100 ms) around the timed
    region; summary() keeps the samples taken inside [mark_start, mark_end]
    (or the nearest ones when the region is shorter than the period)."""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        import tempfile
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.5)
        return self

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def __exit__(self, *a):
        time.sleep(0.3)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import datetime as _dt
        rows = []
        try:
            with open(self.out.name) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) < 8:
                        continue
                    try:
                        ts = _dt.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                        rows.append((ts, float(parts[1]), float(parts[2]), parts[4:8]))
                    except ValueError:
                        continue
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        t0, t1 = self.t0 or rows[0][0], self.t1 or rows[-1][0]
        inside = [r for r in rows if t0 - 0.05 <= r[0] <= t1 + 0.05]
        if not inside:
            mid = 0.5 * (t0 + t1)
            inside = sorted(rows, key=lambda r: abs(r[0] - mid))[:2]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in inside for i in range(4)
                          if r[3][i].lower().startswith("active")})
        return {"sm_mhz": float(np.median([r[1] for r in inside])),
                "sm_max_mhz": max(r[2] for r in inside), "reasons": reasons,
                "samples": len(inside)}


def build_workload(name, seed=0):
    """Prepared problem of a workload.  With HP_BENCH_CACHE=<dir> the
    prepared arrays are pickled there and reused by later runs of the same
    workload (set-up only; nothing of the timed region is cached)."""
    import pickle
    from hrdayapy_b200 import synthetic
    cache = os.environ.get("HP_BENCH_CACHE")
    path = Path(cache) / f"{name}_{seed}.pkl" if cache else None
    if path is not None and path.exists():
        with open(path, "rb") as f:
            prob, info, last = pickle.load(f)
        synthetic.last_inputs().clear()
        synthetic.last_inputs().update(last)
        return prob, info
    if name == "slab64":
        out = synthetic.slab_problem()
    elif name == "biv_shell":
        out = synthetic.biv_shell_problem(seed=seed)
    else:
        raise SystemExit(f"unknown workload {name}")
    if path is not None:
        path.parent.mkdir(parents=True, exist_ok=True)
        with open(path, "wb") as f:
            pickle.dump((out[0], out[1], dict(synthetic.last_inputs())), f, protocol=4)
    return out


def _build_variant(v):
    """Worker of the ensemble build (spawned process, no CUDA)."""
    import pickle
    from hrdayapy_b200 import synthetic
    cache = os.environ.get("HP_BENCH_CACHE")
    path = Path(cache) / f"ensemble_variant_{v}.pkl" if cache else None
    if path is not None and path.exists():
        with open(path, "rb") as f:
            return pickle.load(f)
    out = synthetic.ensemble_variant(v)
    if path is not None:
        path.parent.mkdir(parents=True, exist_ok=True)
        with open(path, "wb") as f:
            pickle.dump(out, f, protocol=4)
    return out


def build_ensemble_variants(which, workers=8):
    """Variants `which` of the seeded ensemble, built in parallel host
    processes (spawned, so no process inherits a CUDA context)."""
    import multiprocessing as mp
    if not which:
        return []
    with mp.get_context("spawn").Pool(min(workers, len(which))) as pool:
        return pool.map(_build_variant, which)


def run_ensemble(args):
    """16 heart variants of uneven size (0.9M-3.4M voxels, shell scaled by
    U[0.7, 1.1], sigma_l, g_Ks, g_Kr varied, own Purkinje trees) advanced by
    one launch per step; brick shape and kernel from the autotuner (tuned on
    the largest variant); compared with the same steps of the 16 variants run
    one after another.  With N ranks the variants are dealt to ranks by
    longest-processing-time-first on their expected voxel counts (s^3); each
    rank advances its share as one ensemble, no data-path collective, and
    the job's time is the slowest rank's."""
    import torch
    from hrdayapy_b200 import monodomain as M, synthetic
    from hrdayapy_b200.autotune import relayout, tune
    from hrdayapy_b200.ensemble import build_ensemble
    from hrdayapy_b200.sharding import gather_to_all, lpt_assign, max_over_ranks
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    n_var = 16
    share = lpt_assign([synthetic.ensemble_params(v)[0] ** 3 for v in range(n_var)],
                       world)[rank]
    t0 = time.perf_counter()
    variants = build_ensemble_variants(share)
    t_build = time.perf_counter() - t0
    probs = [v[0] for v in variants]
    fs = probs[0].frame_steps
    big = int(np.argmax([p.n_myo for p in probs]))
    cache = os.environ.get("HP_BENCH_CACHE")
    best, table = tune(probs[big], steps=100, warmup=20,
                       cache_path=str(Path(cache) / "autotune.json") if cache else None)
    brick, kernel = tuple(best.layout.brick), best.kernel
    n = (args.warmup + args.steps) * fs
    import dataclasses
    probs = [dataclasses.replace(relayout(p, brick), kernel=kernel, n_steps=n, vm_every=0,
                                 frame_every=0, site_on=np.resize(p.site_on, n + 1))
             for p in probs]
    ens = build_ensemble(probs, gks=[v[1] for v in variants], gkr=[v[2] for v in variants])
    ens.problem.kernel = kernel
    stream = torch.cuda.Stream()

    def timed(prob):
        with torch.cuda.stream(stream):
            sim = M.MonoHandle(prob, stream=M._lib.C.c_void_p(stream.cuda_stream))
            sim.run(args.warmup * fs, graph_chunk=fs)
            stream.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.run(args.steps * fs, graph_chunk=fs)
            e1.record(stream)
            e1.synchronize()
            vm = sim.voltage()[0]
            sim.close()
        return e0.elapsed_time(e1), vm

    if dist:
        dist.barrier()
    ms_ens, vm = timed(ens.problem)
    n_local = ens.problem.n_myo
    ms_seq = 0.0
    for p in probs:
        ms, _ = timed(p)
        ms_seq += ms
    ms_ens = max_over_ranks(ms_ens, device="cuda" if dist else None)
    ms_seq = max_over_ranks(ms_seq, device="cuda" if dist else None)
    per_rank = gather_to_all({"variants": share, "voxels": int(n_local),
                              "sizes": [int(p.n_myo) for p in probs]})
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    n_vox = sum(r["voxels"] for r in per_rank)
    steps = args.steps * fs
    value = n_vox * steps / (ms_ens * 1e-3)
    line = {"metric": "ensemble voxel-steps/s", "value": value, "unit": "voxel-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_ens / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": "ensemble16", "variants": n_var, "n_voxels": int(n_vox),
                       "voxels_per_rank": [r["voxels"] for r in per_rank],
                       "variants_per_rank": [r["variants"] for r in per_rank],
                       "parallelism": f"variants sharded over {world} rank(s), LPT",
                       "n_purkinje": int(ens.problem.n_pk), "brick": list(brick),
                       "kernel": {1: "brick", 2: "pipelined", 3: "split"}[kernel],
                       "time_steps_per_bench_step": fs},
            "sequential": {"value": n_vox * steps / (ms_seq * 1e-3),
                           "ms_per_step": ms_seq / args.steps,
                           "speedup_of_one_launch": ms_seq / ms_ens},
            "autotune": table[:8], "setup_seconds": t_build,
            "roofline": {"bound": "hbm", "bytes_per_voxel_step": 177.0,
                         "achieved": n_vox * 177.0 / (ms_ens * 1e-3 / steps) / 1e9 / world,
                         "peak": peaks()[0], "unit": "GB/s (per GPU)",
                         "frac": n_vox * 177.0 / (ms_ens * 1e-3 / steps) / 1e9 / world / peaks()[0]},
            "check": {"vm_finite": bool(np.isfinite(vm).all()),
                      "vm_range_mV": [float(vm.min()), float(vm.max())]}}
    print(json.dumps(line), flush=True)


def run_torso(args):
    """Torso forward solve alone: the biventricular shell embedded in an
    elliptic-cylinder torso of --torso-shape voxels (extent 288 x 240 x 384
    mm, lungs, blood pools), seeded activation-front Vm frames 1 ms apart,
    each frame warm-started from the previous one and solved to the FP64
    true relative residual 1e-6 by plain Jacobi-PCG, by two-level FCG and by
    learned FCG (network trained for a few seconds on earlier frames)."""
    import torch
    from hrdayapy_b200 import synthetic
    from hrdayapy_b200.ecg import torso as T
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    shape = tuple(int(x) for x in args.torso_shape.split(","))
    dx = 288.0 / shape[0]
    geo = synthetic.biv_geometry()
    lab, sm, reg = synthetic.torso_for_heart(geo, shape=shape, dx=dx)
    grid = torso_grid_from_labels(lab, sm, dx)
    labels, table = T.labels_from_grid(grid)
    vox = np.argwhere(geo["S"] == 1)
    coords = vox[:, [1, 0, 2]].astype(np.float64) * geo["h"]
    proj, _ = T.projection_map(coords, reg["R"], reg["t"], 1.0, grid["origin_mm"], dx,
                               grid["active_id_map"], grid["shape"])
    solver = T.TorsoSolver(labels, table, dx, grid["pin_row"], T.heart_neighbours(vox), proj,
                           0.2625, geo["h"], grid["surface_rows"][:266])
    x = vox[:, 0].astype(np.float64) + 0.4 * vox[:, 2]
    n_fr = 8 + args.warmup + args.steps + 1
    lo, hi = x.min(), x.max()
    rng = np.random.default_rng(0)
    frames = np.stack([(-85.0 + 110.0 / (1.0 + np.exp(-(lo + (hi - lo) * (f + 0.5) / n_fr - x) / 1.5))
                        + rng.normal(0, 0.3, len(x))) for f in range(n_fr)]).astype(np.float32)
    fr = torch.from_numpy(frames).cuda()
    out = {}
    pc = None
    for name in args.torso_solvers.split(","):
        if name != "plain_pcg" and pc is None:
            pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=5)
            pc.train(fr[0:8].contiguous(), ks=tuple(range(0, 64, 8)), repeats=1, lr=1e-3)
        solver.reset()
        its, ms, rst = [], [], []
        for f in range(8, n_fr):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            if name == "plain_pcg":
                _, st = solver.solve_frame(fr[f], 1e-6, "rel", 50000)
            else:
                _, st = pc.solve_frame(fr[f], 1e-6, 50000,
                                       args.net_iters if name == "learned_fcg" else 300,
                                       use_net=args.net_every if name == "learned_fcg" else 0)
            torch.cuda.synchronize()
            if f >= 8 + 1 + args.warmup:
                ms.append((time.perf_counter() - t1) * 1e3)
                its.append(int(st.iterations))
                rst.append(int(st.restarts))
        out[name] = {"ms_per_frame": float(np.mean(ms)), "iterations": its}
        if name != "plain_pcg":
            # +100: the network run fell back to the two-level method; +1000:
            # plain PCG finished the frame; below 100: true-residual restarts
            out[name]["restarts"] = rst
        if name == "learned_fcg":
            out[name]["network_every"] = args.net_every
            out[name]["network_iterations"] = args.net_iters
    rows = solver.n_rows
    if pc is not None:
        pc.close()
    solver.close()
    p = out.get("plain_pcg", {"ms_per_frame": float("nan"), "iterations": [1]})
    t_it = p["ms_per_frame"] * 1e-3 / max(np.mean(p["iterations"]), 1)
    peak, kind = peaks()
    head = out[args.torso_solvers.split(",")[-1]]["ms_per_frame"]
    print(json.dumps({"metric": "torso solve ms/frame", "value": head,
                      "unit": "ms/frame", "higher_is_better": False, "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "data": "synthetic (seeded)",
                      "config": {"workload": f"torso {shape} @{dx} mm", "rows": int(rows)}, **out,
                      "pcg_roofline": {"bound": "hbm", "bytes_per_unknown_per_iteration": 40,
                                       "achieved": 40.0 * rows / t_it / 1e9, "peak": peak,
                                       "frac": 40.0 * rows / t_it / 1e9 / peak,
                                       "peak_source": kind}}), flush=True)


# (kernel id, brick, anisotropic) -> (DRAM bytes per myocardial voxel-step,
# the capture it comes from): ncu --metrics dram__bytes_read.sum,
# dram__bytes_write.sum over both launches of one time step
DRAM_BYTES_PER_VOXEL_STEP = {
    (3, (4, 4, 8), True): (5.0e8 / 2544045,
                           "split step: mono_diffuse_kernel 132 MB + mono_ionic_kernel 368 MB "
                           "on the 2,544,045-voxel shell"),
}


def run_torso_learned(args):
    """The learned-preconditioner configuration at its stated size: the
    biventricular shell simulated for 400 ms (Vm every 1 ms, 400 frames,
    kept on the device), the 192 x 160 x 256 torso at 1.5 mm; the network
    trained on residual / error pairs of the plain solver's own iterates on
    frames 0-199 (one plain-PCG trajectory per frame, a pair every 4
    iterations up to 396: 100 pairs a frame, 20,000 in all), then frames
    200-399 each warm-started from the previous one and solved to the FP64
    true relative residual 1e-6 by plain Jacobi-PCG, by two-level flexible
    CG without the network, by learned FCG (network on the first
    --net-iters iterations of a frame, then two-level) and with the network
    on every iteration.  Reported: ms/frame and iterations of each, the
    training time and loss."""
    import dataclasses
    import torch
    from hrdayapy_b200 import monodomain as M, synthetic
    from hrdayapy_b200.ecg import torso as T
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    t0 = time.perf_counter()
    prob, _ = build_workload("biv_shell")
    fs = prob.frame_steps
    n_frames = 400
    prob = dataclasses.replace(prob, n_steps=n_frames * fs, vm_every=fs,
                               site_on=np.resize(prob.site_on, n_frames * fs + 1))
    sim = M.MonoHandle(prob)
    sim.run(prob.n_steps, graph_chunk=fs)
    frames = torch.empty((n_frames, prob.n_myo), dtype=torch.float32, device="cuda")
    sim.vm_frames_device(frames.data_ptr(), 0, n_frames)
    torch.cuda.synchronize()
    sim.close()
    geo = synthetic.biv_geometry()
    lab, sigma_map, reg = synthetic.torso_for_heart(geo)
    dx = 1.5
    grid = torso_grid_from_labels(lab, sigma_map, dx)
    labels, table = T.labels_from_grid(grid)
    vox = np.argwhere(geo["S"] == 1)
    coords = vox[:, [1, 0, 2]].astype(np.float64) * geo["h"]
    proj, _ = T.projection_map(coords, reg["R"], reg["t"], 1.0, grid["origin_mm"], dx,
                               grid["active_id_map"], grid["shape"])
    elec = np.concatenate([synthetic.twelve_lead_electrodes(grid, reg),
                           synthetic.body_surface_grid(grid, reg)])
    rows = T.nearest_surface_rows(elec, grid["surface_xyz"], grid["surface_rows"])
    solver = T.TorsoSolver(labels, table, dx, grid["pin_row"], T.heart_neighbours(vox), proj,
                           0.2625, geo["h"], rows)
    pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=5)
    t_setup = time.perf_counter() - t0
    ks = tuple(range(0, 400, 4))
    t1 = time.perf_counter()
    hist = pc.train(frames[0:200].contiguous(), ks=ks, repeats=1, lr=1e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    test = list(range(200, 400, max(1, 200 // max(1, args.test_frames))))
    out = {}
    for name in ("plain_pcg", "two_level_fcg", "learned_fcg", "learned_fcg_every_iteration"):
        solver.reset()
        solver.solve_frame(frames[test[0] - 1], 1e-6, "rel", 50000)
        its, ms, rst = [], [], []
        prev = test[0] - 1
        for f in test:
            if f - 1 != prev:          # a subset: warm start from the previous frame
                solver.solve_frame(frames[f - 1], 1e-6, "rel", 50000)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            if name == "plain_pcg":
                _, st = solver.solve_frame(frames[f], 1e-6, "rel", 50000)
            elif name == "two_level_fcg":
                _, st = pc.solve_frame(frames[f], 1e-6, 50000, 300, use_net=0)
            elif name == "learned_fcg":
                _, st = pc.solve_frame(frames[f], 1e-6, 50000, args.net_iters, use_net=1)
            else:
                _, st = pc.solve_frame(frames[f], 1e-6, 50000, 300, use_net=1)
            torch.cuda.synchronize()
            ms.append((time.perf_counter() - t2) * 1e3)
            its.append(int(st.iterations))
            rst.append(int(st.restarts))
            prev = f
        out[name] = {"ms_per_frame": float(np.mean(ms)), "iterations_mean": float(np.mean(its)),
                     "iterations_min": int(min(its)), "iterations_max": int(max(its)),
                     "fallbacks_to_plain": int(sum(r >= 1000 for r in rst))}
    pc.close()
    solver.close()
    head = out["learned_fcg"]["ms_per_frame"]
    print(json.dumps({"metric": "torso solve ms/frame, learned vs plain PCG @1e-6", "value": head,
                      "unit": "ms/frame", "higher_is_better": False, "n_gpus": 1,
                      "data": "synthetic (seeded)", "dtype": "f32 (FP64 dots / true residual)",
                      "config": {"workload": "torso_learned: 192x160x256 torso @1.5 mm, 400 frames of "
                                             "the 2.54 M-voxel shell, train 0-199, test 200-399",
                                 "test_frames": len(test), "rows": int(solver.n_rows)
                                 if hasattr(solver, "n_rows") else None},
                      **out,
                      "training": {"frames": 200, "pairs": int(len(hist)), "ks": "0, 4, ..., 396",
                                   "seconds": t_train, "loss_first_100": float(hist[:100].mean()),
                                   "loss_last_100": float(hist[-100:].mean())},
                      "setup_seconds": t_setup}), flush=True)


def bytes_per_voxel_step(prob):
    """Algorithmic HBM bytes per myocardial voxel-step of the fused kernel:
    18 TTP06 state variables + membrane potential read and written (FP32,
    152 B), plus 24 B of per-voxel conductivity data and 1 B of region id for
    the anisotropic operator (177 B)."""
    return 177.0 if prob.anisotropic else 152.0


def run_ours(args):
    import dataclasses
    import torch
    from hrdayapy_b200 import monodomain as M

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        # the CPU baseline (N = 1 only) and the theta-scheme and torso legs
        # belong to the single-GPU line: replicas time the step alone, so no
        # rank waits at the final barrier while rank 0 runs extra work
        args.cpu_baseline = args.theta = args.torso = False
    prob, info = build_workload(args.workload)
    fs = prob.frame_steps
    tune_table = None
    if args.kernel:
        prob.kernel = args.kernel
    elif args.autotune:
        from hrdayapy_b200.autotune import tune
        cache = os.environ.get("HP_BENCH_CACHE")
        prob, tune_table = tune(prob, steps=100, warmup=20,
                                cache_path=str(Path(cache) / "autotune.json") if cache else None)
        prob.frame_steps = fs
    total_steps = (args.warmup + args.steps) * fs
    prob.n_steps = total_steps
    site_on_full = np.array(prob.site_on)       # the whole run's schedule, for the parity leg
    prob.site_on = np.resize(prob.site_on, total_steps + 1)
    n_vox = prob.n_myo
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        sim = M.MonoHandle(prob, stream=M._lib.C.c_void_p(stream.cuda_stream))
        kinfo = sim.kernel_info()
        sim.run(args.warmup * fs, graph_chunk=fs)
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            clk.mark_start()
            ev0.record(stream)
            sim.run(args.steps * fs, graph_chunk=fs)
            ev1.record(stream)
            ev1.synchronize()
            clk.mark_end()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        vm_last = sim.voltage()[0]
        sim.close()
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    voxel_steps = n_vox * fs * args.steps * world
    value = voxel_steps / (ms * 1e-3)
    per_launch_ms = ms / (fs * args.steps)
    bpv = bytes_per_voxel_step(prob)
    achieved = n_vox * bpv / (per_launch_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()

    # DRAM bytes per time step: dram__bytes_read.sum + dram__bytes_write.sum
    # of one step's launches from an ncu capture of the same kernel and brick
    # shape, per myocardial voxel, scaled by this workload's voxel count
    traffic, traffic_note = None, "no ncu capture for this kernel / brick shape"
    cap = DRAM_BYTES_PER_VOXEL_STEP.get((kinfo[0], tuple(prob.layout.brick), bool(prob.anisotropic)))
    if cap is not None:
        traffic = cap[0] * n_vox
        traffic_note = (f"{cap[0]:.1f} B per voxel-step x {n_vox} voxels ({cap[1]}) vs "
                        f"algorithmic {bpv * n_vox / 1e6:.0f} MB")
    # end to end through the C-ABI handle: host buffers in, Vm frames out;
    # three repetitions, the median reported (the first one also pays
    # first-use costs of the process: module loads)
    import torch
    k_e2e = max(1, int(round(args.e2e_ms)))
    out_e2e = torch.empty((k_e2e, prob.n_myo), dtype=torch.float32, pin_memory=True)
    reps = sorted((e2e_run(prob, args, fs, out_e2e) for _ in range(3)), key=lambda r: r["value"])
    del out_e2e
    e2e = dict(reps[1], repetitions=[r["value"] for r in reps])
    if rank == 0:
        line = {
            "metric": "monodomain voxel-steps/s", "value": value, "unit": "voxel-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "n_voxels": int(n_vox),
                       "n_purkinje": int(prob.n_pk), "dt_ms": prob.dt,
                       "time_steps_per_bench_step": fs, "brick": list(prob.layout.brick),
                       "kernel": {1: "brick", 2: "pipelined", 3: "split"}[kinfo[0]], "grid": kinfo[1],
                       "autotuned": tune_table is not None,
                       "l2": "working set > L2 (no flush)", "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_note": traffic_note,
                         "bytes_per_voxel_step": bpv, "peak_source": peak_kind},
            "e2e": e2e,
            "gpu_launches": int(args.steps * fs * (2 if kinfo[0] == 3 else 1) + args.steps),
            "clocks": clk.summary(),
            "check": {"vm_finite": bool(np.isfinite(vm_last).all()),
                      "vm_range_mV": [float(vm_last.min()), float(vm_last.max())]},
        }
        if args.cpu_baseline:
            pp = dataclasses.replace(prob, site_on=site_on_full)
            pp.frame_steps = fs
            line["cpu_baseline"], line["check"]["parity"] = shell_parity_and_cpu_baseline(
                pp, args, parity_ms=args.parity_ms)
        if tune_table is not None:
            line["autotune"] = [{k: v for k, v in t.items()} for t in tune_table[:8]]
        if args.theta:
            line["theta_scheme"] = theta_leg(prob)
        if args.torso:
            line["torso"] = torso_leg(prob, net_every=args.net_every, net_iters=args.net_iters,
                                      parity=args.cpu_baseline)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def theta_leg(prob, n_steps=96, warm=496, theta=0.5, cg_tol=1e-5):
    """The reference's default diffusion half (theta = 0.5, Crank-Nicolson,
    relative tolerance 1e-5) on the same heart, timed over steps 496-592
    (about 10-12 ms: the wavefront is crossing the heart; six replays of the
    16-step graph): ms per time step and CG iterations per step."""
    import dataclasses
    import torch
    from hrdayapy_b200 import monodomain as M
    n = warm + n_steps
    p = dataclasses.replace(prob, theta=theta, cn_tol=cg_tol, cn_max_iter=100, kernel=0,
                            n_steps=n, site_on=np.resize(prob.site_on, n + 1), vm_every=0,
                            frame_every=0)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        sim = M.MonoHandle(p, stream=M._lib.C.c_void_p(stream.cuda_stream))
        sim.run(warm)
        it0, s0, _, _ = sim.cn_stats()
        stream.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        sim.run(n_steps)
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        it1, s1, unconv, brk = sim.cn_stats()
        vm = sim.voltage()[0]
        sim.close()
    return {"theta": theta, "cg_tol": cg_tol, "steps": n_steps, "first_step": warm,
            "ms_per_step": ms / n_steps,
            "voxel_steps_per_s": prob.n_myo * n_steps / (ms * 1e-3),
            "cg_iters_per_step": (it1 - it0) / max(1, s1 - s0),
            "unconverged": unconv, "breakdowns": brk,
            "vm_finite": bool(np.isfinite(vm).all())}


def torso_leg(prob, n_train=8, n_test=5, net_every=1, net_iters=25, parity=True, n_parity=2):
    """Torso forward solve (192 x 160 x 256 voxels at 1.5 mm, lungs, blood
    pools, the biventricular shell embedded; 12-lead + 16 x 16 read-out) on
    Vm frames simulated here by the fused monodomain step (1 ms apart).  The
    preconditioner's network is trained on frames of early activation, then
    held-out frames are solved to the FP64 true relative residual 1e-6, each
    warm-started from the previous one, by plain Jacobi-PCG, by flexible CG
    with the two-level preconditioner without the network, and with it."""
    import dataclasses
    import torch
    from hrdayapy_b200 import monodomain as M, synthetic
    from hrdayapy_b200.ecg import torso as T
    from hrdayapy_b200.ecg.precond import LearnedPreconditioner
    from hrdayapy_b200.ecg.torso_grid import torso_grid_from_labels
    t_setup = time.perf_counter()
    fs = prob.frame_steps
    first = 20                                   # ms: frames from early activation on
    last = first + 4 * n_train + n_test + 1
    prob = dataclasses.replace(prob, n_steps=last * fs, vm_every=fs,
                               site_on=np.resize(prob.site_on, last * fs + 1))
    sim = M.MonoHandle(prob)
    sim.run(prob.n_steps, graph_chunk=fs)
    frames = torch.empty((last - first, prob.n_myo), dtype=torch.float32, device="cuda")
    sim.vm_frames_device(frames.data_ptr(), first, last - first)
    torch.cuda.synchronize()
    sim.close()
    geo = synthetic.biv_geometry()
    lab, sigma_map, reg = synthetic.torso_for_heart(geo)
    dx = 1.5
    grid = torso_grid_from_labels(lab, sigma_map, dx)
    labels, table = T.labels_from_grid(grid)
    vox = np.argwhere(geo["S"] == 1)
    coords = vox[:, [1, 0, 2]].astype(np.float64) * geo["h"]
    proj, _ = T.projection_map(coords, reg["R"], reg["t"], 1.0, grid["origin_mm"], dx,
                               grid["active_id_map"], grid["shape"])
    elec = np.concatenate([synthetic.twelve_lead_electrodes(grid, reg),
                           synthetic.body_surface_grid(grid, reg)])
    rows = T.nearest_surface_rows(elec, grid["surface_xyz"], grid["surface_rows"])
    solver = T.TorsoSolver(labels, table, dx, grid["pin_row"], T.heart_neighbours(vox), proj,
                           0.2625, geo["h"], rows)
    pc = LearnedPreconditioner(solver, labels, len(table), omega=0.6, seed=5)
    t_setup = time.perf_counter() - t_setup
    t0 = time.perf_counter()
    hist = pc.train(frames[0:4 * n_train:4].contiguous(), ks=tuple(range(0, 64, 8)), repeats=1,
                    lr=1e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    test0 = 4 * n_train      # frame index (into `frames`) the held-out chain starts from
    out = {}
    xs = {}                  # solutions of the first n_parity held-out frames, per method
    x_start = None           # plain PCG's solution of the chain's first frame
    for name in ("plain_pcg", "two_level_fcg", "learned_fcg"):
        solver.reset()
        solver.solve_frame(frames[test0], 1e-6, "rel", 50000)
        if parity and name == "plain_pcg":
            x_start = solver.solution()
        its, ms, rel, rst = [], [], [], []
        for f in range(test0 + 1, test0 + 1 + n_test):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            if name == "plain_pcg":
                _, st = solver.solve_frame(frames[f], 1e-6, "rel", 50000)
            else:
                _, st = pc.solve_frame(frames[f], 1e-6, 50000,
                                       net_iters if name == "learned_fcg" else 300,
                                       use_net=net_every if name == "learned_fcg" else 0)
            torch.cuda.synchronize()
            ms.append((time.perf_counter() - t1) * 1e3)
            its.append(int(st.iterations))
            rel.append(float(st.rel_residual))
            rst.append(int(st.restarts))
            if parity and f <= test0 + n_parity:
                xs.setdefault(name, []).append(solver.solution())
        out[name] = {"ms_per_frame": float(np.mean(ms)), "iterations": its,
                     "max_rel_residual": max(rel)}
        if name != "plain_pcg":
            out[name]["restarts"] = rst     # +100 network fallback, +1000 plain PCG
        if name == "learned_fcg":
            out[name]["network_every"] = net_every
            out[name]["network_iterations"] = net_iters   # then the two-level method
    n_rows = solver.n_rows
    ag, nc = pc.coarse_info()
    pc.close()
    solver.close()
    extra = {}
    if parity:
        vm_par = frames[test0 + 1:test0 + 1 + n_parity].cpu().numpy()
        extra["cpu_baseline"], extra["check"] = torso_parity_and_cpu_baseline(
            grid, vox, coords, reg, geo["h"], vm_par, xs, rows, x_start=x_start)
    peak, peak_kind = peaks()
    p = out["plain_pcg"]
    t_it = p["ms_per_frame"] * 1e-3 / max(np.mean(p["iterations"]), 1)
    return {"workload": "torso 192x160x256 @1.5 mm, lungs/blood/heart, 12-lead + 16x16 grid",
            "unit": "ms/frame", "rows": int(n_rows), "tol": "FP64 true relative residual 1e-6",
            "frames": f"{n_test} held-out frames ({first + test0 + 1}-{first + test0 + n_test} ms), "
                      "each warm-started from the previous one",
            **out,
            "coarse_level": {"aggregate": ag, "unknowns": nc},
            "training": {"frames": n_train, "pairs_x_steps": int(len(hist)),
                         "loss_first": float(hist[:8].mean()), "loss_last": float(hist[-8:].mean()),
                         "seconds": t_train},
            "setup_seconds": t_setup,
            "pcg_roofline": {"bound": "hbm", "bytes_per_unknown_per_iteration": 40,
                             "achieved": 40.0 * n_rows / t_it / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": 40.0 * n_rows / t_it / 1e9 / peak, "peak_source": peak_kind,
                             "note": "plain PCG time per iteration incl. its per-frame set-up"},
            **extra}


def e2e_run(prob, args, fs, out):
    """One whole run as a user makes it: hp_mono_create from host arrays
    (the problem upload), then K frames of fs steps, each frame's Vm read
    back into pinned host memory (out, K x n_myo).  K = the run's length in
    ms (--e2e-ms, by default the configuration's 400 ms), so the upload is
    paid once per run as in the configuration."""
    import torch
    from hrdayapy_b200 import monodomain as M
    import dataclasses
    k = out.shape[0]
    p2 = dataclasses.replace(prob, n_steps=k * fs, site_on=np.resize(prob.site_on, k * fs + 1),
                             vm_every=fs)
    h2d = (p2.tag.nbytes + (p2.wface.nbytes + p2.doff.nbytes if p2.anisotropic else 0) +
           p2.layout.brick_nbr.nbytes + p2.pk_ptr.nbytes + p2.pk_idx.nbytes +
           p2.pk_coef.nbytes + p2.pmj_row.nbytes + p2.surf_of_slot.nbytes +
           p2.site_on.nbytes + p2.layout.slot_of_node.nbytes)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim = M.MonoHandle(p2)
    t1 = time.perf_counter()
    # each frame's D2H (pinned) runs on the handle's copy stream while the
    # next frame's steps run
    for f in range(k):
        sim.run(fs, graph_chunk=fs)
        sim.vm_frames_async(f, 1, out[f])
    sim.wait_copies()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    dt_s = t2 - t0
    sim.close()
    return {"value": p2.n_myo * fs * k / dt_s, "unit": "voxel-steps/s",
            "h2d_bytes_per_step": int(h2d // k), "d2h_bytes_per_step": int(p2.n_myo * 4),
            "steps": k, "includes": f"one {k}-ms run: hp_mono_create upload + {k * fs} steps "
                                    f"+ {k} Vm frames D2H (one per ms, each copy overlapping "
                                    "the next frame's steps)",
            "create_s": t1 - t0, "run_and_d2h_s": t2 - t1}


def shell_parity_and_cpu_baseline(prob, args, parity_ms=22.0, chunk=25):
    """The FP64 CPU restatement of the reference method (oracle: the C time
    loop on all host threads) runs the workload from rest for parity_ms of
    simulated time (22 ms: the tree's first junction band fires at 12.7 ms
    and its wavefronts then spread through the myocardium), recording every
    myocardial node's first -20 mV crossing in the loop.  The wall time of
    its time loop is the CPU baseline (voxel-steps/s); its final state and
    activation times are the FP64 run that the GPU's FP32 run of the same
    steps (same kernel and bricks as the timed run) is checked against:
    Vm RMS over all myocardial nodes and over the Purkinje nodes after the
    last step, max activation-time error over the voxels both runs
    activated, and how many voxels only one run activated."""
    import dataclasses
    from hrdayapy_b200 import monodomain as M, synthetic
    from oracle import mono as orc
    n = int(round(parity_ms / prob.dt))
    fs = int(getattr(prob, "frame_steps", 50))
    if len(prob.site_on) < n + 1:
        raise SystemExit("parity leg: stimulus table shorter than the parity window")
    p = dataclasses.replace(prob, n_steps=n, site_on=np.array(prob.site_on[:n + 1]), vm_every=0,
                            frame_every=0, act_threshold=-20.0, deact_threshold=-20.0)
    sim = M.MonoHandle(p)
    sim.run(n, graph_chunk=fs)
    a, na, _, _ = sim.events()
    vm, vp = sim.voltage()
    sim.close()
    g = synthetic.last_inputs()
    ctx = orc.setup(*g["args"], vm_save_dt=None, **g["kw"])
    first, _, _ = orc.advance_events(ctx, n, -20.0, chunk=chunk)
    secs = ctx["_adv_seconds"]
    N, Np = ctx["N"], ctx["Np"]
    Vo = ctx["V"]
    rms = float(np.sqrt(np.mean((vm.astype(np.float64) - Vo[Np:]) ** 2)))
    rms_p = float(np.sqrt(np.mean((vp.astype(np.float64) - Vo[:Np]) ** 2))) if Np else 0.0
    act_g = na >= 1
    act_o = np.isfinite(first)
    both = act_g & act_o
    err = float(np.max(np.abs(a[0][both].astype(np.float64) - first[both]))) if both.any() else None
    # a voxel activated by one run only should be crossing at the window's end
    one = act_g ^ act_o
    t_one = np.where(act_g, a[0], first)[one]
    one_sided_earliest = float(t_one.min()) if one.any() else None
    check = {"reference": f"FP64 oracle of the reference method, same {n} steps from rest",
             "steps": n, "simulated_ms": n * prob.dt,
             "vm_rms_mV": rms, "purkinje_vm_rms_mV": rms_p,
             "max_act_err_ms": err, "act_threshold_mV": -20.0,
             "activated_both": int(both.sum()), "activated_gpu_only": int((act_g & ~act_o).sum()),
             "activated_oracle_only": int((act_o & ~act_g).sum()),
             "one_sided_earliest_ms": one_sided_earliest,
             "tolerances": {"vm_rms_mV": 0.5, "max_act_err_ms": 0.1}}
    base = {"value": N * n / secs, "unit": "voxel-steps/s", "cores": int(orc.lib().orc_num_threads()),
            "kind": "port",
            "sample": f"{n} time steps (0-{n * prob.dt:g} ms) from rest of the full workload "
                      f"({N} nodes incl. Purkinje), FP64; set-up and crossing bookkeeping excluded"}
    return base, check


def torso_parity_and_cpu_baseline(grid, vox, coords, reg, h_fine_mm, vm_frames, xs, rows,
                                  sigma_i=0.2625, x_start=None):
    """FP64 check of the GPU's torso potentials on held-out frames, and the
    reference method timed on the host cores.  The oracle assembles the
    reference's stiffness (harmonic-mean faces, build_torso_grid.py:276-397),
    pins it, builds each frame's FP64 source (compute_bspm.py:381-419) and
    solves it by FP64 Jacobi-CG (orc_csr_pcg) to a 1e-10 relative true
    residual.  Frame 0 starts from the GPU's plain-PCG solution (any start
    reaches the same 1e-10 solution).  Frame 1 is first solved as the
    reference solves a frame -- Jacobi-PCG warm-started from the previous
    frame's solution, here to the 1e-6 relative residual of the
    configuration -- and that solve is timed (the CPU baseline, ms/frame),
    then continued to 1e-10.  Per GPU method: the true relative residual of
    its solution re-evaluated on the host with the FP64 operator, the
    relative L2 of each of the 12 leads over the frames against the FP64
    solution, and of the 16 x 16 body-surface grid (as is, and with each
    frame's mean removed: an FP32 right-hand side carries a rounding-size
    net source that the pinned system turns into a near-uniform offset,
    which leads cancel).

    The 1e-10 solutions measure each method's truncation error at the
    1e-6 stopping rule as well as its arithmetic.  With ``x_start`` (plain
    PCG's solution of the frame before the first held-out frame), plain PCG
    is also compared with an FP64 run of the same method: Jacobi-PCG in FP64
    from that same start over the held-out frames, each warm-started from
    the previous frame's FP64 solution, stopped where the GPU's relative
    rule proposes convergence (recursive residual below 0.5 x 1e-6).  That
    difference is the cost of the FP32 vectors alone."""
    from oracle import mono as orc, torso as O
    from hrdayapy_b200.ecg import torso as T
    dx = float(grid["dx_mm"])
    A, _, _ = O.assemble_stiffness(grid["sigma_vol"], dx * 1e-3, grid["active_mask"])
    pin = int(grid["pin_row"])
    Ap = O.pinned_csr(A, pin)
    del A
    K = O.heart_laplacian(np.asarray(vox, np.int64), len(vox))
    proj, valid = O.projection_map(np.asarray(coords, np.float64), np.asarray(reg["R"], np.float64),
                                   np.asarray(reg["t"], np.float64), 1.0,
                                   np.asarray(grid["origin_mm"], np.float64), dx,
                                   np.asarray(grid["active_id_map"]), grid["shape"])
    nrow = Ap.shape[0]
    bs = [O.frame_rhs(K, v, proj, valid, nrow, pin, sigma_i, h_fine_mm * 1e-3, dx) for v in vm_frames]
    x0, it0, rel0, _ = O.pcg_fp64(Ap, bs[0], xs["plain_pcg"][0], tol=1e-10)
    t = time.perf_counter()
    x1, it1, rel1, _ = O.pcg_fp64(Ap, bs[1], x0, tol=1e-6)
    t_cpu = time.perf_counter() - t
    x1, it1b, rel1b, _ = O.pcg_fp64(Ap, bs[1], x1, tol=1e-10)
    xo = [x0, x1]
    rows = np.asarray(rows, np.int64)

    def leads(xl):
        e = np.stack([x[rows[:10]] for x in xl], 1) * 1e3          # (10, frames) mV
        return T.twelve_lead(e), np.stack([x[rows[10:]] for x in xl], 1) * 1e3

    Lo, Go = leads(xo)
    out = {}
    for name, xl in xs.items():
        Lg, Gg = leads(xl[:len(xo)])
        rel_lead = np.linalg.norm(Lg - Lo, axis=1) / np.linalg.norm(Lo, axis=1)
        Gd = (Gg - Gg.mean(0)) - (Go - Go.mean(0))
        out[name] = {
            "host_true_rel_residual": [float(np.linalg.norm(b - Ap @ x) / np.linalg.norm(b))
                                       for b, x in zip(bs, xl)],
            "ecg_rel_l2_per_lead": [float(v) for v in rel_lead],
            "ecg_rel_l2_max": float(rel_lead.max()),
            "grid_rel_l2": float(np.linalg.norm(Gg - Go) / np.linalg.norm(Go)),
            "grid_rel_l2_offset_free": float(np.linalg.norm(Gd) /
                                             np.linalg.norm(Go - Go.mean(0)))}
    if x_start is not None and "plain_pcg" in xs:
        xm, its_m = [], []
        xp = np.asarray(x_start, np.float64)
        for b in bs:
            xp, itm, _, _ = O.pcg_fp64(Ap, b, xp, tol=0.5e-6)
            xm.append(xp)
            its_m.append(itm)
        Lm, Gm = leads(xm)
        Lg, Gg = leads(xs["plain_pcg"][:len(xm)])
        rel_lead = np.linalg.norm(Lg - Lm, axis=1) / np.linalg.norm(Lm, axis=1)
        Gd = (Gg - Gg.mean(0)) - (Gm - Gm.mean(0))
        out["plain_pcg"]["vs_fp64_same_method"] = {
            "reference": "FP64 Jacobi-PCG from the GPU's warm start, each frame warm-started "
                         "from the previous FP64 solution, stopped at recursive relative "
                         "residual 5e-7 (where the GPU's relative rule proposes convergence)",
            "oracle_iterations": its_m,
            "ecg_rel_l2_per_lead": [float(v) for v in rel_lead],
            "ecg_rel_l2_max": float(rel_lead.max()),
            "grid_rel_l2_offset_free": float(np.linalg.norm(Gd) /
                                             np.linalg.norm(Gm - Gm.mean(0)))}
    check = {"reference": "FP64 Jacobi-CG on the reference's assembled stiffness and FP64 "
                          "source, to a 1e-10 relative true residual",
             "frames": len(xo), "oracle_rel_residual": [rel0, rel1b],
             "oracle_iterations": [it0, it1 + it1b], "tolerance_ecg_rel_l2": 1e-3, **out}
    base = {"value": t_cpu * 1e3, "unit": "ms/frame", "iterations": it1,
            "cores": int(orc.lib().orc_num_threads()), "kind": "port",
            "sample": "one held-out frame: FP64 Jacobi-PCG on the assembled reference operator, "
                      "warm-started from the previous frame's solution, to the 1e-6 relative "
                      "true residual"}
    return base, check


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import mono as orc
    from hrdayapy_b200 import synthetic
    prob, info = build_workload(args.workload)
    g = synthetic.last_inputs()
    n_per = 2 if args.workload == "biv_shell" else 50
    kw = dict(g["kw"])
    kw["T"] = (args.warmup + args.steps) * n_per * kw["dt"] + kw["dt"]
    ctx = orc.setup(*g["args"], vm_save_dt=None, **kw)
    N = ctx["N"]
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        orc.advance(ctx, n_per, snapshots=False)
        dt_s = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt_s)
    tot = sum(times)
    value = N * n_per * len(times) / tot
    cores = orc.lib().orc_num_threads()
    line = {"impl": "reference", "metric": "monodomain voxel-steps/s", "value": value,
            "unit": "voxel-steps/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / len(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "n_voxels": int(prob.n_myo),
                       "n_purkinje": int(prob.n_pk), "dt_ms": prob.dt,
                       "time_steps_per_bench_step": n_per},
            "cpu_baseline": {"value": value, "unit": "voxel-steps/s", "cores": int(cores),
                             "kind": "port",
                             "sample": f"{n_per} time steps per bench step, FP64, set-up excluded"},
            "e2e": {"value": value, "unit": "voxel-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="biv_shell")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false",
                    help="skip the FP64 oracle legs (CPU baselines and the parity checks)")
    ap.add_argument("--parity-ms", type=float, default=22.0,
                    help="simulated ms of the FP64 oracle run the shell is checked against")
    ap.add_argument("--torso-shape", default="192,160,256",
                    help="torso voxels for --workload torso (extent fixed at 288 x 240 x 384 mm)")
    ap.add_argument("--torso-solvers", default="plain_pcg,two_level_fcg,learned_fcg",
                    help="torso workload: solvers to time (the last one is the headline)")
    ap.add_argument("--test-frames", type=int, default=200,
                    help="torso_learned: held-out frames solved (evenly spaced in 200-399)")
    ap.add_argument("--net-every", type=int, default=1, choices=[1, 2, 4],
                    help="learned FCG: the network term on every k-th iteration")
    ap.add_argument("--net-iters", type=int, default=25,
                    help="learned FCG: iterations with the network before the two-level "
                         "method takes over the frame")
    ap.add_argument("--no-theta", dest="theta", action="store_false",
                    help="skip the theta = 0.5 (Crank-Nicolson) leg")
    ap.add_argument("--no-torso", dest="torso", action="store_false",
                    help="skip the torso ms/frame leg (plain PCG vs learned FCG)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default brick shape and kernel instead of timing candidates")
    ap.add_argument("--e2e-ms", type=float, default=400.0,
                    help="simulated length of the end-to-end run (one Vm frame per ms); the "
                         "configuration's 400 ms by default")
    ap.add_argument("--kernel", type=int, default=0,
                    help="monodomain step kernel: 0 auto, 1 per-brick, 2 pipelined, 3 split")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble16":
        run_ensemble(args)
    elif args.workload == "torso":
        run_torso(args)
    elif args.workload == "torso_learned":
        run_torso_learned(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
