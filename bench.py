"""Benchmark: monodomain voxel-steps/s of the fused sm_100a time step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                    [--impl ours|reference]

One bench step = one Vm frame of simulated time (frame_steps time steps,
1 ms at dt = 0.02 ms) of the whole workload, inputs resident in HBM.  The
per-step working set (19 FP32 state arrays + coefficients, hundreds of MB)
is larger than the 126 MB L2, so no explicit flush is needed between
steps.  Prints ONE JSON line (rank 0).

Workloads (seeded synthetic inputs, see hrdayapy_b200/synthetic.py):
  biv_shell  -- biventricular shell, ~2.5M voxels in 256^3 at 0.4 mm,
                helical fibres, endo/M/epi layers, fractal Purkinje tree
                (the configuration the headline metric is quoted on)
  slab64     -- 64x64x16 isotropic slab at 0.25 mm (the CPU-runnable case)

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
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}",
                                      f"--query-gpu={self.Q}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def build_workload(name, seed=0):
    from hrdayapy_b200 import synthetic
    if name == "slab64":
        return synthetic.slab_problem()
    if name == "biv_shell":
        return synthetic.biv_shell_problem(seed=seed)
    raise SystemExit(f"unknown workload {name}")


def bytes_per_voxel_step(prob):
    """Algorithmic HBM bytes per myocardial voxel-step of the fused kernel:
    18 TTP06 state variables + membrane potential read and written (FP32,
    152 B), plus 24 B of per-voxel conductivity data and 1 B of region id for
    the anisotropic operator (177 B)."""
    return 177.0 if prob.anisotropic else 152.0


def run_ours(args):
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
    prob, info = build_workload(args.workload)
    fs = prob.frame_steps
    total_steps = (args.warmup + args.steps) * fs
    prob.n_steps = total_steps
    prob.site_on = np.resize(prob.site_on, total_steps + 1)
    n_vox = prob.n_myo
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        sim = M.MonoHandle(prob, stream=M._lib.C.c_void_p(stream.cuda_stream))
        sim.run(args.warmup * fs, graph_chunk=fs)
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            ev0.record(stream)
            sim.run(args.steps * fs, graph_chunk=fs)
            ev1.record(stream)
            ev1.synchronize()
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

    # end to end through the C-ABI handle: host buffers in, Vm frames out
    e2e = e2e_run(prob, args, fs)
    if rank == 0:
        line = {
            "metric": "monodomain voxel-steps/s", "value": value, "unit": "voxel-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "n_voxels": int(n_vox),
                       "n_purkinje": int(prob.n_pk), "dt_ms": prob.dt,
                       "time_steps_per_bench_step": fs, "brick": list(prob.layout.brick),
                       "l2": "working set > L2 (no flush)", "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "bytes_per_voxel_step": bpv, "peak_source": peak_kind},
            "e2e": e2e,
            "gpu_launches": int(args.steps * fs + args.steps),
            "clocks": clk.summary(),
            "check": {"vm_finite": bool(np.isfinite(vm_last).all()),
                      "vm_range_mV": [float(vm_last.min()), float(vm_last.max())]},
        }
        if args.cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(prob, info, args)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def e2e_run(prob, args, fs):
    """hp_mono_create from host arrays + K frames + D2H of each frame."""
    import torch
    from hrdayapy_b200 import monodomain as M
    import dataclasses
    k = max(1, min(args.steps, 10))
    p2 = dataclasses.replace(prob, n_steps=k * fs, site_on=prob.site_on[: k * fs + 1].copy(),
                             vm_every=fs)
    h2d = (p2.tag.nbytes + (p2.wface.nbytes + p2.doff.nbytes if p2.anisotropic else 0) +
           p2.layout.brick_nbr.nbytes + p2.pk_ptr.nbytes + p2.pk_idx.nbytes +
           p2.pk_coef.nbytes + p2.pmj_row.nbytes + p2.surf_of_slot.nbytes +
           p2.site_on.nbytes + p2.layout.slot_of_node.nbytes)
    out = torch.empty((k, p2.n_myo), dtype=torch.float32, pin_memory=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim = M.MonoHandle(p2)
    for f in range(k):
        sim.run(fs, graph_chunk=fs)
        sim.vm_frames(f, 1, out=out[f].numpy())
    torch.cuda.synchronize()
    dt_s = time.perf_counter() - t0
    sim.close()
    return {"value": p2.n_myo * fs * k / dt_s, "unit": "voxel-steps/s",
            "h2d_bytes_per_step": int(h2d // k), "d2h_bytes_per_step": int(p2.n_myo * 4),
            "steps": k, "includes": "hp_mono_create upload + run + per-frame Vm D2H"}


def cpu_baseline(prob, info, args, budget_s=15.0):
    """FP64 CPU restatement of the reference method (oracle), all host
    threads, on a bounded number of time steps of the same workload."""
    from oracle import mono as orc
    from hrdayapy_b200 import synthetic
    g = synthetic.last_inputs()
    nthreads = orc.lib().orc_num_threads()
    ctx = orc.setup(*g["args"], vm_save_dt=None, **g["kw"])
    t0 = time.perf_counter()
    orc.advance(ctx, 2, snapshots=False)
    per_step = (time.perf_counter() - t0) / 2
    n = int(max(2, min(500, budget_s / max(per_step, 1e-6))))
    t0 = time.perf_counter()
    orc.advance(ctx, n, snapshots=False)
    elapsed = time.perf_counter() - t0
    N = ctx["N"]
    return {"value": N * n / elapsed, "unit": "voxel-steps/s", "cores": int(nthreads),
            "kind": "port",
            "sample": f"{n} time steps of the full workload ({N} nodes incl. Purkinje), "
                      f"FP64, set-up excluded"}


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
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
