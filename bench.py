#!/usr/bin/env python3
"""Benchmark of the D2Q9 collide-stream hot path (one JSON line on rank 0).

Workload (the channel-flow-past-a-cylinder configuration): 4096 x 1024 D2Q9,
MRT + Smagorinsky (Cs = 0.1), FP32, Zou-He velocity inlet u = 0.05 (cosine
ramp as in the reference), zero-gradient outlet, bounce-back channel walls,
cylinder D = 128 centred at (1024, 512), nu = 6.4e-4 (tau = 0.50192),
initial u_y noise uniform +-1e-4 from numpy PCG64 seed 0.  --T sets the
steps fused per launch (default 2, the register wavefront kernel, the fastest
path for this workload; 1 runs the streaming kernel, 3-8 the other temporally
blocked kernels).
Synthetic inputs with that shape (there is no external dataset).

One bench "step" is one frame of `--frame` physical steps (default 50, the
reference driver's 25 graph launches of 2 steps per displayed frame,
lbm_mine2.py:88-91).  The e2e figure runs that frame through the public API
with the solid mask uploaded from pinned host memory and the vorticity image
(RGBA8, W x H x 4 bytes) read back to pinned host memory every frame.
Metric: MLUPS = W*H*physical steps / time, counting every cell as the
reference does (lbm_mine2.py:106).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--T 1..8] [--storage f32|f16|bf16] [--inplace] [--closure smag|mlp]
                    [--workload cylinder|batch|dropins|c2|c3|c4|like-reference]

--inplace runs the workload in one state buffer (lbm_run_inplace: the AA
pattern, one pull-push and one local kernel per pair of steps; T = 1 per kernel).
--workload batch times 256 independent channel domains of uneven size in one
persistent launch per T steps (FP16 storage) against one launch per domain.
--workload c2 runs the cylinder workload for 50 000 steps with drag and lift
sampled every 100 steps (mean drag coefficient, RMS lift, Strouhal number).
--workload c3 runs the 8192 x 2048 cylinder (D = 256, Re = 20 000) in FP64 (the
judge: double storage and arithmetic), FP32, FP16 and BF16 deviation storage to
1k / 10k / 50k steps and reports each format's velocity error against the FP64
run, and each format's MLUPS at that size.
--workload c4 runs decaying periodic turbulence at 1024^2 with no closure,
Smagorinsky and the learned closure (FP32 and FP16 storage) against a 4096^2
judge filtered 4x, the network trained on the GPU on another seed's judge, and
reports each variant's velocity error per snapshot and MLUPS.
--workload dropins times the drop-in entry points for the reference's three
kernels (lbm_smemaa_step T=4, lbm_blocked_step T=6, lbm_core4_step) and the
general solver's BGK path at the drivers' 2048 x 512 and at 4096 x 1024; with
--impl reference, the reference's own kernels on the same inputs.

--workload like-reference runs the reference arm's configuration (the reference's
constants Cs = 0.20, s = 1.1) through this repository's drop-in entry points with
u, v, rho written every step (lbm_core4_step), every two steps (lbm_core4_run,
T = 2 per call) and once per frame, next to the reference kernel in the same
process.

--impl reference times the reference's own kernel for this path
(fused_lbmkernel of lbm_core4.cu, MRT + Smagorinsky, one step per launch,
compiled from its source into oracle/_ref/) on the same workload.  Under
torchrun every rank runs an independent replica (weak scaling, no data-path
collective); the reference arm runs on rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lbm-cuda_b200"))

W, H = 4096, 1024
CYL = (1024, 512, 128)
NU = 6.4e-4
TAU = 3.0 * NU + 0.5
U_IN = 0.05
CS = 0.1
B_ALG = 72.0  # algorithmic bytes per lattice update, FP32: one read + one write of 9 populations
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
HBM_FALLBACK_GBS = 6650.0


def hbm_peak():
    try:
        with open(PEAKS_FILE) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def workload():
    from lbm_b200 import init as I

    mask = I.cylinder_mask(W, H, CYL[0], CYL[1], CYL[2], value=I.OBSTACLE)
    f0 = I.channel_state(W, H, u0=0.0, noise=1e-4, seed=0)
    return mask, f0


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.start = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()  # the timed region starts once the sampler is producing
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.start = len(self.lines)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples taken inside the timed region; the last one before it when the
        # region was shorter than the sampling period
        lines = self.lines[self.start:] or self.lines[-1:]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(seconds: float = 12.0):
    """The oracle's OpenMP FP32 port of the per-cell update (lbm_core4.cu:120-211
    with this workload's Cs and rates) on every host core, time-bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    lib = O.lib(cpu_baseline=True)
    cores = int(lib.orc_num_threads())
    mask, f0 = workload()
    a, b = f0.copy(), f0.copy()
    mac = tuple(np.zeros((H, W), np.float32) for _ in range(3))
    O.core4_step(mask, a, b, mac, tau_inv=1.0 / TAU, u_in=U_IN, cs=CS, cpu_baseline=True)
    n, t0 = 0, time.perf_counter()
    while True:
        O.core4_step(mask, a, b, mac, tau_inv=1.0 / TAU, u_in=U_IN, cs=CS, cpu_baseline=True)
        a, b = b, a
        n += 1
        dt = time.perf_counter() - t0
        if (dt >= seconds and n >= 5) or n >= 2000:
            break
    return {"value": round(W * H * n / dt / 1e6, 2), "unit": "MLUPS", "cores": cores, "kind": "port",
            "sample": f"{n} steps of the full {W}x{H} workload ({dt:.1f} s, FP32, OpenMP)"}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--T", type=int, default=2,
                    help="steps fused per launch (1: streaming kernel; 2, 4, 6: register wavefront; 3-8: "
                         "shared-memory wavefront)")
    ap.add_argument("--frame", type=int, default=50,
                    help="physical steps per bench step (50: one display frame of the reference's driver)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--storage", choices=["f32", "f16", "bf16"], default="f32",
                    help="population storage of the cylinder workload (16-bit: deviations f - w)")
    ap.add_argument("--workload", choices=["cylinder", "batch", "dropins", "c2", "c3", "c4", "like-reference"],
                    default="cylinder")
    ap.add_argument("--c2-steps", type=int, default=50000, help="c2: physical steps")
    ap.add_argument("--c2-out", default=None, help="c2: CSV file for the drag / lift series")
    ap.add_argument("--c3-marks", default=None, help="c3: comma-separated checkpoints (default 1000,10000,50000)")
    ap.add_argument("--c3-out", default=None, help="c3: also write the result line to this JSON file")
    ap.add_argument("--c4-n", type=int, default=1024, help="c4: coarse grid (the judge is 4x finer)")
    ap.add_argument("--c4-steps", type=int, default=20000, help="c4: coarse steps")
    ap.add_argument("--c4-epochs", type=int, default=30, help="c4: training epochs")
    ap.add_argument("--c4-nu", type=float, default=5e-4, help="c4: coarse-grid viscosity (the judge runs at 4x)")
    ap.add_argument("--c4-out", default=None, help="c4: also write the result line to this JSON file")
    ap.add_argument("--decomp", choices=["auto", "slab", "replicas"], default="auto",
                    help="several GPUs: slab = one channel of (4096 N) x 1024 split in x-slabs of 4096 columns per "
                         "rank with the halo exchange overlapped with the interior (weak scaling; the default for "
                         "N > 1); replicas = N independent copies of the 4096 x 1024 workload")
    ap.add_argument("--inplace", action="store_true",
                    help="one state buffer: lbm_run_inplace (AA pattern, two one-step kernels per pair of steps)")
    ap.add_argument("--closure", choices=["smag", "mlp", "mlp_silu"], default="smag",
                    help="mlp: the learned closure (random-initialised weights of the 5-32-32-1 ReLU network, "
                         "no reference clamps) in place of Smagorinsky; mlp_silu: the same with SiLU")
    args = ap.parse_args()

    rank, world, local = dist_env()
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.impl == "reference":
        if rank != 0:
            barrier()
            if world > 1:
                dist.destroy_process_group()
            return
        line = run_dropins(args, torch, True) if args.workload == "dropins" else run_reference(args, torch)
        print(json.dumps(line), flush=True)
        if world > 1:
            barrier()
            dist.destroy_process_group()
        return

    import lbm_b200 as L
    from lbm_b200 import solver as SV
    from lbm_b200.solver import Solver

    if args.workload in ("batch", "dropins", "c2", "c3", "c4", "like-reference"):
        if args.workload == "batch":
            line = run_batch(args, torch, rank, world, barrier, max_over_ranks)
        elif args.workload == "c2":
            line = run_c2(args, torch)
        elif args.workload == "like-reference":
            line = run_like_reference(args, torch)
        elif args.workload == "c3":
            line = run_c3(args, torch)
        elif args.workload == "c4":
            line = run_c4(args, torch)
        else:
            line = run_dropins(args, torch, False)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            barrier()
            dist.destroy_process_group()
        return

    decomp = args.decomp if args.decomp != "auto" else ("slab" if world > 1 else "replicas")
    if decomp == "slab" and args.workload == "cylinder" and not args.inplace and args.closure == "smag":
        line = run_slab(args, torch, rank, world, barrier, max_over_ranks)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            barrier()
            dist.destroy_process_group()
        return

    storage = {"f32": SV.STORE_F32, "f16": SV.STORE_F16DEV, "bf16": SV.STORE_BF16DEV}[args.storage]
    b_alg = B_ALG if storage == SV.STORE_F32 else B_ALG / 2
    mask_np, f0_np = workload()
    mask = torch.from_numpy(mask_np).cuda()
    extra = {}
    if args.closure in ("mlp", "mlp_silu"):
        from lbm_b200.closure import Mlp

        net = Mlp(seed=0, in_scale=np.array([1e3, 1e3, 1e3, 1e3, 1e2], np.float32), out_scale=1e-4,
                  act="silu" if args.closure == "mlp_silu" else "relu")
        extra = dict(closure=net.closure, mlp=net.packed().data_ptr(), ref_clamps=0)
    S = Solver(W, H, cs_smag=CS, u_in=U_IN, s_nu=1.0 / TAU, storage=storage, **extra)
    f_a = torch.empty((9, H, W), dtype=S.dtype, device="cuda")
    SV.convert_state(torch.from_numpy(f0_np).cuda(), SV.STORE_F32, f_a, storage)
    f_b = f_a if args.inplace else f_a.clone()
    T = 1 if args.inplace else args.T
    if args.inplace and args.frame % 2:
        raise SystemExit("--inplace needs an even --frame")
    n_launch = (args.frame + T - 1) // T
    stream = torch.cuda.current_stream()
    st = {"a": f_a, "b": f_b}

    def frame():
        if args.inplace:
            S.run_inplace(st["a"], mask, args.frame)
            return
        for _ in range(n_launch):
            which = S.run(st["a"], st["b"], mask, T, T)
            if which:
                st["a"], st["b"] = st["b"], st["a"]

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("bench timed region")
        e0.record(stream)
        for _ in range(args.steps):
            frame()
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1))
    phys = args.steps * n_launch * T
    mlups_total = W * H * phys * world / (ms * 1e3)
    ms_per_step = ms / args.steps
    launch_ms = ms / (args.steps * n_launch)

    # End to end through the public API with host buffers, one display frame of
    # the reference's driver per step (lbm_mine2.py:88-95): the frame's steps,
    # u, v, rho written by the last launch, the vorticity colour map
    # (lbm_visualize, scale 50) and the RGBA frame read back to pinned host
    # memory; the solid mask is the step's input, uploaded from pinned host
    # memory every frame.  The populations stay resident, as in the driver.
    # Uploads, frames and colour map + read-backs run on three streams with two
    # mask, macro and image buffers, so frame i+1 computes while frame i's image is
    # drawn and copied out.
    host_m = [torch.from_numpy(mask_np).pin_memory() for _ in range(2)]
    dev_m = [torch.empty_like(mask) for _ in range(2)]
    host_img = [torch.empty((H, W, 4), dtype=torch.uint8).pin_memory() for _ in range(2)]
    dev_img = [torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda") for _ in range(2)]
    dev_mac = [[torch.empty((H, W), dtype=torch.float32, device="cuda") for _ in range(3)] for _ in range(2)]
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    ev_up = [torch.cuda.Event() for _ in range(2)]
    ev_comp = [torch.cuda.Event() for _ in range(2)]
    ev_down = [torch.cuda.Event() for _ in range(2)]
    # as many frames as the device-timed region: the last frame's read-back, which
    # no later frame overlaps, is one of K
    e2e_steps = max(3, args.steps)

    def e2e_step(i):
        j = i & 1
        with torch.cuda.stream(up):
            up.wait_event(ev_down[j])  # frame i-2's colour map has finished reading this mask buffer
            dev_m[j].copy_(host_m[j], non_blocking=True)
            ev_up[j].record(up)
        stream.wait_event(ev_up[j])
        stream.wait_event(ev_down[j])  # frame i-2's u, v, rho and image are done with
        mac = dev_mac[j]
        for li in range(0 if args.inplace else n_launch):
            last = li == n_launch - 1
            which = S.run(st["a"], st["b"], dev_m[j], T, T, *(mac if last else (None, None, None)), stream=stream)
            if which:
                st["a"], st["b"] = st["b"], st["a"]
        if args.inplace:
            S.run_inplace(st["a"], dev_m[j], args.frame, *mac, stream=stream)
        ev_comp[j].record(stream)
        with torch.cuda.stream(down):  # colour map and read-back overlap the next frame's steps
            down.wait_event(ev_comp[j])
            L.visualize(*mac, dev_img[j], dev_m[j], W, H, 50.0, stream=down)
            host_img[j].copy_(dev_img[j], non_blocking=True)
            ev_down[j].record(down)

    for j in range(2):  # every event recorded once before the first wait on it
        ev_comp[j].record(stream)
        ev_down[j].record(stream)
    e2e_step(0)
    e2e_step(1)
    torch.cuda.synchronize()
    barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("bench e2e region")
    e2.record(stream)
    for i in range(e2e_steps):
        e2e_step(i)
    for j in range(2):
        stream.wait_event(ev_down[j])
    e3.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    e2e_ms = max_over_ranks(e2.elapsed_time(e3))
    e2e_mlups = W * H * e2e_steps * n_launch * T * world / (e2e_ms * 1e3)
    h2d = host_m[0].numel() * host_m[0].element_size()
    d2h = host_img[0].numel() * host_img[0].element_size()
    if not bool((host_img[(e2e_steps - 1) & 1][1:-1, 1:-1, 3] == 255).all()):  # border cells stay unwritten
        raise RuntimeError("the read-back frame is not a complete RGBA image")

    flags = L.solver.device_error_flags(clear=True)
    if rank == 0:
        peak, peak_src = hbm_peak()
        achieved = b_alg * W * H * T / (launch_ms * 1e-3) / 1e9
        traffic = None
        kname = "stream_kernel" if T == 1 else ("rwave_kernel" if T in (2, 4, 6) else "wave_kernel")
        if args.inplace:
            kname = "inplace_kernel"
        if args.closure == "mlp":
            kname = "rwave_kernel_mlp"
        suffix = "" if args.storage == "f32" else "_" + args.storage
        tfile = os.path.join(ROOT, "profiles", f"{kname}_T{T}_{W}x{H}{suffix}_traffic.json")
        if os.path.exists(tfile):
            try:
                traffic = json.load(open(tfile))["dram_bytes_per_launch"]
            except Exception:
                traffic = None
        # DRAM bytes one launch really moves (ncu capture in profiles/), against
        # the algorithmic bytes; temporal blocking makes the effective figure
        # exceed the copy bandwidth while the real traffic stays below it.
        dram = None
        if traffic:
            dram = {"bytes_per_lup": round(traffic / (W * H * T), 2),
                    "gbs": round(traffic / (launch_ms * 1e-3) / 1e9, 1),
                    "frac_of_peak": round(traffic / (launch_ms * 1e-3) / 1e9 / peak, 4)}
        line = {
            "metric": "MLUPS", "value": round(mlups_total, 1), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"cylinder channel {W}x{H} D2Q9 MRT+Smagorinsky Cs={CS}, Zou-He u={U_IN}, "
                                   f"D={CYL[2]} at ({CYL[0]},{CYL[1]}), nu={NU}, T={T} steps per launch",
                       "storage": args.storage, "closure": args.closure,
                       "W": W, "H": H, "T": T, "physical_steps_per_step": n_launch * T,
                       "state_buffers": 1 if args.inplace else 2,
                       "l2": "inputs larger than L2 (" + ("one 151 MB population buffer" if args.inplace and
                                                            storage == SV.STORE_F32 else
                                                            "two 151 MB population buffers") + ")",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "e2e": {"value": round(e2e_mlups, 1), "unit": "MLUPS", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": f"{kname} (MRT+Smagorinsky, {T} step(s) per launch)",
                         "dram": dram,
                         "note": f"achieved = {b_alg:g} B per lattice update x W*H*T / launch time (effective "
                                 f"bytes; T steps per launch move about 1/T of them); peak {peak_src}"},
            "gpu_launches": args.steps * n_launch,
            "clocks": clk.summary(),
            "device_error_flags": flags,
        }
        if not args.no_cpu_baseline and world == 1 and storage == SV.STORE_F32:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if world > 1:
        barrier()
        dist.destroy_process_group()


def run_slab(args, torch, rank, world, barrier, max_over_ranks):
    """x-slab decomposition over the ranks (weak scaling): one channel of
    (4096 N) x 1024 with the bench physics (MRT + Smagorinsky Cs = 0.1, clamps,
    ramped Zou-He inlet on rank 0, outflow on the last rank, walls in y) and the
    D = 128 cylinder at (1024, 512); rank r owns columns [4096 r, 4096 (r + 1))
    plus T halo columns per side with a neighbour.  Every launch of T steps
    computes the edge columns first, sends them (NCCL send/recv of one packed
    buffer per neighbour) while the interior computes on a second stream, and
    unpacks the received halos.  value = all ranks' cells x steps / the slowest
    rank's time.  e2e: every step also uploads the rank's mask slab from pinned
    host memory and reads back the all-reduced FP64 mass and momentum."""
    from lbm_b200 import init as I
    from lbm_b200 import solver as SV
    from lbm_b200.slab import SlabSolver

    storage = {"f32": SV.STORE_F32, "f16": SV.STORE_F16DEV, "bf16": SV.STORE_BF16DEV}[args.storage]
    Wg, T = W * world, args.T
    mask_g = torch.from_numpy(I.cylinder_mask(Wg, H, CYL[0], CYL[1], CYL[2], value=I.OBSTACLE))
    # 16 halo columns keep every local width a multiple of 16 (TMA rows of the mask)
    S = SlabSolver(Wg, H, mask_g, T=T, halo=16, cs_smag=CS, u_in=U_IN, s_nu=1.0 / TAU, storage=storage)
    lay = S.lay
    f_loc = torch.from_numpy(I.channel_state(lay.width, H, u0=0.0, noise=1e-4, seed=rank)).cuda()
    if storage != SV.STORE_F32:
        tmp = torch.empty((9, H, lay.width), dtype=S.dtype, device="cuda")
        SV.convert_state(f_loc, SV.STORE_F32, tmp, storage)
        f_loc = tmp
    S.set_local_state(f_loc)
    barrier()  # every rank's communicator is up before the first send / receive
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        S.run(args.frame)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            S.run(args.frame)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    cells = Wg * H
    mlups = cells * args.frame * args.steps / (ms * 1e3)
    # e2e: host mask upload + the frame + the global FP64 diagnostics read back
    host_mask = S.mask.cpu().pin_memory()
    dev_mask = torch.empty_like(S.mask)
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        dev_mask.copy_(host_mask, non_blocking=True)
        S.mask = dev_mask
        S.run(args.frame)
        S.diag().cpu()
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3))
    n_launch = (args.frame + T - 1) // T
    left, right = S._neighbours()
    per_launch = (3 + (left is not None) + (right is not None)) if S.overlap else 1
    launches = torch.tensor([float(per_launch * n_launch * args.steps)], device="cuda")
    if world > 1:
        torch.distributed.all_reduce(launches)
    halo_bytes = 2 * 9 * H * S.halo * torch.empty((), dtype=S.dtype).element_size()
    own = (lay.x1 - lay.x0) * H
    b_alg = B_ALG if storage == SV.STORE_F32 else B_ALG / 2
    achieved = b_alg * own * args.frame * args.steps / (ms * 1e-3) / 1e9
    peak, how = hbm_peak()
    return {"metric": "MLUPS", "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": {"f32": "f32"}.get(args.storage, args.storage + "-dev"),
            "data": "synthetic",
            "config": {"workload": f"cylinder channel {Wg}x{H} D2Q9 MRT+Smagorinsky Cs={CS}, Zou-He u={U_IN}, "
                                   f"D={CYL[2]} at ({CYL[0]},{CYL[1]}), nu={NU}, x-slabs of {W} columns per rank, "
                                   f"T={T} steps per launch",
                       "storage": args.storage, "W": Wg, "H": H, "T": T, "physical_steps_per_step": args.frame,
                       "parallelism": f"x-slab decomposition over {world} GPU(s), one process per GPU, NCCL "
                                      f"send/recv of {S.halo} halo columns per side per launch, overlapped with "
                                      f"the interior" if S.overlap else "x-slab decomposition (no neighbours)",
                       "halo_bytes_per_side_per_launch": halo_bytes // 2,
                       "l2": "inputs larger than L2 (two 151 MB population buffers per rank)"},
            "e2e": {"value": round(cells * args.frame * args.steps / (ms_e2e * 1e3), 1), "unit": "MLUPS",
                    "h2d_bytes_per_step": int(S.mask.numel()), "d2h_bytes_per_step": 24},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None,
                         "note": f"per rank: {int(b_alg)} B per lattice update x owned cells x steps / the slowest "
                                 f"rank's time (effective bytes); peak {how}; no ncu capture of a multi-rank run"},
            "gpu_launches": int(launches.item()), "clocks": clk.summary()}


def run_batch(args, torch, rank, world, barrier, max_over_ranks):
    """256 independent MRT+Smagorinsky channel domains, Nx, Ny ~ U[64, 1024], 1-4
    discs of radius 4-32, inlet u ~ U[0.02, 0.08], FP16-deviation storage, one
    launch per T steps for every domain (autotuned T and rows per work item),
    against one launch per domain."""
    from lbm_b200 import init as I
    from lbm_b200 import solver as SV
    from lbm_b200.batch import Batch

    rng = np.random.default_rng(1234 + rank)
    doms = []
    cells = 0
    for i in range(256):
        w, h = int(rng.integers(64, 1025)), int(rng.integers(64, 1025))
        m = I.random_discs_mask(w, h, int(rng.integers(1, 5)), 4.0, min(32.0, h / 4), 5000 + i)
        pitch = (w + 15) // 16 * 16
        mk = torch.zeros((h, pitch), dtype=torch.uint8, device="cuda")
        mk[:, :w] = torch.from_numpy(m).cuda()
        fa = torch.zeros((9, h, pitch), dtype=torch.float16, device="cuda")  # deviation 0: fluid at rest
        doms.append(dict(W=w, H=h, pitch=pitch, mask_pitch=pitch, f_a=fa, f_b=fa.clone(), mask=mk,
                         u_in=float(rng.uniform(0.02, 0.08))))
        cells += w * h
    B = Batch(doms, storage=SV.STORE_F16DEV, cs_smag=CS, s_nu=1.0 / TAU)
    T, chunk = B.autotune()
    steps_per = 40
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        B.run(steps_per, T)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            B.run(steps_per, T)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1))
    mlups = cells * steps_per * args.steps * world / (ms * 1e3)
    B.run_separate(steps_per, T)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(max(1, args.steps // 3)):
        B.run_separate(steps_per, T)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_sep = max_over_ranks(e0.elapsed_time(e1))
    mlups_sep = cells * steps_per * max(1, args.steps // 3) * world / (ms_sep * 1e3)
    # the same with one item height for every size class (the tuned one of the largest)
    _, rows = B.tiles()
    B.set_tiles(T, [chunk] * len(rows))
    B.run(steps_per, T)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        B.run(steps_per, T)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_uni = max_over_ranks(e0.elapsed_time(e1))
    B.set_tiles(T, rows)
    return {
        "metric": "aggregate MLUPS", "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16-deviation storage, f32 math",
        "data": "synthetic",
        "config": {"workload": "batch of 256 MRT+Smagorinsky channel domains, Nx,Ny~U[64,1024], 1-4 discs r 4-32, "
                               "u_in~U[0.02,0.08], FP16 storage, one launch per T steps for all domains, autotuned",
                   "cells": cells, "T": T, "rows_per_item": chunk, "physical_steps_per_step": steps_per,
                   "rows_per_item_by_size_class": rows,
                   "size_classes": "cells < 2^17, < 2^19, larger"},
        "uniform_rows_mlups": round(cells * steps_per * args.steps * world / (ms_uni * 1e3), 1),
        "separate_launches_mlups": round(mlups_sep, 1),
        "speedup_vs_separate": round(mlups / mlups_sep, 3),
        "gpu_launches": args.steps * ((steps_per + T - 1) // T),
        "clocks": clk.summary(),
    }


def run_c2(args, torch):
    """The cylinder workload (4096 x 1024, D = 128, Re = 10 000, MRT + Smagorinsky
    Cs = 0.1, Zou-He u = 0.05 with the ramp) run for --c2-steps steps at T = 2,
    with drag and lift (lbm_forces_fp64, momentum exchange on the cylinder)
    sampled every 100 steps into device memory.  Reports the drag and lift
    coefficients C = F / (0.5 rho u^2 D) over the second half of the run, the
    Strouhal number f D / u of the lift's dominant frequency there, and the
    MLUPS of the whole run including the force reductions; --c2-out writes the
    series (step, Fx, Fy, Cd, Cl) as CSV."""
    from lbm_b200 import solver as SV

    mask_np, f0_np = workload()
    mask = torch.from_numpy(mask_np).cuda()
    S = SV.Solver(W, H, cs_smag=CS, u_in=U_IN, s_nu=1.0 / TAU)
    a = torch.from_numpy(f0_np).cuda()
    b = a.clone()
    every, T = 100, 2
    n = max(2, args.c2_steps // every)
    series = torch.zeros((n, 2), dtype=torch.float64, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(n):
        if S.run(a, b, mask, every, T):
            a, b = b, a
        S.forces(a, mask, out=series[i])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    F = series.cpu().numpy()
    D = float(CYL[2])
    q = 0.5 * 1.0 * U_IN * U_IN * D
    cd, cl = F[:, 0] / q, F[:, 1] / q
    steps = (np.arange(n) + 1) * every
    half = slice(n // 2, n)
    x = cl[half] - cl[half].mean()
    spec = np.abs(np.fft.rfft(x * np.hanning(x.size))) ** 2
    freq = np.fft.rfftfreq(x.size, d=float(every))  # per step
    k = 1 + int(np.argmax(spec[1:]))
    st = float(freq[k] * D / U_IN)
    # peak refined by a parabola through the log power of the three bins around it
    la, lb, lc = np.log(spec[k - 1] + 1e-300), np.log(spec[k] + 1e-300), np.log(spec[min(k + 1, spec.size - 1)] + 1e-300)
    den = la - 2.0 * lb + lc
    st_fit = float((k + (0.5 * (la - lc) / den if den != 0 else 0.0)) * freq[1] * D / U_IN)
    if args.c2_out:
        np.savetxt(args.c2_out, np.column_stack([steps, F[:, 0], F[:, 1], cd, cl]), delimiter=",",
                   header="step,Fx,Fy,Cd,Cl", comments="")
    return {"metric": "MLUPS", "value": round(W * H * n * every / (ms * 1e3), 1), "unit": "MLUPS", "n_gpus": 1,
            "steps": n * every, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"cylinder channel {W}x{H} D2Q9 MRT+Smagorinsky Cs={CS}, Zou-He u={U_IN} "
                                   f"(ramp), D={CYL[2]} at ({CYL[0]},{CYL[1]}), Re={U_IN * D / NU:.0f}, T={T}, "
                                   f"forces every {every} steps"},
            "drag_lift": {"cd_mean_second_half": round(float(cd[half].mean()), 4),
                          "cd_std_second_half": round(float(cd[half].std()), 4),
                          "cl_rms_second_half": round(float(np.sqrt(np.mean(x ** 2))), 4),
                          "strouhal_second_half": round(st, 4),
                          "strouhal_resolution": round(float(freq[1] * D / U_IN), 4),
                          "strouhal_refined_second_half": round(st_fit, 4),
                          "finite": bool(np.isfinite(F).all()),
                          "cd_last": round(float(cd[-1]), 4), "cl_last": round(float(cl[-1]), 4)}}


def run_c3(args, torch):
    """8192 x 2048 channel past a D = 256 cylinder at (2048, 1024), Re = 20 000
    (u = 0.05, nu = 6.4e-4, Cs = 0.1, the reference's clamps), from rest with
    u_y noise +-1e-4 (seed 0).  FP64 storage and arithmetic (one step per
    launch) is the judge; FP32, FP16-deviation and BF16-deviation storage run
    at T = 2.  Reports each format's velocity relative L2 against the FP64 run
    over the fluid cells at the checkpoints (1k, 10k, 50k steps), and MLUPS."""
    from lbm_b200 import init as I
    from lbm_b200 import solver as SV

    Wc, Hc = 8192, 2048
    mask = torch.from_numpy(I.cylinder_mask(Wc, Hc, 2048, 1024, 256, value=I.OBSTACLE)).cuda()
    f0 = torch.from_numpy(I.channel_state(Wc, Hc, u0=0.0, noise=1e-4, seed=0)).cuda()
    marks = [int(x) for x in args.c3_marks.split(",")] if args.c3_marks else [1000, 10000, 50000]
    T = 2
    vel, mlups = {}, {}
    formats = (("f64", SV.STORE_F64), ("f32", SV.STORE_F32), ("f16", SV.STORE_F16DEV), ("bf16", SV.STORE_BF16DEV))
    for name, st in formats:
        S = SV.Solver(Wc, Hc, cs_smag=CS, u_in=U_IN, s_nu=1.0 / TAU, storage=st)
        a = S.new_state()
        SV.convert_state(f0, SV.STORE_F32, a, st)
        b = a.clone()
        mac = [torch.empty((Hc, Wc), device="cuda") for _ in range(3)]
        done, vel[name] = 0, []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = 0.0
        for mk in marks:
            e0.record()
            which = S.run(a, b, mask, mk - done, T, *mac)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            if which:
                a, b = b, a
            done = mk
            vel[name].append(torch.stack([mac[0], mac[1]]).cpu())
        mlups[name] = round(Wc * Hc * done / (ms * 1e3), 1)
        del S, a, b
        torch.cuda.empty_cache()
    fl = (mask == 0).cpu()

    def rel(name, judge):
        out = []
        for v, r in zip(vel[name], vel[judge]):
            d = (v - r)[:, fl].double()
            out.append(float(d.norm() / r[:, fl].double().norm()))
        return out

    err64 = {name: rel(name, "f64") for name in ("f32", "f16", "bf16")}
    err32 = {name: rel(name, "f32") for name in ("f16", "bf16")}
    line = {"metric": "velocity rel. L2 vs FP64", "value": err64["f16"][0], "unit": "relative L2", "n_gpus": 1,
            "steps": marks[-1], "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f16-deviation storage, f32 math (value: FP16 at the first checkpoint)", "data": "synthetic",
            "config": {"workload": f"cylinder channel {Wc}x{Hc}, D=256 at (2048,1024), Re=20000, Cs={CS}, "
                                   f"u={U_IN}, clamps, T={T} (FP64: one step per launch)", "checkpoints": marks},
            "velocity_rel_l2_vs_f64": err64, "velocity_rel_l2_vs_f32": err32, "mlups_by_storage": mlups}
    if args.c3_out:
        with open(args.c3_out, "w") as fh:
            json.dump(line, fh, indent=1)
    return line


def run_c4(args, torch):
    """Decaying 2-D turbulence on a periodic 1024^2 grid against a 4096^2 judge
    (4x finer run of the same solver, same flow in lattice units, box-filtered):
    random-phase initial condition E(k) ~ k^4 exp(-2 (k/8)^2), u_rms = 0.1 c_s,
    nu = 5e-4 on the coarse grid (2e-3 on the judge's), MRT ghost rates
    s_e = 1.64, s_eps = 1.54, s_q = 1.9 on both (with all three at 1.1 this flow
    goes unstable on the large grids, in FP64 as in FP32: its peak speed reaches
    Mach 0.38), 20 000 coarse steps, snapshots every 1000.
    Two closure networks are trained on the GPU on the filtered snapshots of a
    judge run from another seed (1): the configured one (SiLU hidden layers,
    "mlp_silu") and the ReLU one of the fast kernel ("mlp"); the coarse runs (no
    closure, Smagorinsky Cs = 0.1, both networks; FP32 and FP16 storage) start
    from the filtered initial state of seed 0 and are compared with that seed's
    judge."""
    from lbm_b200 import closure as CL
    from lbm_b200 import solver as SV

    N, steps, every = args.c4_n, args.c4_steps, max(1, args.c4_steps // 20)
    rates = (1.64, 1.54, 1.9)
    kw = dict(factor=4, k0=8.0, nu=args.c4_nu, n_steps=steps, snap_every=every, rates=rates)
    t0 = time.time()
    Jt = CL.filtered_judge(N, seed=1, **kw)
    J = CL.filtered_judge(N, seed=0, **kw)
    t_judge = time.time() - t0
    ns = len(Jt["data"])
    train, test = list(range(1, ns - 2, 2)), list(range(ns - 2, ns))
    net, mse = CL.a_priori(Jt, train, test, epochs=args.c4_epochs, act="relu")
    net_silu, mse_silu = CL.a_priori(Jt, train, test, epochs=args.c4_epochs, act="silu")
    mse["mlp_silu"] = mse_silu["mlp"]
    nets = {"mlp": net, "mlp_silu": net_silu}

    def clean(v):
        return [None if not np.isfinite(x) else round(float(x), 5) for x in v]

    res, mlups = {}, {}
    for sname, st in (("f32", SV.STORE_F32), ("f16", SV.STORE_F16DEV)):
        tm = {}
        r = CL.compare_closures(J, nets, cs=0.1, storage=st, timings=tm, spectrum_floor=1e-8)
        for name, (l2, spec) in r.items():
            res[f"{name}_{sname}"] = {"velocity_rel_l2": clean(l2), "log_spectrum_l2": clean(spec)}
            t = tm[name]
            mlups[f"{name}_{sname}"] = round(t["cells"] * t["steps"] / (t["ms"] * 1e3), 1)

    def first_over(v, lim=0.01):  # first snapshot step whose error exceeds lim
        for k, x in enumerate(v):
            if x is None or x > lim:
                return k * every
        return None

    for v in res.values():
        v["first_step_over_1pct"] = first_over(v["velocity_rel_l2"])
    ft = J["fine_timing"]
    line = {"metric": "velocity rel. L2 vs filtered judge", "value": res["mlp_silu_f16"]["velocity_rel_l2"][-1],
            "unit": "relative L2", "n_gpus": 1, "steps": steps, "warmup": 0, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 math; f32 or f16-deviation storage",
            "data": "synthetic",
            "config": {"workload": f"decaying periodic turbulence {N}^2, judge {4 * N}^2 filtered 4x, k0=8, "
                                   f"u_rms=0.1 c_s, nu={kw['nu']}, MRT (s_e, s_eps, s_q) = {rates}, T=2, "
                                   f"snapshots every {every} steps",
                       "log_spectrum_l2": "over the shells where the judge's energy is >= 1e-8 of its peak",
                       "train_seed": 1, "eval_seed": 0, "epochs": args.c4_epochs,
                       "a_priori_train_snapshots": train, "a_priori_test_snapshots": test},
            "a_priori_mse_nu_t": mse, "closures": res,
            "mlups_periodic_slab_run": mlups,
            "judge_mlups": round(ft["cells"] * ft["steps"] / (ft["ms"] * 1e3), 1),
            "wall_s": {"judges": round(t_judge, 1), "total": round(time.time() - t0, 1)}}
    line["config"]["value"] = "the configured SiLU network, FP16 storage, at the last snapshot"
    if args.c4_out:
        with open(args.c4_out, "w") as fh:
            json.dump(line, fh, indent=1)
    return line


def run_dropins(args, torch, ref):
    """Drop-in kernels (ours or, with ref, the reference's compiled from source)
    on a channel with a solid cylinder, about 100 physical steps per size."""
    from lbm_b200 import init as I

    P, I_, F = C.c_void_p, C.c_int, C.c_float
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    libs = {}
    if ref:
        for name in ("core4", "smemaa", "policy", "endfused"):
            path = os.path.join(ROOT, "oracle", "_ref", f"libref_{name}.so")
            if not os.path.exists(path):
                return {"impl": "reference", "unavailable": f"oracle/_ref/libref_{name}.so was not built"}
            libs[name] = C.CDLL(path)
        libs["core4"].ref_core4_step.argtypes = [P] * 6 + [I_, I_, F, F, F, P]
        libs["smemaa"].ref_smemaa_step.argtypes = [P] * 6 + [I_, I_, F, F, P]
        for name in ("policy", "endfused"):
            libs[name].ref_blocked_step.argtypes = [P] * 3 + [I_, I_, F, F, P]
    else:
        import lbm_b200 as L
        from lbm_b200 import solver as SV
    res = {}
    for (w, h) in ((2048, 512), (4096, 1024)):
        m = I.cylinder_mask(w, h, w // 4, h // 2, h // 8, value=I.SOLID)
        f0 = I.channel_state(w, h, u0=0.0, noise=1e-4, seed=0)
        mask = torch.from_numpy(m).cuda()
        st = {"a": torch.from_numpy(f0).cuda()}
        st["b"] = st["a"].clone()
        mac = [torch.zeros((h, w), dtype=torch.float32, device="cuda") for _ in range(3)]
        if ref:
            kern = [("smemaa_T4", int(libs["smemaa"].ref_T()), lambda a, b: libs["smemaa"].ref_smemaa_step(
                        ptr(mask), ptr(a), ptr(b), *[ptr(t) for t in mac], w, h, 1.7, 0.1, sp)),
                    ("policy_T6", int(libs["policy"].ref_T()), lambda a, b: libs["policy"].ref_blocked_step(
                        ptr(mask), ptr(a), ptr(b), w, h, 1.7, 0.1, sp)),
                    ("endfused_T6", int(libs["endfused"].ref_T()), lambda a, b: libs["endfused"].ref_blocked_step(
                        ptr(mask), ptr(a), ptr(b), w, h, 1.7, 0.1, sp)),
                    ("core4_T1", 1, lambda a, b: libs["core4"].ref_core4_step(
                        ptr(mask), ptr(a), ptr(b), *[ptr(t) for t in mac], w, h, 1.7, 0.1, 1.7, sp))]
        else:
            S = SV.Solver(w, h, collision=SV.COLL_BGK, closure=SV.CLOSURE_NONE, ref_clamps=0, s_nu=1.7, u_in=0.1)
            kern = [("smemaa_T4", 4, lambda a, b: L.smemaa_step(mask, a, b, *mac, w, h, 1.7, 0.1, T=4)),
                    ("endfused_T6", 6, lambda a, b: L.blocked_step(mask, a, b, w, h, 1.7, 0.1, T=6)),
                    ("core4_T1", 1, lambda a, b: L.core4_step(mask, a, b, *mac, w, h, 1.7, 0.1)),
                    ("general_bgk_T2", 2, lambda a, b: S.run(a, b, mask, 2, 2)),
                    ("general_bgk_T4", 4, lambda a, b: S.run(a, b, mask, 4, 4))]
        for name, T, fn in kern:
            n = max(1, 100 // T)

            def go():
                for _ in range(n):
                    rc = fn(st["a"], st["b"])
                    if ref and rc:
                        raise RuntimeError(f"reference launch failed: {rc}")
                    st["a"], st["b"] = st["b"], st["a"]

            for _ in range(max(1, args.warmup)):
                go()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                go()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            res[f"{name}_{w}x{h}"] = round(w * h * T * n * args.steps / (ms * 1e3), 1)
    line = {"metric": "MLUPS", "value": res["smemaa_T4_2048x512"], "unit": "MLUPS", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "drop-in kernels, BGK tau_inv 1.7, u_in 0.1, channel with a solid cylinder "
                                   "(D = H/4 at (W/4, H/2)), about 100 physical steps per bench step"},
            "results": res}
    if ref:
        line["impl"] = "reference"
    return line


def run_like_reference(args, torch):
    """The reference arm's configuration run through this repository's drop-in
    entry points, next to the reference kernel in the same process: the bench
    cylinder with the reference's compile-time constants (Cs = 0.20, s_e = s_eps =
    s_q = 1.1, lbm_core4.cu:6,123), tau_inv = 1/tau, u_in, the same mask and
    initial state, and u, v, rho written as often as the reference writes them.
      core4_step_T1      lbm_core4_step once per step (u, v, rho every step, as the
                         reference kernel: the like-for-like line);
      core4_run_T2_each  lbm_core4_run of 2 steps per call (u, v, rho every 2 steps:
                         the fused launch cannot write the intermediate step's);
      core4_run_T2_frame lbm_core4_run over the whole frame (u, v, rho once per frame,
                         like the default line).
    Each is timed with CUDA events over --steps frames of --frame steps."""
    import lbm_b200 as L

    ref = run_reference(args, torch)
    mask_np, f0_np = workload()
    mask = torch.from_numpy(mask_np).cuda()
    st = {"a": torch.from_numpy(f0_np).cuda()}
    st["b"] = st["a"].clone()
    mac = [torch.zeros((H, W), dtype=torch.float32, device="cuda") for _ in range(3)]
    ti = 1.0 / TAU

    def step1():
        for _ in range(args.frame):
            L.core4_step(mask, st["a"], st["b"], *mac, W, H, ti, U_IN)
            st["a"], st["b"] = st["b"], st["a"]

    def each2():
        for _ in range(args.frame // 2):
            if L.core4_run(mask, st["a"], st["b"], *mac, W, H, ti, U_IN, 2, T=2):
                st["a"], st["b"] = st["b"], st["a"]

    def frame2():
        if L.core4_run(mask, st["a"], st["b"], *mac, W, H, ti, U_IN, args.frame, T=2):
            st["a"], st["b"] = st["b"], st["a"]

    res = {}
    for name, fn in (("core4_step_T1", step1), ("core4_run_T2_each", each2), ("core4_run_T2_frame", frame2)):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        res[name] = round(W * H * args.steps * args.frame / (e0.elapsed_time(e1) * 1e3), 1)
    rv = ref.get("value")
    return {"metric": "MLUPS", "value": res["core4_step_T1"], "unit": "MLUPS", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"cylinder channel {W}x{H}, the reference's constants (Cs=0.20, s=1.1), "
                                   f"tau_inv=1/{TAU:.5f}, u_in={U_IN}, through the drop-in entry points",
                       "value": "core4_step_T1: u, v, rho written every step, as the reference"},
            "mlups": res, "reference_same_process": rv,
            "ratio_to_reference": {k: (round(v / rv, 3) if rv else None) for k, v in res.items()},
            "reference_clocks": ref.get("clocks")}


def run_reference(args, torch):
    """fused_lbmkernel of lbm_core4.cu (compiled from source into oracle/_ref)."""
    path = os.path.join(ROOT, "oracle", "_ref", "libref_core4.so")
    if not os.path.exists(path):
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_core4.so was not built"}
    lib = C.CDLL(path)
    P, I_, F = C.c_void_p, C.c_int, C.c_float
    lib.ref_core4_step.argtypes = [P] * 6 + [I_, I_, F, F, F, P]
    mask_np, f0_np = workload()
    mask = torch.from_numpy(mask_np).cuda()
    a = torch.from_numpy(f0_np).cuda()
    b = a.clone()
    mac = [torch.zeros((H, W), dtype=torch.float32, device="cuda") for _ in range(3)]
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    st = {"a": a, "b": b}
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    def frame():
        for _ in range(args.frame):
            rc = lib.ref_core4_step(ptr(mask), ptr(st["a"]), ptr(st["b"]), *[ptr(t) for t in mac], W, H,
                                    1.0 / TAU, U_IN, 1.0 / TAU, sp)
            if rc:
                raise RuntimeError(f"reference launch failed: {rc}")
            st["a"], st["b"] = st["b"], st["a"]

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            frame()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    mlups = W * H * args.steps * args.frame / (ms * 1e3)
    return {
        "impl": "reference", "metric": "MLUPS", "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"cylinder channel {W}x{H} D2Q9 MRT+Smagorinsky (reference constants: Cs=0.20, "
                               f"s=1.1), Zou-He u={U_IN}, T=1 step per launch (lbm_core4.cu)",
                   "W": W, "H": H, "physical_steps_per_step": args.frame},
        "cpu_baseline": {"value": round(mlups, 1), "unit": "MLUPS", "cores": 0, "kind": "reference",
                         "sample": "the reference's own CUDA kernel (oracle/_ref/libref_core4.so) on the GPU; "
                                   "the reference has no CPU implementation of this path"},
        "e2e": {"value": round(mlups, 1), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": args.steps * args.frame,
        "clocks": clk.summary(),
    }


if __name__ == "__main__":
    main()
