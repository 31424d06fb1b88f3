#!/usr/bin/env python
"""Benchmark: askAdam voxel-fits/s on the monoexponential R2* + 3-D TV
workload (128x128x64 ellipsoidal mask, 629,432 voxels, 12 echoes
TE = 2:3.5:40.5 ms, MSE, Adam lr 0.01, 4000 iterations, lambda 1e-3 on R2*).

A step is one full fit of one such volume.  `value` times the fit with the
inputs already resident in device memory; `e2e` times the same call through
the C-ABI with pinned host buffers (host<->device copies inside the timed
region).  With torchrun each rank fits its own volume (independent objects,
no collective): weak scaling.  `--impl reference` times the FP64 CPU
restatement of the reference algorithm (the oracle) on this box's cores.
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
sys.path.insert(0, ROOT)

NITER = 4000
ALG_BYTES_PER_VOXEL_ITER = 100.0   # 12 echoes x 4 B data + (z, m, v) x 2 params read+write + 4 B TV map
# compute per voxel-iteration of the standard R2* + TV step, counted from the kernel source:
# MUFU ops = 12 ex2 (echoes) + 2 x (ex2 + rcp) (sigmoid of each parameter once per iteration: the
# regularised one's serves the map and the next fidelity pass) + 2 x (sqrt + rcp) (Adam);
# FP32 FLOP (FMA = 2) = 12 x 9 (echoes) + 2 x 8 (sigmoid) + 8 (loss / gradient scaling)
# + 24 (TV, 3 axes) + 2 x 13 (Adam)
SFU_OPS_PER_VOXEL_ITER = 20.0
FP32_FLOP_PER_VOXEL_ITER = 182.0
METRIC = "askAdam voxel-fits/s & MCMC samples/s, fused vs plain GPU, equal FP64 error"
WORKLOAD = ("askAdam R2* MSE + 3-D TV (lambda 1e-3 on R2*), 128x128x64 ellipsoid mask (629,432 voxels), "
            "12 echoes TE=2:3.5:40.5 ms, Adam lr 0.01, 4000 iterations")


def bench_config(nvox_total, world, grid="128x128x64", iters=NITER):
    """The config object both arms print (the same workload, the same keys)."""
    return {"workload": WORKLOAD if grid == "128x128x64" and iters == NITER else
            f"askAdam R2* MSE + 3-D TV, grid {grid}, {iters} iterations",
            "global_batch": nvox_total, "seq_len": iters, "parallelism": f"replicas{world}",
            "l2": "GPU: flushed between steps (256 MB write); CPU: the working set exceeds the host caches"}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--no-extra", action="store_true", help="skip the plain-path and MCMC side measurements")
    p.add_argument("--cpu-iters", type=int, default=40, help="iterations of the bounded CPU sample")
    p.add_argument("--iters", type=int, default=NITER, help="askAdam iterations per fit (profiling runs)")
    p.add_argument("--c3-iters", type=int, default=1000, help="iterations of the batched joint R1R2* side run")
    p.add_argument("--c4-iters", type=int, default=100, help="iterations of the NEXI Rician side run")
    p.add_argument("--surf-iters", type=int, default=200, help="iterations of the cortical-surface NEXI side run")
    p.add_argument("--grid", default="128x128x64", help="phantom grid (profiling runs)")
    p.add_argument("--mcmc-steps", type=int, default=200, help="GW steps of the MCMC side measurement")
    p.add_argument("--parity-iters", type=int, default=400, help="epochs of the fused/plain vs FP64 parity leg")
    p.add_argument("--mcmc-cpu-voxels", type=int, default=256, help="voxels of the MCMC CPU baseline sample")
    p.add_argument("--mcmc-summary-steps", type=int, default=200,
                   help="GW steps of the on-device median/iqr/mode run (5000: the full 102 GB posterior in HBM)")
    p.add_argument("--mcmc-cpu-steps", type=int, default=100, help="GW steps of the MCMC CPU baseline sample")
    p.add_argument("--no-parity", action="store_true", help="skip the fused/plain vs FP64 parity leg")
    p.add_argument("--extras", default="", help="comma-separated side runs (default all): " + ",".join(EXTRAS))
    p.add_argument("--path", default="fused", choices=["fused", "plain"],
                   help="askAdam path of the main timed fit (plain: profiling runs of the op-by-op kernels)")
    return p.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "engine" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def workload(seed=1002, grid="128x128x64", iters=NITER):
    from gacelle_b200 import phantoms
    dims = tuple(int(x) for x in grid.split("x"))
    P = phantoms.r2s_tv_volume(seed, dims)
    mask, y, idx, th0, n = P["mask"], P["y"], P["idx"], P["th0"], P["nvox"]
    fitting = {"iteration": iters, "initialLearnRate": 0.01, "decayRate": 0.0, "lossFunction": "mse",
               "tol": 0.0, "convergenceValue": 1e-6, "patienceConvergence": float("inf"),
               "convergenceStepTol": 0.0, "convergenceGradTol": 0.0, "lambda": [1e-3], "regmap": ["R2star"],
               "TVmode": "3D", "voxelSize": [2, 2, 2], "parameterTransform": "sigmoid"}
    return {"mask": mask, "y": y, "idx": idx, "th0": th0, "fitting": fitting, "nvox": n,
            "te": phantoms.R2S_TE, "lb": [0.0, 0.1], "ub": [2.0, 200.0]}


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.rows = []
        self.proc = None
        self.dev = device_index

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel: str):
    """DRAM bytes per launch of the named hot kernel from its committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_r2s_c2_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_launch")
    return None


def host_cpu() -> str:
    """The host's CPU model and logical CPU count (the CPU baselines' cores)."""
    model = "unknown CPU"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return f"{model}, {os.cpu_count()} logical CPUs"


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU legs (oracle): bounded sample of the same workload
# ---------------------------------------------------------------------------
def cpu_sample(W, iters):
    import oracle
    f = dict(W["fitting"])
    from gacelle_b200 import askadam_solver as gxa
    f = gxa.check_set_default_basic(f)
    f["iteration"] = iters
    f["_reg_index"] = [1]
    f["_reg_lambda"] = [1e-3]
    cores = os.cpu_count() or 1
    f["nthreads"] = cores
    vol = oracle.Volume(W["y"].astype(np.float64), dims=W["mask"].shape, grid_index=W["idx"],
                        theta0=W["th0"].astype(np.float64))
    o = oracle.adam_opts(W["lb"], W["ub"], f)
    t0 = time.perf_counter()
    oracle.askadam(oracle.r2s(W["te"]), vol, o, want_min=False, want_history=False)
    dt = time.perf_counter() - t0
    per_iter = dt / (iters + 1)  # init evaluation + iters epochs
    fits_per_s = W["nvox"] / (per_iter * NITER)
    return fits_per_s, cores, dt


def reference_arm(args, world, rank):
    if rank != 0:
        return
    W = workload()
    for _ in range(args.warmup):
        cpu_sample(W, max(2, args.cpu_iters // 4))
    vals, tot = [], 0.0
    for _ in range(args.steps):
        v, cores, dt = cpu_sample(W, args.cpu_iters)
        vals.append(v)
        tot += dt
    value = statistics.median(vals)
    sample = (f"{W['nvox']}-voxel R2*+3-D TV volume, {args.cpu_iters} of {NITER} iterations per step "
              f"on all {cores} host threads, extrapolated to the full {NITER}-iteration fit")
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "voxel-fits/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded phantom, seed 1002)",
            "config": bench_config(W["nvox"] * args.gpus, args.gpus),
            "cpu_baseline": {"value": value, "unit": "voxel-fits/s", "cores": cores, "kind": "port",
                             "sample": sample, "host": host_cpu()},
            "e2e": {"value": value, "unit": "voxel-fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Engine arm
# ---------------------------------------------------------------------------
def engine_arm(args, world, rank, local):
    import torch

    import gacelle_b200
    from gacelle_b200 import _lib, askadam_solver as gxa
    from gacelle_b200.models import _GxModelHandle

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    W = workload(seed=1002 + rank, grid=args.grid, iters=args.iters)
    ctx = gacelle_b200.Context(local)
    # one stream for everything timed: the library's launches, the L2 flush and the CUDA events
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    f = gxa.check_set_default_basic(W["fitting"])
    opts = gxa.build_opts(f, ["M0", "R2star"], W["lb"], W["ub"], args.path)
    model = _GxModelHandle(_lib.MODEL_R2S, te=W["te"])
    n, nm = W["nvox"], 12
    fp = lambda t: C.cast(C.c_void_p(t.data_ptr()), _lib._fp)  # noqa: E731

    # device-resident inputs and outputs
    d_y = torch.from_numpy(W["y"]).to(dev)
    d_idx = torch.from_numpy(W["idx"]).to(dev)
    d_th0 = torch.from_numpy(W["th0"]).to(dev)
    d_out = [torch.empty((2, n), dtype=torch.float32, device=dev) for _ in range(2)]
    hist = np.zeros(args.iters + 1)

    def make_vol(y, idx, th0):
        v = _lib.GxVolume()
        for i in range(3):
            v.dims[i] = W["mask"].shape[i]
        v.nvox = n
        v.grid_index = C.cast(C.c_void_p(idx.data_ptr()), _lib._i32p)
        v.data = fp(y)
        v.theta0 = fp(th0)
        return v

    def make_res(outs):
        r = _lib.GxAskadamResult()
        r.final_theta = fp(outs[0])
        r.min_theta = fp(outs[1])
        r.loss_history = hist.ctypes.data_as(_lib._dp)
        return r

    vol_d = make_vol(d_y, d_idx, d_th0)
    res_d = make_res(d_out)
    L = _lib.lib()

    def step_device():
        _lib.check(L.gx_askadam(ctx.ptr, C.byref(model.s), _lib.MEM_DEVICE, C.byref(vol_d), 1, C.byref(opts),
                                C.byref(res_d)))

    # pinned host inputs and outputs for the end-to-end leg
    h_y = torch.from_numpy(W["y"]).pin_memory()
    h_idx = torch.from_numpy(W["idx"]).pin_memory()
    h_th0 = torch.from_numpy(W["th0"]).pin_memory()
    h_out = [torch.empty((2, n), dtype=torch.float32).pin_memory() for _ in range(2)]
    vol_h = make_vol(h_y, h_idx, h_th0)
    res_h = make_res(h_out)

    def step_host():
        _lib.check(L.gx_askadam(ctx.ptr, C.byref(model.s), _lib.MEM_HOST, C.byref(vol_h), 1, C.byref(opts),
                                C.byref(res_h)))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local).start()
    time.sleep(0.25)
    launches = 0
    main_ms, main_n = 0.0, 0
    times = []
    torch.cuda.synchronize()
    barrier(world)
    for _ in range(args.steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        step_device()
        e.record(stream)
        t = ctx.timing()
        launches += t["kernel_launches"]
        main_ms += t["main_kernel_ms"]
        main_n += t["main_launches"]
        times.append((s, e))
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms_total = sum(s.elapsed_time(e) for s, e in times)
    ms_total = max_over_ranks(ms_total, world)
    ms_step = ms_total / args.steps
    value = world * n * args.steps / (ms_total / 1000.0) * (args.iters / NITER)

    # end to end through the C-ABI with pinned host buffers
    for _ in range(min(args.warmup, 2)):
        step_host()
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = 0.0
    h2d = d2h = 0
    for _ in range(args.steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        step_host()
        e.record(stream)
        e.synchronize()
        e2e_ms += s.elapsed_time(e)
        t = ctx.timing()
        h2d, d2h = t["h2d_bytes"], t["d2h_bytes"]
    e2e_ms = max_over_ranks(e2e_ms, world)
    e2e_value = world * n * args.steps / (e2e_ms / 1000.0) * (args.iters / NITER)

    # parity spot check of the measured fit against the oracle on a voxel subset is done in tests;
    # here only sanity: parameters finite and inside bounds
    th = d_out[0].cpu().numpy()
    assert np.all(np.isfinite(th)) and th[1].min() >= 0.1 and th[1].max() <= 200.0

    # one launch of the hot kernel covers iters / (launches per fit) epochs: all of them for the
    # persistent kernel, one for the per-epoch kernel (GACELLE_B200_TV_KERNEL=step)
    avg_launch_ms = main_ms / max(main_n, 1)
    launches_per_fit = main_n / args.steps
    epochs_per_launch = args.iters / max(launches_per_fit, 1.0)
    persistent = launches_per_fit < args.iters
    vit = n * epochs_per_launch / (avg_launch_ms / 1000.0)   # voxel-iterations/s of the hot kernel
    # The binding roof is the SFU (MUFU) pipe: the kernel keeps its optimiser state on chip and moves
    # 1.5 % of a streaming implementation's bytes through DRAM, so the HBM figure below is a
    # streaming-equivalent rate, not a bound.  SFU peak: 16 MUFU ops/clk/SM x SMs x sampled SM clock
    # (the measured peaks file holds copy bandwidth and GEMM rates only).
    ghz = (clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0) / 1000.0
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    sfu_peak, fp32_peak = 16 * nsm * ghz * 1e9, 2 * 128 * nsm * ghz * 1e9
    sfu_achieved = vit * SFU_OPS_PER_VOXEL_ITER
    hbm_peak, hbm_kind = measured_peaks()
    stream_bytes = ALG_BYTES_PER_VOXEL_ITER * n * epochs_per_launch
    kname = "tv_persistent" if persistent else "tv_step"
    roofline = {"bound": "sfu", "achieved": sfu_achieved / 1e9, "peak": sfu_peak / 1e9, "unit": "G MUFU op/s",
                "frac": sfu_achieved / sfu_peak,
                "peak_kind": "nominal 16 MUFU op/clk/SM x %d SMs x sampled %.3f GHz (no measured SFU peak)" % (nsm, ghz),
                "traffic": profile_traffic(kname),
                "traffic_source": f"ncu capture committed under profiles/ ({kname}_r2s_c2_traffic.json), "
                                  "DRAM bytes read + written per launch; not measured in this run",
                "kernel": ("tv_persistent_kernel<MSE,12> (every epoch of the fit in one cooperative launch: "
                           "forward, loss, adjoint, TV, Adam)") if persistent else
                          "tv_step_kernel<R2S,MSE> (one epoch: forward, loss, adjoint, TV, Adam)",
                "units_per_launch": f"{n} voxels x {epochs_per_launch:.0f} epochs",
                "sfu_ops_per_voxel_iter": SFU_OPS_PER_VOXEL_ITER,
                "epochs_per_launch": epochs_per_launch,
                "avg_launch_ms": avg_launch_ms,
                "voxel_iterations_per_s": vit,
                "fp32": {"flop_per_voxel_iter": FP32_FLOP_PER_VOXEL_ITER,
                         "achieved_tflops": vit * FP32_FLOP_PER_VOXEL_ITER / 1e12,
                         "peak_tflops": fp32_peak / 1e12, "frac": vit * FP32_FLOP_PER_VOXEL_ITER / fp32_peak},
                "hbm_streaming_equivalent": {
                    "bytes_per_voxel_iter": ALG_BYTES_PER_VOXEL_ITER, "bytes_per_launch": stream_bytes,
                    "gbs": stream_bytes / (avg_launch_ms / 1000.0) / 1e9, "peak_gbs": hbm_peak,
                    "peak_kind": hbm_kind,
                    "note": "bytes a streaming (state in HBM) implementation would move; this kernel does not"}}
    line = {"metric": METRIC, "value": value, "unit": "voxel-fits/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom, seed 1002+rank)",
            "config": bench_config(world * n, world, args.grid, args.iters),
            "gpu_launches": launches, "clocks": clk, "roofline": roofline,
            "e2e": {"value": e2e_value, "unit": "voxel-fits/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h}}
    if rank == 0:
        cv, cores, dt = cpu_sample(W, args.cpu_iters)
        line["cpu_baseline"] = {"value": cv, "unit": "voxel-fits/s", "cores": cores, "kind": "port", "host": host_cpu(),
                                "sample": f"{n}-voxel volume, {args.cpu_iters} of {NITER} iterations "
                                          f"({dt:.1f} s on {cores} threads), extrapolated"}
        if not args.no_extra:
            line["extra"] = extras(ctx, W, opts, model, stream, args, ghz, nsm)
        print(json.dumps(line), flush=True)


# MUFU operations per Goodman-Weare proposal on NEXI (lmax 0, 24 shells x 14
# nodes), counted from the kernel source: per node one rsqrt and two
# exponentials; per proposal two logf (stretch factor, acceptance uniform)
MCMC_SFU_PER_PROPOSAL = 24 * 14 * 3 + 2
EXTRAS = ("plain", "parity", "mcmc", "mcmc_summaries", "mcmc_cpu", "c1", "c3", "c4", "surface", "autotune")


def extras(ctx, W, opts, model, stream, args, ghz=1.965, nsm=148):
    """Side measurements, each selectable with --extras: the plain (op-by-op)
    path on the same volume; the fused/plain parity leg; Goodman-Weare MCMC on
    the NEXI model (200k voxels x 64 walkers, 24 shells, 14-node powder
    average, sigma fixed at 0.02) over a bounded number of steps, and its CPU
    baseline; the C1, C3, C4 and cortical-surface configurations."""
    from gacelle_b200 import askadam_solver as gxa
    from gacelle_b200 import mcmc_solver, phantoms
    from gacelle_b200.models import gpuNEXI
    want = set(args.extras.split(",")) if args.extras else set(EXTRAS)
    out = {}
    n = W["nvox"]
    if "plain" in want:
        # the op-by-op (plain) path on the same volume, the full 4000 iterations
        f = gxa.check_set_default_basic(dict(W["fitting"], iteration=NITER))
        solver = gxa.askadam(ctx, "plain")
        o2 = gxa.build_opts(f, ["M0", "R2star"], W["lb"], W["ub"], "plain")
        solver._run(model, W["y"], None, W["th0"], None, None, W["idx"], W["mask"].shape, o2, 12, 2)
        t = solver.last_timing
        out["plain_voxel_fits_per_s"] = n / (t["main_kernel_ms"] / 1000.0)
        out["plain_ms_per_iteration"] = t["main_kernel_ms"] / NITER
        out["plain_iterations_timed"] = NITER
    if "parity" in want and not args.no_parity:
        out.update(parity_leg(ctx, W, model, args.parity_iters))
    if "mcmc" in want:
        nv, steps = 200_000, args.mcmc_steps
        y, gt = phantoms.nexi_volume(nv, 1005, sigma=0.02, rician=False, nx=14)
        b, d = phantoms.nexi_shells()
        m = gpuNEXI(b, d, nx=14)
        m.updateProperty({"solver": "mcmc", "lmax": 0})
        x0 = np.vstack([gt["fa"], gt["Da"], gt["De"], gt["ra"], np.full(nv, 0.02)]).astype(np.float32)
        fit = mcmc_solver.check_set_default_basic({"algorithm": "ensemble", "iteration": steps, "burnin": 0.2,
                                                   "thinning": 10, "Nwalker": 64, "StepSize": 2,
                                                   "modelParams": m.modelParams,
                                                   "lb": list(m.lb[:4]) + [0.02], "ub": list(m.ub[:4]) + [0.02],
                                                   "returnPosterior": False})
        mc = mcmc_solver.mcmc(ctx)
        mask = np.ones((1, nv), bool)
        pars0 = {p: x0[k] for k, p in enumerate(m.modelParams)}
        mc.optimisation(y, mask, None, pars0, fit, m)   # first call of this key: the autotuner's trials
        mc.optimisation(y, mask, None, pars0, fit, m)
        t = mc.last_timing
        st = mc.last_stats
        sec = t["main_kernel_ms"] / 1000.0
        out["mcmc_workload"] = (f"GW NEXI, {nv} voxels x 64 walkers, 24 shells, Nx 14, {steps} steps "
                                f"(of the 5000-step run), simultaneous update")
        out["mcmc_proposals_per_s"] = st["n_proposals"] / sec
        out["mcmc_accepted_samples_per_s"] = st["n_accepted"] / sec
        out["mcmc_acceptance"] = st["n_accepted"] / st["n_proposals"]
        out["mcmc_ms_per_step"] = t["main_kernel_ms"] / steps
        out["mcmc_block_size"] = t["block_size"]
        sfu_peak = 16 * nsm * ghz * 1e9
        out["mcmc_roofline"] = {"bound": "sfu", "mufu_per_proposal": MCMC_SFU_PER_PROPOSAL,
                                "achieved": out["mcmc_proposals_per_s"] * MCMC_SFU_PER_PROPOSAL / 1e9,
                                "peak": sfu_peak / 1e9, "unit": "G MUFU op/s",
                                "frac": out["mcmc_proposals_per_s"] * MCMC_SFU_PER_PROPOSAL / sfu_peak,
                                "kernel": "gw_kernel<NEXI,5,simultaneous>"}
    if "mcmc_summaries" in want:
        out.update(mcmc_summaries_leg(ctx, args))
    if "mcmc_cpu" in want:
        out.update(mcmc_cpu_leg(args))
    if "c1" in want:
        out.update(extra_c1(ctx, args))
    if "c3" in want:
        out.update(extra_r1r2s_batch(ctx, args))
    if "c4" in want:
        out.update(extra_nexi_rician(ctx, args))
    if "surface" in want:
        out.update(extra_nexi_surface(ctx, args))
    if "autotune" in want:
        out["autotune"] = autotune_leg(ctx)
    return out


def autotune_leg(ctx):
    """Every launch shape the autotuner chooses from, timed explicitly, next
    to its choice (block_size 0): the joint R1-R2* batch (1.26M voxels, 200
    iterations), NEXI Rician Nx 100 (500k voxels, 10 iterations) and
    Goodman-Weare NEXI (200k voxels x 64 walkers, 20 steps).  Device time of
    the main kernel, ms."""
    from gacelle_b200 import askadam_solver as gxa, mcmc_solver, phantoms
    from gacelle_b200.models import _GxModelHandle, gpuNEXI
    _lib = _lib_mod()
    res = {}
    # joint R1-R2* batch
    sizes = [50_000, 110_000, 170_000, 230_000, 300_000, 400_000]
    ys = [phantoms.r1r2s_volume(n, 1003 + i)[0] for i, n in enumerate(sizes)]
    th0s = [np.ascontiguousarray(np.tile(np.array([[1.0], [1.0], [30.0]], np.float32), (1, n))) for n in sizes]
    model = _GxModelHandle(_lib.MODEL_R1R2S, te=phantoms.R1R2S_TE, fa_deg=phantoms.R1R2S_FA, tr=phantoms.R1R2S_TR)
    vols = (_lib.GxVolume * 6)(*[_gx_volume(y, t) for y, t in zip(ys, th0s)])
    outs = [np.zeros((3, n), np.float32) for n in sizes]
    rr = (_lib.GxAskadamResult * 6)()
    for r, o in zip(rr, outs):
        r.final_theta = o.ctypes.data_as(_lib._fp)

    def fit_ms(model, vols, nvol, res_arr, f, names, lb, ub, block):
        opts = gxa.build_opts(dict(f, blockSize=block), names, lb, ub, "fused")
        ms = []
        for _ in range(3):
            _lib.check(_lib.lib().gx_askadam(ctx.ptr, C.byref(model.s), _lib.MEM_HOST, vols, nvol, C.byref(opts),
                                             res_arr))
            t = ctx.timing()
            ms.append(t["main_kernel_ms"])
        return min(ms[1:]), t["block_size"]
    base = {"initialLearnRate": 0.01, "decayRate": 0.0, "lossFunction": "mse", "tol": 0.0,
            "patienceConvergence": float("inf"), "convergenceStepTol": 0.0, "convergenceGradTol": 0.0}
    f = gxa.check_set_default_basic(dict(base, iteration=200))
    row = {}
    for b in (64, 128, 256, 512, 0):
        ms, used = fit_ms(model, vols, 6, rr, f, ["M0", "R1", "R2star"], [0.0, 0.1, 0.1], [2.0, 10.0, 200.0], b)
        row["auto" if b == 0 else str(b)] = ms
        if b == 0:
            row["auto_block"] = used
    res["joint_r1r2s_batch_200_iterations"] = row
    # NEXI Rician, Nx 100
    nv = 500_000
    y, _ = phantoms.nexi_volume(nv, 1004, sigma=0.02, rician=True, nx=14)
    b_, d_ = phantoms.nexi_shells()
    model = _GxModelHandle(_lib.MODEL_NEXI, bval=b_, delta=d_, lmax=0, nx=100)
    th0 = np.ascontiguousarray(np.tile(np.array([[0.4], [2.0], [1.0], [0.05]], np.float32), (1, nv)))
    vol = _gx_volume(np.ascontiguousarray(y), th0)
    out = np.zeros((4, nv), np.float32)
    r1 = _lib.GxAskadamResult()
    r1.final_theta = out.ctypes.data_as(_lib._fp)
    f = gxa.check_set_default_basic(dict(base, iteration=10, lossFunction="rician", noiseSigma=0.02,
                                         tol=-float("inf")))
    row = {}
    lb, ub = [2.2e-16, 2.2e-16, 2.2e-16, 1 / 250], [1.0, 3.0, 3.0, 1.0]
    for b in (64, 128, 256, 512, 0):
        ms, used = fit_ms(model, C.byref(vol), 1, C.byref(r1), f, ["fa", "Da", "De", "ra"], lb, ub, b)
        row["auto" if b == 0 else str(b)] = ms
        if b == 0:
            row["auto_block"] = used
    res["nexi_rician_nx100_10_iterations"] = row
    # Goodman-Weare NEXI
    nv = 200_000
    y, gt = phantoms.nexi_volume(nv, 1005, sigma=0.02, rician=False, nx=14)
    m = gpuNEXI(b_, d_, nx=14)
    m.updateProperty({"solver": "mcmc", "lmax": 0})
    x0 = np.vstack([gt["fa"], gt["Da"], gt["De"], gt["ra"], np.full(nv, 0.02)]).astype(np.float32)
    row = {}
    for b in (64, 128, 256, 512, 1024, 0):
        fit = mcmc_solver.check_set_default_basic({"algorithm": "ensemble", "iteration": 20, "burnin": 0.2,
                                                   "thinning": 10, "Nwalker": 64, "StepSize": 2,
                                                   "modelParams": m.modelParams, "blockSize": b,
                                                   "lb": list(m.lb[:4]) + [0.02], "ub": list(m.ub[:4]) + [0.02],
                                                   "returnPosterior": False})
        mc = mcmc_solver.mcmc(ctx)
        ms = []
        for _ in range(3):
            mc.optimisation(y, np.ones((1, nv), bool), None, {p: x0[k] for k, p in enumerate(m.modelParams)}, fit, m)
            ms.append(mc.last_timing["main_kernel_ms"])
        row["auto" if b == 0 else str(b)] = min(ms[1:])
        if b == 0:
            row["auto_block"] = mc.last_timing["block_size"]
    res["gw_nexi_20_steps"] = row
    return res


def mcmc_summaries_leg(ctx, args):
    """res2out's median / iqr / mode of the Goodman-Weare NEXI run (200k voxels
    x 64 walkers), computed on the device from the kept samples, which stay in
    HBM (no posterior returned): the summaries' kernel time and the samples
    per voxel it ranks."""
    from gacelle_b200 import mcmc_solver, phantoms
    from gacelle_b200.models import gpuNEXI
    nv, steps = 200_000, args.mcmc_summary_steps
    y, gt = phantoms.nexi_volume(nv, 1005, sigma=0.02, rician=False, nx=14)
    b, d = phantoms.nexi_shells()
    m = gpuNEXI(b, d, nx=14)
    m.updateProperty({"solver": "mcmc", "lmax": 0})
    x0 = np.vstack([gt["fa"], gt["Da"], gt["De"], gt["ra"], np.full(nv, 0.02)]).astype(np.float32)
    fit = mcmc_solver.check_set_default_basic({"algorithm": "ensemble", "iteration": steps, "burnin": 0.2,
                                               "thinning": 10, "Nwalker": 64, "StepSize": 2,
                                               "modelParams": m.modelParams,
                                               "metric": ["mean", "std", "median", "iqr", "mode"],
                                               "lb": list(m.lb[:4]) + [0.02], "ub": list(m.ub[:4]) + [0.02],
                                               "returnPosterior": False})
    mc = mcmc_solver.mcmc(ctx)
    out = mc.optimisation(y, np.ones((1, nv), bool), None, {p: x0[k] for k, p in enumerate(m.modelParams)}, fit, m)
    t = mc.last_timing
    ns = mcmc_solver.number_of_samples(fit)
    assert np.all(np.isfinite(out["median"]["fa"])) and np.all(np.isfinite(out["mode"]["Da"]))
    return {"mcmc_summaries_workload": f"GW NEXI, {nv} voxels x 64 walkers, {steps} steps, {ns} kept samples per "
                                       f"walker: median, iqr, mode of 5 parameters over {64 * ns} samples per voxel",
            "mcmc_summaries_ms": t["aux_kernel_ms"], "mcmc_summaries_posterior_bytes": 4 * 5 * nv * 64 * ns,
            "mcmc_summaries_chain_ms": t["main_kernel_ms"]}


def mcmc_cpu_leg(args):
    """CPU baseline of the Goodman-Weare side run: the FP64 oracle's sampler on
    a voxel subset of the same phantom (same protocol, walkers and stretch
    scale) on all host threads, proposals/s extrapolated per voxel-walker-step."""
    import oracle
    from gacelle_b200 import phantoms
    nv, steps, W = args.mcmc_cpu_voxels, args.mcmc_cpu_steps, 64
    y, gt = phantoms.nexi_volume(nv, 1005, sigma=0.02, rician=False, nx=14)
    b, d = phantoms.nexi_shells()
    x0 = np.vstack([gt["fa"], gt["Da"], gt["De"], gt["ra"], np.full(nv, 0.02)])
    lb = [2.220446049250313e-16] * 3 + [1 / 250, 0.02]
    ub = [1.0, 3.0, 3.0, 1.0, 0.02]
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    r = oracle.mcmc(oracle.nexi(b, d, nx=14), oracle.Volume(y.astype(np.float64)), x0, lb, ub,
                    iteration=steps, thinning=10, burnin=0.2, nwalker=W, step_size=2.0, seed=1005, nthreads=cores)
    dt = time.perf_counter() - t0
    return {"mcmc_cpu_baseline": {"value": r["n_proposals"] / dt, "unit": "proposals/s", "cores": cores,
                                  "kind": "port", "accepted_samples_per_s": r["n_accepted"] / dt,
                                  "sample": f"{nv} voxels x {W} walkers x {steps} steps of a phantom with the "
                                            f"same distributions and protocol ({dt:.1f} s)"}}


def extra_c1(ctx, args):
    """The CPU-baseline configuration: mono-exponential R2*, 64x64x1 voxels
    (full mask, 4096), 12 echoes, MSE, Adam lr 0.01, 2000 iterations, start
    (1, 30), seed 1001: the FP64 oracle on one host thread and on all of
    them, the plain and the fused GPU paths (host buffers, whole calls)."""
    import oracle
    from gacelle_b200 import askadam_solver as gxa, phantoms, utils
    from gacelle_b200.models import _GxModelHandle
    from gacelle_b200 import _lib
    mask = np.ones((64, 64, 1), bool)
    data, _ = phantoms.r2s_phantom(mask, 1001)
    idx = utils.mask_index(mask).astype(np.int32)
    y = utils.reshape_ND2GD(data, idx)
    n = y.shape[1]
    th0 = np.tile(np.array([[1.0], [30.0]], np.float32), (1, n))
    iters = 2000
    f = gxa.check_set_default_basic({"iteration": iters, "initialLearnRate": 0.01, "decayRate": 0.0,
                                     "lossFunction": "mse", "tol": 0.0, "patienceConvergence": float("inf"),
                                     "convergenceStepTol": 0.0, "convergenceGradTol": 0.0})
    lb, ub = [0.0, 0.1], [2.0, 200.0]
    out = {"c1_workload": f"R2* MSE, 64x64x1 voxels ({n}), 12 echoes, {iters} iterations, no TV"}
    model = _GxModelHandle(_lib.MODEL_R2S, te=phantoms.R2S_TE)
    for path in ("plain", "fused"):
        o = gxa.build_opts(f, ["M0", "R2star"], lb, ub, path)
        solver = gxa.askadam(ctx, path)
        for _ in range(2):  # the first fused call of this configuration runs the autotuner's trials
            solver._run(model, y, None, th0, None, None, idx, mask.shape, o, 12, 2)
        t = solver.last_timing
        out[f"c1_{path}_voxel_fits_per_s"] = n / (t["total_ms"] / 1000.0)
        out[f"c1_{path}_call_ms"] = t["total_ms"]
    vol = oracle.Volume(y.astype(np.float64), theta0=th0.astype(np.float64))
    for tag, thr in (("1thread", 1), ("allcores", os.cpu_count() or 1)):
        t0 = time.perf_counter()
        oracle.askadam(oracle.r2s(phantoms.R2S_TE), vol, oracle.adam_opts(lb, ub, dict(f, nthreads=thr)),
                       want_min=False, want_history=False)
        dt = time.perf_counter() - t0
        out[f"c1_cpu_{tag}_voxel_fits_per_s"] = n / dt
        out[f"c1_cpu_{tag}_threads"] = thr
    return out


def parity_leg(ctx, W, model, iters):
    """The "equal FP64 error" half of the metric on the benchmark volume: the
    fused and the plain path run `iters` epochs of the same fit, the FP64
    oracle (the checker) runs it in double precision and once more with its
    parameter state rounded to FP32 after every update; per parameter map the
    relative RMSE of each GPU path against FP64, and the FP32-state band."""
    import oracle
    from gacelle_b200 import askadam_solver as gxa
    f = gxa.check_set_default_basic(dict(W["fitting"], iteration=iters))
    res = {}
    for path in ("fused", "plain"):
        o = gxa.build_opts(f, ["M0", "R2star"], W["lb"], W["ub"], path)
        r = gxa.askadam(ctx, path)._run(model, W["y"], None, W["th0"], None, None, W["idx"], W["mask"].shape,
                                        o, 12, 2)
        res[path] = r["final_theta"].astype(np.float64)
    fo = dict(f, _reg_index=[1], _reg_lambda=[1e-3], nthreads=os.cpu_count() or 1)
    vol = oracle.Volume(W["y"].astype(np.float64), dims=W["mask"].shape, grid_index=W["idx"],
                        theta0=W["th0"].astype(np.float64))
    t0 = time.perf_counter()
    o64 = oracle.askadam(oracle.r2s(W["te"]), vol, oracle.adam_opts(W["lb"], W["ub"], fo), want_min=False)
    o32 = oracle.askadam(oracle.r2s(W["te"]), vol, oracle.adam_opts(W["lb"], W["ub"], dict(fo, _state_f32=True)),
                         want_min=False)
    dt = time.perf_counter() - t0

    def rr(a, b):
        return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))
    out = {"parity_workload": f"the benchmark volume, {iters} epochs, final parameter maps vs the FP64 oracle",
           "parity_oracle_s": dt}
    for k, p in enumerate(("M0", "R2star")):
        band = rr(o32["final"][k], o64["final"][k])
        out[f"parity_{p}_fused_rel_rmse"] = rr(res["fused"][k], o64["final"][k])
        out[f"parity_{p}_plain_rel_rmse"] = rr(res["plain"][k], o64["final"][k])
        out[f"parity_{p}_fp32_state_band"] = band
        out[f"parity_{p}_within_2x_band"] = bool(max(out[f"parity_{p}_fused_rel_rmse"],
                                                     out[f"parity_{p}_plain_rel_rmse"]) <= 2 * band + 1e-5)
    return out


def _gx_volume(y, th0, sigma=None):
    v = _lib_mod().GxVolume()
    nm, n = y.shape
    v.dims[0], v.dims[1], v.dims[2] = n, 1, 1
    v.nvox = n
    v.data = y.ctypes.data_as(_lib_mod()._fp)
    v.theta0 = th0.ctypes.data_as(_lib_mod()._fp)
    if sigma is not None:
        v.sigma = sigma.ctypes.data_as(_lib_mod()._fp)
    return v


def _lib_mod():
    from gacelle_b200 import _lib
    return _lib


def extra_r1r2s_batch(ctx, args):
    """Joint R1-R2* askAdam on a batch of six volumes with uneven voxel counts
    (50k-400k, 1.26M voxels) in one call: 24 measurements (12 TE x 2 flip
    angles), MSE, Adam lr 0.01, start (1, 1, 30), fused path."""
    from gacelle_b200 import askadam_solver as gxa, phantoms
    from gacelle_b200.models import _GxModelHandle
    _lib = _lib_mod()
    sizes = [50_000, 110_000, 170_000, 230_000, 300_000, 400_000]
    ys = [phantoms.r1r2s_volume(n, 1003 + i)[0] for i, n in enumerate(sizes)]
    th0s = [np.ascontiguousarray(np.tile(np.array([[1.0], [1.0], [30.0]], np.float32), (1, n))) for n in sizes]
    model = _GxModelHandle(_lib.MODEL_R1R2S, te=phantoms.R1R2S_TE, fa_deg=phantoms.R1R2S_FA, tr=phantoms.R1R2S_TR)
    f = gxa.check_set_default_basic({"iteration": args.c3_iters, "initialLearnRate": 0.01, "decayRate": 0.0,
                                     "lossFunction": "mse", "tol": 0.0, "patienceConvergence": float("inf"),
                                     "convergenceStepTol": 0.0, "convergenceGradTol": 0.0})
    opts = gxa.build_opts(f, ["M0", "R1", "R2star"], [0.0, 0.1, 0.1], [2.0, 10.0, 200.0], "fused")
    vols = (_lib.GxVolume * 6)(*[_gx_volume(y, t) for y, t in zip(ys, th0s)])
    outs = [np.zeros((3, n), np.float32) for n in sizes]
    res = (_lib.GxAskadamResult * 6)()
    for r, o in zip(res, outs):
        r.final_theta = o.ctypes.data_as(_lib._fp)
    for _ in range(2):  # the first call of this configuration runs the autotuner's trials
        _lib.check(_lib.lib().gx_askadam(ctx.ptr, C.byref(model.s), _lib.MEM_HOST, vols, 6, C.byref(opts), res))
    t = ctx.timing()
    nv = sum(sizes)
    sec = t["main_kernel_ms"] / 1000.0
    return {"c3_workload": f"joint R1R2* batch of 6 volumes ({nv} voxels), 24 measurements, MSE, "
                           f"{args.c3_iters} iterations, one call",
            "c3_voxel_fits_per_s": nv / sec, "c3_voxel_iterations_per_s": nv * args.c3_iters / sec,
            "c3_call_ms": t["total_ms"], "c3_block_size": t["block_size"]}


def extra_nexi_rician(ctx, args):
    """NEXI lmax 0 with the Rician likelihood loss, 100-node powder average,
    500k voxels (sigma 0.02), a bounded number of iterations; and the
    likelihood starting points of the same voxels against a 10^4-entry
    dictionary (gpuNEXI.likelihood)."""
    from gacelle_b200 import askadam_solver as gxa, phantoms
    from gacelle_b200.models import _GxModelHandle, gpuNEXI
    _lib = _lib_mod()
    nv, nx = 500_000, 100
    rng = np.random.default_rng(1004)
    fa = rng.uniform(0.1, 0.9, nv)
    tex = rng.uniform(2.0, 50.0, nv)
    ra = (1 - fa) / tex
    while (ra < 1 / 250).any():
        bad = ra < 1 / 250
        tex[bad] = rng.uniform(2.0, 50.0, bad.sum())
        ra = (1 - fa) / tex
    th = np.ascontiguousarray(np.vstack([fa, rng.uniform(1, 3, nv), rng.uniform(0.5, 1.5, nv), ra]),
                              dtype=np.float32)
    b, d = phantoms.nexi_shells()
    model = _GxModelHandle(_lib.MODEL_NEXI, bval=b, delta=d, lmax=0, nx=nx)
    S = np.zeros((24, nv), np.float32)
    _lib.check(_lib.lib().gx_forward(ctx.ptr, C.byref(model.s), _lib.MEM_HOST, th.ctypes.data, None, nv,
                                     S.ctypes.data))
    sig = 0.02
    y = np.ascontiguousarray(np.sqrt((S + sig * rng.standard_normal(S.shape)) ** 2 +
                                     (sig * rng.standard_normal(S.shape)) ** 2), dtype=np.float32)
    lb, ub = [2.2e-16, 2.2e-16, 2.2e-16, 1 / 250], [1.0, 3.0, 3.0, 1.0]
    th0 = np.ascontiguousarray(np.tile(np.array([[0.4], [2.0], [1.0], [0.05]], np.float32), (1, nv)))
    f = gxa.check_set_default_basic({"iteration": args.c4_iters, "initialLearnRate": 0.01, "decayRate": 0.0,
                                     "lossFunction": "rician", "noiseSigma": sig, "tol": -float("inf"),
                                     "patienceConvergence": float("inf"), "convergenceStepTol": 0.0,
                                     "convergenceGradTol": 0.0})
    opts = gxa.build_opts(f, ["fa", "Da", "De", "ra"], lb, ub, "fused")
    out = np.zeros((4, nv), np.float32)
    vol = _gx_volume(y, th0)
    res = _lib.GxAskadamResult()
    res.final_theta = out.ctypes.data_as(_lib._fp)
    for _ in range(2):  # the first call of this configuration runs the autotuner's trials
        _lib.check(_lib.lib().gx_askadam(ctx.ptr, C.byref(model.s), _lib.MEM_HOST, C.byref(vol), 1, C.byref(opts),
                                         C.byref(res)))
    assert res.final_niteration == args.c4_iters
    t = ctx.timing()
    sec = t["main_kernel_ms"] / 1000.0
    r = {"c4_workload": f"NEXI lmax 0, Rician loss, Nx {nx}, {nv} voxels, {args.c4_iters} iterations",
         "c4_voxel_iterations_per_s": nv * args.c4_iters / sec, "c4_ms_per_iteration": t["main_kernel_ms"] / args.c4_iters,
         "c4_block_size": t["block_size"]}
    # dictionary starting points of the same voxels
    m = gpuNEXI(b, d)
    m.context = ctx
    x_train, S_train, _ = m.traindata(10_000, 0)
    m.likelihood(y, x_train, S_train, 0)
    t = ctx.timing()
    r["dictionary_workload"] = f"likelihood starting points, {nv} voxels x {x_train.shape[1]} entries x 24 measurements"
    r["dictionary_ms"] = t["main_kernel_ms"]
    r["dictionary_pairs_per_s"] = nv * x_train.shape[1] / (t["main_kernel_ms"] / 1000.0)
    return r


def extra_nexi_surface(ctx, args):
    """NEXI fits on cortical-surface data at fsaverage scale: two hemisphere
    meshes of 405 x 405 vertices (164,025 each; a triangulated sheet stands in
    for the subject's surface), 24 shells, Nx 14, MSE, the same start and
    iteration count three times: no regulariser, surface TV on fa (mesh
    neighbour tables, one launch per epoch) and the prior distribution on fa
    and ra (fused).  Reports each fit's voxel-iterations/s."""
    from gacelle_b200 import askadam_solver as gxa
    from gacelle_b200 import phantoms, surface, utils
    from gacelle_b200.models import _GxModelHandle
    _lib = _lib_mod()
    side, iters = 405, args.surf_iters
    nvh = side * side
    idx = np.arange(side * side).reshape(side, side)
    faces = np.concatenate([np.stack([idx[:-1, :-1], idx[1:, :-1], idx[1:, 1:]], -1).reshape(-1, 3),
                            np.stack([idx[:-1, :-1], idx[1:, 1:], idx[:-1, 1:]], -1).reshape(-1, 3)])
    nb, _ = surface.mesh_neighbours(faces, nvh)
    nbs = np.concatenate([nb, nb + nvh]).T                                   # [maxnb][2 nvh], grid indices
    lens = np.where(nbs == np.arange(2 * nvh)[None, :], 1e6, 1.0).astype(np.float32)  # edge lengths 1
    nv = 2 * nvh
    y, gt = phantoms.nexi_volume(nv, 1006, sigma=0.02, rician=False, nx=14)
    b, d = phantoms.nexi_shells()
    model = _GxModelHandle(_lib.MODEL_NEXI, bval=b, delta=d, lmax=0, nx=14)
    lb, ub = [2.2e-16, 2.2e-16, 2.2e-16, 1 / 250], [1.0, 3.0, 3.0, 1.0]
    th0 = np.ascontiguousarray(np.tile(np.array([[0.4], [2.0], [1.0], [0.05]], np.float32), (1, nv)))
    y = np.ascontiguousarray(y, np.float32)
    gidx = np.arange(nv, dtype=np.int32)
    nbs = np.ascontiguousarray(nbs, np.int32)
    mu = np.ascontiguousarray(np.vstack([gt["fa"], gt["ra"]]), np.float32)
    sd = np.ascontiguousarray(np.vstack([np.full(nv, 0.1), np.full(nv, 0.02)]), np.float32)
    out = {"surface_workload": f"NEXI lmax 0, MSE, Nx 14, 24 shells, 2 x {nvh} surface vertices, {iters} iterations"}
    for tag, reg in (("none", {}), ("surface_tv", {"lambda": [1e-3], "regmap": ["fa"], "dataType": "surface"}),
                     ("prior", {"lambda": [1e-3, 1e-3], "regmap": ["fa", "ra"], "regularisationType": "prior"})):
        f = gxa.check_set_default_basic(dict({"iteration": iters, "initialLearnRate": 0.01, "lossFunction": "mse",
                                              "tol": 0.0, "patienceConvergence": float("inf"),
                                              "convergenceStepTol": 0.0, "convergenceGradTol": 0.0}, **reg))
        opts = gxa.build_opts(f, ["fa", "Da", "De", "ra"], lb, ub, "fused")
        vol = _gx_volume(y, th0)
        vol.dims[0], vol.dims[1], vol.dims[2] = 1, nvh, 2
        vol.grid_index = gidx.ctypes.data_as(_lib._i32p)
        if tag == "surface_tv":
            vol.max_neighbours = nbs.shape[0]
            vol.neighbours = nbs.ctypes.data_as(_lib._i32p)
            vol.edge_length = lens.ctypes.data_as(_lib._fp)
        if tag == "prior":
            vol.prior_mu = mu.ctypes.data_as(_lib._fp)
            vol.prior_sd = sd.ctypes.data_as(_lib._fp)
        th = np.zeros((4, nv), np.float32)
        res = _lib.GxAskadamResult()
        res.final_theta = th.ctypes.data_as(_lib._fp)
        _lib.check(_lib.lib().gx_askadam(ctx.ptr, C.byref(model.s), _lib.MEM_HOST, C.byref(vol), 1,
                                         C.byref(opts), C.byref(res)))
        t = ctx.timing()
        out[f"surface_{tag}_voxel_iterations_per_s"] = nv * iters / (t["main_kernel_ms"] / 1000.0)
        out[f"surface_{tag}_ms_per_iteration"] = t["main_kernel_ms"] / iters
    return out


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        else:
            engine_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
