"""Benchmark of the coupled EK-PNP step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload channel-4096x1024] [--storage f32|f16|f64]

One step = one coupled update of one channel: the fused LBM kernel (fluid +
two ion species, walls, streaming, Guo force) and the Poisson solve (row FFTs,
tridiagonal column solves, inverse row FFTs).  Metric: coupled MLUPS =
nx*ny*steps / seconds, summed over ranks.  N > 1 runs one independent channel
per GPU (replicas; the single-channel path does not shard), so scaling is weak.

The device-timed region holds exactly K steps between CUDA events on the
solver's stream, after W warm-up steps, with a barrier and a stream
synchronisation on both sides; the working set (two population buffers of
27 planes) is several times the 126 MB L2, so no flush is needed.  `e2e` runs
the same K steps through the public API from pinned host buffers: fields in
(H2D), equilibrium initialisation, steps in chunks of 100 with a residual
read-back after each, fields out (D2H), timed by the host clock.

--impl reference times the CPU oracle (the OpenMP restatement of the
reference's update rules; the reference itself has no CPU path) on the same
workload, on rank 0 only, for a bounded number of full steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ek-pnp_b200"))

STORAGE = {"f64": 0, "f32": 1, "f16": 2}
POP_BYTES = {"f64": 8, "f32": 4, "f16": 2}
CPU_SAMPLE_S = 15.0


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peak_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(workload, storage):
    """DRAM bytes per launch of the LBM kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"lbm_{storage}_{workload}.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["dram_bytes_per_launch"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        self.index = vis.split(",")[local_rank] if vis else str(local_rank)
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.index, f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.strip().splitlines():
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


from ekpnp.dist import Dist, shard_by_nodes  # noqa: E402


def cpu_oracle_rate(params, seed, max_steps, budget_s):
    """Coupled MLUPS of the CPU oracle with all host threads, full steps of the
    same channel until budget_s elapsed (at least one step)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from ekpnp import noisy_uniform_state
    oracle.build()
    threads = oracle.set_threads(0)
    p = dict(params, storage=0)
    o = oracle.OracleChannel(p)
    o.set_fields(**noisy_uniform_state(p["nx"], p["ny"], seed))
    o.init_equilibrium()
    o.step(1)  # warm-up: page in, build FFT plans
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        o.step(1)
        steps += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    return p["nx"] * p["ny"] * steps / dt / 1e6, threads, steps, dt


def run_reference(args, d):
    from ekpnp import workload_params, WORKLOADS
    if d.rank != 0:
        return 0
    p = workload_params(args.workload)
    w = WORKLOADS[args.workload]
    budget = min(120.0, max(10.0, 0.05 * args.steps))
    rate, threads, steps, dt = cpu_oracle_rate(p, w["seed"], args.steps, budget)
    sample = f"{steps} full coupled FP64 steps of the {w['nx']}x{w['ny']} channel in {dt:.1f} s"
    line = {
        "metric": "coupled_mlups", "value": rate, "unit": "MLUPS", "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": 1, "ms_per_step": dt / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded noisy uniform state)",
        "config": {"workload": args.workload, "nx": w["nx"], "ny": w["ny"], "storage": "f64",
                   "host_threads": threads},
        "cpu_baseline": {"value": rate, "unit": "MLUPS", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, d):
    import torch
    import ekpnp
    from ekpnp import Channel, WORKLOADS, noisy_uniform_state, workload_params
    w = WORKLOADS[args.workload]
    nx, ny, nn = w["nx"], w["ny"], w["nx"] * w["ny"]
    ekpnp.set_device(d.local)
    p = workload_params(args.workload, storage=STORAGE[args.storage])
    init = noisy_uniform_state(nx, ny, w["seed"] + d.rank)

    # ---- device-timed region ----
    ch = Channel(p)
    if args.lbm_kernel != "auto":
        ch.set_lbm_kernel(args.lbm_kernel)
    ch.set_fields(**init)
    ch.init_equilibrium()
    ch.step(args.warmup)
    ch.sync()
    clocks = ClockSampler(d.local)
    clocks.start()
    time.sleep(0.3)
    d.barrier()
    ch.sync()
    n_launch0 = ch.launches
    ch.mark(0)
    ch.step(args.steps)
    ch.mark(1)
    ms = ch.elapsed_ms(0, 1)
    ch.sync()
    d.barrier()
    launches = ch.launches - n_launch0
    clk = clocks.stop()
    ms_max = d.max(ms)
    # second pass of K steps with an event pair around every kernel: per-kernel
    # durations for the roofline (the events add gaps, so `value` is not taken here)
    ch.profile(True)
    ch.step(args.steps)
    prof = ch.profile_read()
    ch.profile(False)
    value = d.world * nn * args.steps / (ms_max / 1e3) / 1e6

    # ---- roofline of the dominant kernel (the fused LBM step) ----
    lbm_ms, lbm_n = prof["lbm"]
    per_launch_s = lbm_ms / max(lbm_n, 1) / 1e3
    # 27 pops in + 27 out, psi in, right-hand side out: FP64 planes for FP64
    # storage, FP32 planes (psi and rhs about FP64 row constants) for shifted
    fld = 8 if args.storage == "f64" else 4
    bytes_node = 54 * POP_BYTES[args.storage] + 2 * fld
    achieved = nn * bytes_node / per_launch_s / 1e9
    peak, peak_kind = measured_peak_gbs()
    traffic = ncu_traffic(args.workload, args.storage)
    # whole step at B_node = 54 s_pop + 8 s_fld (LBM, Poisson passes A, B, C)
    step_bytes = 54 * POP_BYTES[args.storage] + 8 * fld
    step_ms = ms / args.steps
    shares = {k: round(v[0] / max(sum(x[0] for x in prof.values()), 1e-12), 4) for k, v in prof.items()}
    ch.close()

    # ---- end to end through the public API, pinned host buffers ----
    pin = {k: torch.from_numpy(init[k]).pin_memory() for k in ("rho", "ux", "uy", "cp", "cn", "psi")}
    outs = {k: torch.empty((ny, nx), dtype=torch.float64).pin_memory() for k in ("ux", "cp", "cn", "psi")}
    order = ("rho", "ux", "uy", "cp", "cn", "psi", "ex", "ey")
    chunk = 100
    reps = max(1, args.steps // chunk)
    ch = Channel(p)
    if args.lbm_kernel != "auto":
        ch.set_lbm_kernel(args.lbm_kernel)
    ch.set_fields(**init)
    ch.init_equilibrium()
    ch.step(min(args.warmup, 10))
    ch.sync()
    d.barrier()
    t0 = time.perf_counter()
    ch.set_fields_from_pointers([pin[k].data_ptr() if k in pin else 0 for k in order])
    ch.init_equilibrium()
    for _ in range(reps):
        ch.step(chunk)
        ch.residual(chunk)
    ch.get_fields_to_pointers([outs[k].data_ptr() if k in outs else 0 for k in order])
    e2e_s = d.max(time.perf_counter() - t0)
    ch.close()
    e2e_steps = reps * chunk
    e2e = {"value": d.world * nn * e2e_steps / e2e_s / 1e6, "unit": "MLUPS",
           "h2d_bytes_per_step": 6 * nn * 8 / e2e_steps,
           "d2h_bytes_per_step": (4 * nn * 8 + reps * 5 * 8) / e2e_steps,
           "steps": e2e_steps}

    cpu = None
    if d.world == 1 and d.rank == 0 and not args.no_cpu_baseline:
        rate, threads, steps, dt = cpu_oracle_rate(workload_params(args.workload), w["seed"], 10 ** 6, CPU_SAMPLE_S)
        cpu = {"value": rate, "unit": "MLUPS", "cores": threads, "kind": "port",
               "sample": f"{steps} full coupled FP64 steps of the {nx}x{ny} channel in {dt:.1f} s"}

    if d.rank == 0:
        line = {
            "metric": "coupled_mlups", "value": value, "unit": "MLUPS", "n_gpus": d.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"f64": "f64", "f32": "f32", "f16": "f32 (f16 storage)"}[args.storage],
            "data": "synthetic (seeded noisy uniform state, u = psi = 0)",
            "config": {"workload": args.workload, "nx": nx, "ny": ny, "storage": args.storage + "-shifted"
                       if args.storage != "f64" else "f64", "kappa_h": w["kappa_h"], "zeta": w["zeta"],
                       "e_x": w["ex"], "parallelism": f"replicas x{d.world}", "lbm_kernel": args.lbm_kernel,
                       "l2": "working set > 126 MB L2 (2 x 27 population planes), no flush"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "fused LBM step", "bytes_per_node": bytes_node,
                         "launch_ms": per_launch_s * 1e3,
                         "timing": "CUDA events around each launch, second pass of the same K steps",
                         "traffic_source": (f"profiles/lbm_{args.storage}_{args.workload}.json: ncu "
                                            "dram__bytes_read.sum + dram__bytes_write.sum of this kernel on "
                                            "this workload (a separate capture, not this run)")
                         if traffic is not None else None},
            "step_roofline": {"bytes_per_node": step_bytes, "achieved": value * 1e6 * step_bytes / 1e9,
                              "unit": "GB/s", "frac": value * 1e6 * step_bytes / 1e9 / peak,
                              "basis": "54 s_pop + 8 s_fld per node and step (LBM + Poisson passes)"},
            "step_breakdown": {"ms_per_step": step_ms,
                               "kernel_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
                               "share": shares},
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    return 0


def run_batch(args, d):
    """Batched workload: 512 channels of uneven size and physics (seeded draw),
    stepped in lockstep in cycles of 200 steps replayed from CUDA graphs."""
    import ekpnp
    from ekpnp import Batch, batch_specs, spec_params
    ekpnp.set_device(d.local)
    count = env_int("EK_BATCH_CHANNELS", 512)
    all_specs = batch_specs(count, seed=2)
    mine = shard_by_nodes(all_specs, d.world, d.rank)  # channels of this rank; no data exchange
    specs = [all_specs[i] for i in mine]
    total_nodes = sum(s["nx"] * s["ny"] for s in all_specs)
    ps = [spec_params(s, STORAGE[args.storage]) for s in specs]
    b = Batch(ps)
    nn = b.nodes
    for ch in b:
        ch.init_poisson_boltzmann("newton")
    graph = env_int("EK_BATCH_GRAPH", 1) != 0
    b.set_cycle(200, graph=graph)
    b.init_equilibrium()
    chosen, tune_ms = b.autotune(10)
    b.step(args.warmup)
    b.sync()
    clocks = ClockSampler(d.local)
    clocks.start()
    time.sleep(0.3)
    d.barrier()
    b.sync()
    ch0 = b[0]  # the channels run on the batch's stream
    n0 = b.launches
    ch0.mark(0)
    b.step(args.steps)
    ch0.mark(1)
    ms = ch0.elapsed_ms(0, 1)
    b.sync()
    d.barrier()
    launches = b.launches - n0
    clk = clocks.stop()
    ms_max = d.max(ms)
    value = total_nodes * args.steps / (ms_max / 1e3) / 1e6  # all ranks' channels / the slowest rank's time
    res = b.residual(200)
    finite = bool(np.isfinite(res[:, :4]).all() or np.isinf(res[:, :4]).all())
    b.close()
    if d.rank == 0:
        line = {
            "metric": "coupled_mlups", "value": value, "unit": "MLUPS", "n_gpus": d.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": {"f32": "f32", "f16": "f32 (f16 storage)"}[args.storage],
            "data": "synthetic (seeded channel draw, Poisson-Boltzmann start)",
            "config": {"workload": args.workload, "channels": count, "nodes": total_nodes,
                       "nodes_rank0": nn,
                       "storage": args.storage + "-shifted",
                       "block_shape": dict(zip(("threads", "tile_width", "blocks_per_sm"), Batch.shapes()[chosen])),
                       "autotune_ms_per_step": {"x".join(map(str, sh)): round(m, 4)
                                                for sh, m in zip(Batch.shapes(), tune_ms)},
                       "cycle": 200, "graph": graph,
                       "parallelism": f"channel shards x{d.world} (balanced by node count)",
                       "l2": "working set > 126 MB L2, no flush"},
            "gpu_launches": launches,
            "clocks": clk,
            "finite": finite,
        }
        print(json.dumps(line), flush=True)
    return 0


def run_batch_steady(args, d):
    """The batched workload run to steady state: the 512 channels of the seed-2
    draw from their noisy cold start (u = psi = 0, c+- = c0 (1 + 1e-3 N), the
    deviates from the same stream), autotuned block shape, CUDA-graph cycles of
    200 steps, residual < 1e-8 checked every 2000 steps, converged or diverged
    channels frozen (their work leaves the batch), cap EK_STEADY_CAP steps
    (200,000).  Aggregate MLUPS = node updates of the stepping channels / wall
    time of the run (host clock, residual checks included)."""
    import ekpnp
    from ekpnp import Batch, batch_noisy_states, batch_specs, spec_params, warmstart as ws
    if d.rank != 0:
        return 0
    ekpnp.set_device(d.local)
    count = env_int("EK_BATCH_CHANNELS", 512)
    cap = env_int("EK_STEADY_CAP", 200_000)
    check = 2000
    specs = batch_specs(count, seed=2)
    b = Batch([spec_params(s, STORAGE[args.storage]) for s in specs])
    for ch, f in zip(b, batch_noisy_states(count, seed=2)):
        ch.set_fields(**f)
    b.set_cycle(200)
    b.init_equilibrium()
    chosen, tune_ms = b.autotune(10)
    for ch, f in zip(b, batch_noisy_states(count, seed=2)):  # start over after the timing steps
        ch.set_fields(**f)
    b.init_equilibrium()
    clocks = ClockSampler(d.local)
    clocks.start()
    info = ws.run_to_steady(b, tol=1e-8, check=check, max_steps=cap)
    clk = clocks.stop()
    launches = b.launches
    b.close()
    st = info["steps"]
    ok = st >= 0
    cap_ch = ~ok & ~info["diverged"]  # stepped to the cap without converging or diverging
    nodes = sum(s["nx"] * s["ny"] for s in specs)
    line = {
        "metric": "coupled_mlups", "value": info["node_steps"] / info["wall_s"] / 1e6, "unit": "MLUPS",
        "n_gpus": 1, "steps": int(cap), "warmup": 0, "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": {"f32": "f32", "f16": "f32 (f16 storage)"}[args.storage],
        "data": "synthetic (seeded channel draw and noisy cold start from the same stream)",
        "config": {"workload": f"batch-{count}-to-steady", "channels": count, "nodes": nodes,
                   "storage": args.storage + "-shifted", "tol": 1e-8, "cap_steps": cap, "check_every": check,
                   "block_shape": dict(zip(("threads", "tile_width", "blocks_per_sm"), Batch.shapes()[chosen])),
                   "cycle": 200, "graph": True, "freeze_converged": True},
        "wall_s": info["wall_s"], "node_steps": int(info["node_steps"]),
        "converged": int(ok.sum()), "diverged": int(np.sum(info["diverged"])),
        "at_cap": int(np.sum(cap_ch)),
        "steps_to_steady": {"median": float(np.median(st[ok])) if ok.any() else None,
                            "p90": float(np.percentile(st[ok], 90)) if ok.any() else None,
                            "max": int(st[ok].max()) if ok.any() else None},
        "residual_at_cap": {"median": float(np.median(info["history"][-1][cap_ch])) if cap_ch.any() else None,
                            "max": float(np.max(info["history"][-1][cap_ch])) if cap_ch.any() else None},
        "converged_nodes": int(sum(s["nx"] * s["ny"] for s, o in zip(specs, ok) if o)),
        "gpu_launches": int(launches), "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    return 0


def _start_summary(r, cap):
    st = np.asarray(r["steps"])
    ok = st >= 0
    return {"wall_s": r["wall_s"], "converged": int(ok.sum()), "channels": int(len(st)),
            "diverged": int(np.sum(r["diverged"])), "fallback": int(len(r["fallback"])),
            "median_steps_converged": float(np.median(st[ok])) if ok.any() else None,
            "steps_p90": float(np.percentile(np.where(ok, st, cap), 90)),
            "mean_steps_capped": float(np.mean(np.where(ok, st, cap)))}


def ws_training_set(n_train, gen_cap, check):
    """Steady states of the training channels (seed 3, 16 columns each) from
    the batched solver: loaded from EK_WS_CACHE when that file exists (written
    by an earlier run of this same function), else generated and, with
    EK_WS_CACHE set, saved there.  Returns (specs, targets, converged, steps,
    generation seconds)."""
    from ekpnp import batch_specs, warmstart as ws
    t0 = time.perf_counter()
    tr = batch_specs(n_train, seed=3)
    cache = os.environ.get("EK_WS_CACHE")
    if cache and os.path.exists(cache):
        z = np.load(cache)
        if len(z["T"]) != n_train:
            raise RuntimeError(f"{cache} holds {len(z['T'])} channels, not {n_train}")
        T, conv, steps = z["T"], z["conv"], z["steps"]
    else:
        T, conv, info = ws.generate_steady_states(tr, nx=16, max_steps=gen_cap, check=check)
        steps = info["steps"]
        if cache:
            np.savez(cache, T=T, conv=conv, steps=steps)
    return tr, T, conv, steps, time.perf_counter() - t0


def steps_to_tol(hist, check, tol=1e-8):
    """Steps at which a residual history (one value every `check` steps)
    reaches tol: the first check below it, else the log-linear extrapolation
    of the later half of the history (None where it does not decrease)."""
    h = np.asarray(hist, dtype=np.float64)
    s = check * (np.arange(len(h)) + 1)
    below = np.nonzero(np.isfinite(h) & (h < tol))[0]
    if len(below):
        return {"steps": int(s[below[0]]), "extrapolated": False}
    k = len(h) // 2
    ok = np.isfinite(h[k:]) & (h[k:] > 0)
    if ok.sum() < 2:
        return None
    slope, icpt = np.polyfit(s[k:][ok], np.log(h[k:][ok]), 1)
    if slope >= 0:
        return None
    return {"steps": int((np.log(tol) - icpt) / slope), "extrapolated": True,
            "decay_per_100k_steps": float(np.exp(slope * 1e5))}


def run_warmstart(args, d):
    """Learned warm start: steady states of `train` channels (seed 3) from the
    batched solver, the network trained on them (tensor-core kernels), then
    time to residual < 1e-8 of `eval` held-out channels (seed 4) from the
    network's start against the uniform cold start."""
    import ekpnp
    from ekpnp import batch_specs, warmstart as ws
    if d.rank != 0:
        return 0
    ekpnp.set_device(d.local)
    n_train = env_int("EK_WS_TRAIN", 8192)
    n_eval = env_int("EK_WS_EVAL", 256)
    cap = env_int("EK_WS_CAP", 200_000)
    gen_cap = env_int("EK_WS_GEN_CAP", 120_000)
    check = 2000
    tr, T, conv, gen_steps, gen_s = ws_training_set(n_train, gen_cap, check)
    ok = np.all(np.isfinite(T), axis=1)
    trs = [s for s, o in zip(tr, ok) if o]
    ev = batch_specs(n_eval, seed=4)
    kw = dict(max_steps=cap, check=check)
    out, train = {}, {}
    modes = os.environ.get("EK_WS_MODES", "residual,direct").split(",")
    sgs = {}
    for mode in modes:
        sg = ws.Surrogate(mode, seed=7)
        t1 = time.perf_counter()
        loss = sg.fit(trs, T[ok], iters=env_int("EK_WS_ITERS", 12000), lr=2e-3)
        train[mode] = {"seconds": time.perf_counter() - t1, "final_loss": float(loss[-200:].mean()),
                       "iterations": int(len(loss)), "gpu_launches": sg.net.launches}
        out[mode] = ws.warm_start_run(sg, ev, **kw)
        sgs[mode] = sg
    cold = ws.cold_start_run(ev, **kw)
    # the method without the network: the Newton Poisson-Boltzmann ions and
    # potential with the electro-osmotic velocity (the reference's own start,
    # LBM.cu:95-145, solved to convergence, plus the Helmholtz-Smoluchowski flow)
    phys = ws.physics_start_run(ev, **kw)
    best = modes[0]
    # x-reduced relaxation (16 columns, then tiled along x), from the best
    # network's start and from the cold start
    xr = {}
    for start in [a for a in os.environ.get("EK_WS_XR", "surrogate,physics,cold").split(",") if a]:
        xr[start] = ws.xreduced_start_run(ev, start=start, surrogate=sgs[best],
                                          narrow_max_steps=env_int("EK_WS_NARROW_CAP", 600_000), **kw)
    for sg in sgs.values():
        sg.close()
    # error of each start against the channel's final state of the warm run
    errs = {}
    for mode in modes:
        e = np.array([[ws.surrogate_error(s, f, p)[q] for q in ("psi", "cp", "cn", "ux")]
                      for s, f, p in zip(ev, out[mode]["fields"], out[best]["final"])])
        errs[mode] = {q: {"median": float(np.median(e[:, i])), "max": float(e[:, i].max())}
                      for i, q in enumerate(("psi", "cp", "cn", "ux"))}
    both = (np.asarray(out[best]["steps"]) >= 0) & (np.asarray(cold["steps"]) >= 0)
    line = {
        "metric": "time_to_steady_s", "value": out[best]["wall_s"], "unit": "s", "higher_is_better": False,
        "n_gpus": 1, "steps": None, "warmup": 0, "scaling": "none", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded channel draws; training from the batched solver's own steady states)",
        "config": {"workload": f"warmstart-{n_eval}", "train_channels": n_train, "train_usable": int(ok.sum()),
                   "train_converged": int(np.sum(conv)), "train_gen_cap": gen_cap, "eval_channels": n_eval,
                   "tol": 1e-8, "cap_steps": cap, "narrow_cap_steps": env_int("EK_WS_NARROW_CAP", 600_000),
                   "check_every": check, "storage": "f32-shifted",
                   "network": "4-256-256-256-512 SiLU, BF16 tcgen05, Adam"},
        "generation_s": gen_s, "training": train,
        "cold": _start_summary(cold, cap),
        "physics": _start_summary(phys, cap),
        "surrogate": {m: _start_summary(out[m], cap) for m in modes},
        "xreduced": {a: dict(_start_summary(r, cap), narrow_wall_s=r["narrow_wall_s"],
                             narrow_median_steps=float(np.median(np.where(r["narrow_steps"] >= 0, r["narrow_steps"], cap))),
                             full_steps_max=int(np.max(r["full_steps"])))
                     for a, r in xr.items()},
        "wall_speedup_vs_cold": dict({m: cold["wall_s"] / out[m]["wall_s"] for m in modes},
                                     physics=cold["wall_s"] / phys["wall_s"],
                                     **{f"xreduced_{a}": cold["wall_s"] / r["wall_s"] for a, r in xr.items()}),
        "wall_speedup_vs_physics": dict({m: phys["wall_s"] / out[m]["wall_s"] for m in modes},
                                        **{f"xreduced_{a}": phys["wall_s"] / r["wall_s"] for a, r in xr.items()}),
        "median_step_ratio_both_converged": (float(np.median(np.asarray(cold["steps"])[both] /
                                                             np.maximum(np.asarray(out[best]["steps"])[both], 1)))
                                             if both.any() else None),
        "start_error_vs_final": errs,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_hetero(args, d):
    """Heterogeneous wall: one 8192 x 2048 channel, zeta(x) = -2 + 1.5 sin(2 pi x / 1024),
    kappa*H = 64, E_x = 1e-4, seed 5.  Arms, each stepped to residual < 1e-8
    or the step cap (EK_HET_CAP), residual checked every 1000 steps:
      f32_surrogate  FP32 shifted from the residual surrogate evaluated at the
                     mean zeta (trained here on the batched solver's steady
                     states, ws_training_set),
      f32_physics    FP32 shifted from the per-column Poisson-Boltzmann ions
                     and potential with the electro-osmotic velocity (the start
                     without the network),
      f64_cold       the FP64 path from the uniform noisy cold start.
    Reports MLUPS, the LBM roofline, the FP32 error against the FP64 path from
    the same start after the timed steps, steps and wall time to the cap, the
    final residual and, where the cap came first, the steps to 1e-8
    extrapolated from the residual's decay (steps_to_tol)."""
    import ekpnp
    from ekpnp import Channel, noisy_uniform_state, warmstart as ws
    if d.rank != 0:
        return 0
    ekpnp.set_device(d.local)
    nx, ny = env_int("EK_HET_NX", 8192), env_int("EK_HET_NY", 2048)
    K = args.steps
    cap = env_int("EK_HET_CAP", 20000)
    check = 1000
    spec = dict(nx=nx, ny=ny, kappa_h=64.0, zeta=-2.0, ex=1e-4, diff=0.05, eps=0.01, rest_quirk=False)
    x = np.arange(nx)
    zeta = -2.0 + 1.5 * np.sin(2 * np.pi * x / 1024.0)
    walls = dict(zeta_lo=zeta, zeta_hi=zeta, cp_lo=np.exp(-zeta), cp_hi=np.exp(-zeta), cn_lo=np.exp(zeta),
                 cn_hi=np.exp(zeta))
    peak, peak_kind = measured_peak_gbs()

    def make(storage):
        p = ekpnp.spec_params(spec, storage)
        ch = Channel(p)
        ch.set_wall_profile(**walls)
        if storage != ekpnp.STORE_F64:
            ch.set_rebase_interval(200)
        return ch

    # ---- starts ----
    starts = {}
    n_train = env_int("EK_WS_TRAIN", 8192)
    tr, T, conv, _, gen_s = ws_training_set(n_train, env_int("EK_WS_GEN_CAP", 120_000), 2000)
    ok = np.all(np.isfinite(T), axis=1)
    sg = ws.Surrogate("residual", seed=7)
    t1 = time.perf_counter()
    sg.fit([s_ for s_, o in zip(tr, ok) if o], T[ok], iters=env_int("EK_WS_ITERS", 12000), lr=2e-3)
    train_s = time.perf_counter() - t1
    t1 = time.perf_counter()
    starts["f32_surrogate"] = sg.fields([spec])[0]
    infer_s = time.perf_counter() - t1
    sg.close()
    t1 = time.perf_counter()
    with make(ekpnp.STORE_F32) as ch:
        ch.init_poisson_boltzmann("newton")
        phys = ch.get_fields(("rho", "ux", "uy", "cp", "cn", "psi"))
    phys["ux"] = ws.u_hs(ekpnp.spec_params(spec, 0)) / spec["zeta"] * (zeta[None, :] - phys["psi"])
    starts["f32_physics"] = phys
    phys_s = time.perf_counter() - t1

    def timed(ch, steps):
        ch.sync()
        ch.mark(0)
        ch.step(steps)
        ch.mark(1)
        return ch.elapsed_ms(0, 1)

    def to_steady(ch):
        t0 = time.perf_counter()
        ch.residual(check)
        hist = []
        while ch.steps < cap:
            ch.step(check)
            try:
                r = float(ch.residual(check)[4])
            except ekpnp.EkError:  # non-finite fields: the run diverged
                r = float("nan")
            hist.append(r)
            if not np.isfinite(r) or r < 1e-8:
                break
        return {"steps": int(ch.steps), "residual": hist[-1] if hist else None,
                "wall_s": time.perf_counter() - t0, "to_1e-8": steps_to_tol(hist, check),
                "residual_every_10k": hist[9::10]}

    out = {}
    f32_k = {}
    for arm in ("f32_surrogate", "f32_physics"):
        with make(ekpnp.STORE_F32) as ch:
            ch.set_fields(**starts[arm])
            ch.init_equilibrium()
            ch.step(args.warmup)
            ms = timed(ch, K)
            ch.profile(True)
            ch.step(min(K, 200))
            prof = ch.profile_read()
            ch.profile(False)
            f32_k[arm] = ch.get_fields(("ux", "cp", "cn", "psi"))
            lbm_ms, lbm_n = prof["lbm"]
            per = lbm_ms / max(lbm_n, 1) / 1e3
            out[arm] = {"mlups": nx * ny * K / (ms / 1e3) / 1e6, "ms_per_step": ms / K,
                        "lbm_launch_ms": per * 1e3, "lbm_gbs": nx * ny * 224 / per / 1e9,
                        "lbm_frac": nx * ny * 224 / per / 1e9 / peak, "peak_kind": peak_kind,
                        "step_frac": nx * ny * K / (ms / 1e3) * 248 / 1e9 / peak}
            out[arm].update(to_steady(ch))
    # FP32 error against the FP64 path from the surrogate start (same steps)
    with make(ekpnp.STORE_F64) as ch:
        ch.set_fields(**starts["f32_surrogate"])
        ch.init_equilibrium()
        ch.step(args.warmup + K + min(K, 200))
        f64_k = ch.get_fields(("ux", "cp", "cn", "psi"))
    err = {k: float(np.abs(f32_k["f32_surrogate"][k] - f64_k[k]).max() / np.abs(f64_k[k]).max()) for k in f64_k}
    c = ny // 4
    plug = lambda u: float(u[c:ny - c].mean())
    err["plug"] = abs(plug(f32_k["f32_surrogate"]["ux"]) - plug(f64_k["ux"])) / np.abs(f64_k["ux"]).max()
    # FP64 from the uniform cold start
    with make(ekpnp.STORE_F64) as ch:
        ch.set_fields(**noisy_uniform_state(nx, ny, seed=5))
        ch.init_equilibrium()
        ch.step(args.warmup)
        ms = timed(ch, K)
        out["f64_cold"] = {"mlups": nx * ny * K / (ms / 1e3) / 1e6, "ms_per_step": ms / K}
        out["f64_cold"].update(to_steady(ch))
    est = {a: (out[a]["to_1e-8"] or {}).get("steps") for a in out}
    wall_est = {a: est[a] * out[a]["ms_per_step"] / 1e3 if est[a] else None for a in out}
    line = {"metric": "coupled_mlups", "value": out["f32_surrogate"]["mlups"], "unit": "MLUPS", "n_gpus": 1,
            "steps": K, "warmup": args.warmup, "ms_per_step": out["f32_surrogate"]["ms_per_step"],
            "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seed 5 noise for the cold start; training channels seed 3)",
            "config": {"workload": f"hetero-wall-{nx}x{ny}", "kappa_h": 64.0, "e_x": 1e-4,
                       "zeta": "-2 + 1.5 sin(2 pi x / 1024)", "eps": 0.01, "rest_quirk": False,
                       "cap_steps": cap, "tol": 1e-8, "check_every": check, "train_channels": n_train,
                       "train_usable": int(ok.sum())},
            "start_seconds": {"training_set": gen_s, "training": train_s, "surrogate_inference": infer_s,
                              "physics_start": phys_s},
            **out,
            "f32_error_vs_f64": err,
            "time_to_1e-8_s": wall_est,
            "time_to_1e-8_speedup_vs_f64_cold": {a: (wall_est["f64_cold"] / wall_est[a])
                                                 if wall_est[a] and wall_est["f64_cold"] else None
                                                 for a in ("f32_surrogate", "f32_physics")}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="channel-4096x1024")
    ap.add_argument("--storage", choices=tuple(STORAGE), default="f32")
    ap.add_argument("--hetero", action="store_true",
                    help="the 8192 x 2048 heterogeneous-wall channel: FP32 warm start against FP64 cold start")
    ap.add_argument("--warmstart", action="store_true",
                    help="time to steady state from the learned warm start against the cold start")
    ap.add_argument("--batch", action="store_true",
                    help="the batched workload (512 uneven channels) instead of one channel")
    ap.add_argument("--to-steady", action="store_true",
                    help="with --batch: run the 512 channels from their cold start to residual < 1e-8")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lbm-kernel", choices=("auto", "plain", "tma"), default="auto",
                    help="form of the shifted-storage LBM kernel (bit-identical forms)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    d = Dist(use_pg=args.impl == "ours")
    try:
        if args.impl == "reference":
            rc = run_reference(args, d)
        elif args.hetero:
            rc = run_hetero(args, d)
        elif args.warmstart:
            rc = run_warmstart(args, d)
        elif args.batch:
            args.workload = "batch-512"
            rc = run_batch_steady(args, d) if args.to_steady else run_batch(args, d)
        else:
            rc = run_ours(args, d)
    finally:
        d.close()
    return rc


if __name__ == "__main__":
    sys.exit(main())
