#!/usr/bin/env python
"""Spin-flip attempts/s of the batched uneven-instance workload on B200.

Workload (one "step"): 4096 random-regular QUBO instances, N log-uniform in
[64, 4096], degree uniform in {3..16}, even-indexed instances with integer
couplings in [-8, 8] (bit-exact integer mode), odd-indexed with float32
N(0, 1) couplings widened to f64 (f64 mode), each run as one cell of 64
replicas through an SA schedule with beta linear 0.1 -> 5.0 over 2000 sweeps,
all in one persistent launch. Attempts = sum_i N_i * 64 * sweeps.

  value : attempts/s with the problems resident in HBM (device time, CUDA
          events on the library's stream, max over ranks).
  e2e   : the same metric through the public API from host buffers: create
          (host->device copy of the problems), init, run, read spins and
          energies back (device->host), wall clock.
  parity: the e2e run's spins and energies against the oracle on every 64th
          instance over the full schedule, and the plain arm's against the
          batched run's on its instances.
  --impl reference : the CPU restatement of the reference's Rayon path (the
          oracle), all host threads, on a bounded sample of the workload:
          all instances over a strided subset of the schedule's sweeps.

Multi-GPU: replicas only; every rank runs its own batch (weak scaling), no
collective on the data path.
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
sys.path.insert(0, ROOT)

METRIC = "spin-flip attempts/s: batched vs plain GPU, same energies; serve p50/p99 ms"
UNIT = "attempts/s"
OPS_PER_ATTEMPT = 22  # algorithmic int32 ops per attempt: Xoshiro256++ step (20) + 64-bit compare (2)
CPU_SWEEPS = 32       # sweeps of the strided schedule sample timed on the host
WORKLOAD = ("uneven batch: 4096 random-regular QUBO instances, N log-uniform [64,4096], degree "
            "3..16, half integer couplings [-8,8], half float32 N(0,1); SA beta 0.1->5.0 over 2000 "
            "sweeps; 64 replicas per instance")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--count", type=int, default=4096)
    p.add_argument("--sweeps", type=int, default=2000)
    p.add_argument("--seed", type=int, default=20260)
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--threads-per-block", type=int, default=0)
    p.add_argument("--blocks-per-sm", type=int, default=0)
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--serve-count", type=int, default=128)
    p.add_argument("--serve-rates", type=float, nargs="+", default=[5.0, 100.0, 300.0, 1000.0, 5000.0])
    p.add_argument("--serve-sweeps", type=int, nargs=2, default=[1000, 20000])
    p.add_argument("--serve-budget", type=int, default=1 << 20)
    p.add_argument("--serve-tick-ms", type=float, default=200.0)
    p.add_argument("--config", type=int, default=3, choices=[1, 2, 3, 4],
                   help="3: the batched headline workload; 1, 2, 4: the PT configurations alone")
    p.add_argument("--no-configs", action="store_true", help="skip configs 1, 2, 4 in the headline line")
    p.add_argument("--c4-steps", type=int, default=500)
    return p.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    def __init__(self, ws, rank, backend):
        self.ws, self.rank = ws, rank
        self.pg = None
        if ws > 1:
            import datetime

            import torch.distributed as td
            td.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
            self.td = td

    def barrier(self):
        if self.ws > 1:
            self.td.barrier()

    def max(self, x: float) -> float:
        if self.ws == 1:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self.ws == 1:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.ws > 1:
            self.td.destroy_process_group()


def make_workload(count, seed, sweeps):
    """The seeded batch; cached as a pickle under $BENCH_CACHE when set."""
    import pickle

    from ising_engine_b200 import instances as I
    cache = os.environ.get("BENCH_CACHE")
    path = os.path.join(cache, f"batch_{count}_{seed}.pkl") if cache else None
    if path and os.path.exists(path):
        with open(path, "rb") as f:
            models, seeds = pickle.load(f)
    else:
        models, seeds = I.uneven_batch(count, seed)
        if path:
            os.makedirs(cache, exist_ok=True)
            with open(path, "wb") as f:
                pickle.dump((models, seeds), f)
    temps = I.sa_temps(sweeps)
    return models, seeds, temps


def attempts_of(models, sweeps):
    return float(sum(m.num_vars for m in models)) * 64.0 * sweeps


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = []
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[4]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return None
        loaded = [r for r in rows if r[2] >= 50.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in loaded for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in loaded),
                "reasons": reasons, "samples": len(loaded)}


def host_bytes(models):
    """Bytes the library copies per problem (its device layout): rows u32,
    cols u32, vals f64, lin f64, packed integer entries u32 and per-site
    constants i32 for integer-mode problems, clamp flags/values u8."""
    h2d = 0
    for m in models:
        n, nnz = m.num_vars, m.nnz
        h2d += 4 * (n + 1) + 4 * nnz + 8 * nnz + 8 * n + 2 * n + 32 + 64
        if m.is_integral():
            h2d += 4 * nnz + 4 * n
    return h2d


def run_ours(args):
    ws, rank, local = dist_setup()
    dist = Dist(ws, rank, "gloo")
    from ising_engine_b200 import _ffi
    from ising_engine_b200.engine import BatchEngine

    models, seeds, temps = make_workload(args.count, args.seed + 7919 * rank, args.sweeps)
    attempts = attempts_of(models, args.sweeps)
    eng = BatchEngine(models, seeds, device=local, threads_per_block=args.threads_per_block,
                      blocks_per_sm=args.blocks_per_sm, graph=True)
    eng.init_random()
    tuned = eng.autotune(temps, 100) if not args.no_autotune else None
    shape = dict(item_sites=tuned[0], threads_per_block=tuned[1]) if tuned else {}
    for _ in range(args.warmup):
        eng.run_schedule(temps)
    dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    dev_ms = 0.0
    launches = 0
    for _ in range(args.steps):
        dev_ms += eng.run_schedule(temps)
        launches += eng.last_launches()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    classes = eng.class_report()
    dist.barrier()
    dev_s = dist.max(dev_ms / 1e3)
    total_attempts = dist.sum(attempts * args.steps)
    value = total_attempts / dev_s
    # one step is a group of concurrent class launches (one per size/mode class);
    # the roofline is taken over that group, per step
    per_step_s = dev_ms / 1e3 / args.steps

    # roofline: measured int32 ALU peak and Xoshiro step rate on this GPU
    import ctypes as C
    ip = C.c_double()
    xp = C.c_double()
    _ffi.check(_ffi.lib().ie_probe_peaks(local, C.byref(ip), C.byref(xp)))
    achieved_ops = attempts / per_step_s * OPS_PER_ATTEMPT
    # algorithmic bytes per launch: each sweep reads the CSR row entries
    # (4 B integer / 12 B f64 per entry), the per-site constants, and reads and
    # writes each spin word once per sweep (8 + 8 B), nothing cached.
    alg_bytes = 0.0
    for m in models:
        per_entry = 4 if m.is_integral() else 12
        alg_bytes += args.sweeps * (m.nnz * per_entry + m.num_vars * (8 + 16 + 4))
    hbm_peak = None
    try:
        hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except Exception:
        hbm_peak = 6650.0
    traffic = None
    prof = os.path.join(ROOT, "profiles", "batched_step_traffic.json")
    if os.path.exists(prof):
        try:
            t = json.load(open(prof))
            traffic = t["dram_bytes_per_attempt"] * attempts  # per step
        except Exception:
            traffic = None

    # e2e: one fresh run of the full schedule through the public API from
    # host buffers; its results are the ones the parity checks read
    e2e = None
    w_run = e_run = None
    offs = np.zeros(len(models) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([m.num_vars for m in models])
    if not args.no_e2e:
        ts = []
        for _ in range(max(1, min(args.steps, 2))):
            dist.barrier()
            t1 = time.perf_counter()
            b = BatchEngine(models, seeds, device=local, **shape)
            b.init_random()
            b.run_schedule(temps)
            w = b.spins()
            e = b.energies()
            b.close()
            ts.append(time.perf_counter() - t1)
            w_run, e_run = w, e
        e2e_s = dist.max(float(np.mean(ts)))
        e2e = {"value": dist.sum(attempts) / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(host_bytes(models)),
               "d2h_bytes_per_step": int(w.nbytes + e.nbytes)}

    plain = None
    plain_pick = []
    plain_mismatch = None
    if not args.no_plain and rank == 0:
        order = np.argsort([m.num_vars for m in models])
        plain_pick = [int(order[i]) for i in np.linspace(0, len(order) - 1, 12).astype(int)]
        sub = [models[i] for i in plain_pick]
        pe = BatchEngine(sub, seeds[plain_pick], device=local, **shape)
        pe.init_random()
        ms = pe.run_schedule_plain(temps)
        plain = {"value": attempts_of(sub, len(temps)) / (ms / 1e3), "unit": UNIT,
                 "sample": f"{len(sub)} instances spread over the size range, full {len(temps)}-sweep "
                           "schedule, one launch (one CTA of the batched run's kernel) per instance in sequence",
                 "launches": pe.last_launches()}
        if w_run is not None:
            pw, pen = pe.spins(), pe.energies()
            plain_mismatch = 0
            for j, i in enumerate(plain_pick):
                same = (pw[pe.offsets[j]:pe.offsets[j + 1]] == w_run[offs[i]:offs[i + 1]]).all()
                same = same and pen[j].tobytes() == e_run[i].tobytes()
                plain_mismatch += 0 if same else 1
        pe.close()

    parity = None
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        # the parity run (oracle, full schedule) comes first and warms the
        # host code, as the reference arm's warm-up steps do
        if w_run is not None:
            parity = check_parity(models, seeds, temps, w_run, e_run, offs)
            if plain_mismatch is not None:
                parity["plain_instances"] = len(plain_pick)
                parity["plain_mismatched"] = plain_mismatch
        cpu = cpu_baseline(models, seeds, temps)

    serve = None
    if not args.no_serve and rank == 0:
        serve = run_serve(args, local)

    configs = None
    if not args.no_configs and rank == 0 and ws == 1:
        configs = [run_config(c, local, args) for c in (1, 2, 4)]

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "i32+f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "instances": len(models), "sweeps": args.sweeps,
                       "replicas": 64, "sites": int(sum(m.num_vars for m in models)),
                       "couplings": int(sum(m.nnz for m in models)),
                       "l2": "inputs larger than L2 (problem data %.0f MB per GPU)" % (host_bytes(models) / 1e6),
                       "parallelism": f"replicas x{ws}",
                       "launch": "one persistent launch per work class, replayed from a CUDA graph",
                       "launch_shape": ({"item_sites": tuned[0], "threads_per_cta": tuned[1],
                                         "source": "autotuner (ie_batch_autotune)"} if tuned else "default")},
            "roofline": {"bound": "alu", "achieved": achieved_ops / 1e9, "peak": ip.value / 1e9,
                         "unit": "Gop/s", "frac": achieved_ops / ip.value, "traffic": traffic,
                         "traffic_source": ("scaled: ncu DRAM bytes per attempt of a smaller capture "
                                            "(profiles/batched_step_traffic.json) x attempts per step")
                         if traffic else None,
                         "ops_per_attempt": OPS_PER_ATTEMPT,
                         "peak_source": "measured in-run: int32 LOP3/IADD3 microkernel (ie_probe_peaks)",
                         "per": "step: one group of concurrent class launches",
                         "xoshiro_sol_attempts_per_s": xp.value,
                         "frac_of_xoshiro_sol": (attempts / per_step_s) / xp.value,
                         "hbm": {"achieved_gbs": alg_bytes / per_step_s / 1e9, "peak_gbs": hbm_peak,
                                 "frac": alg_bytes / per_step_s / 1e9 / hbm_peak,
                                 "alg_bytes_per_step": alg_bytes}},
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "plain": plain,
            "batched_over_plain": (value / ws / plain["value"]) if plain else None,
            "wall_s_timed": wall,
            "classes": [{"mode": c[0], "threads_per_lane": c[1], "cap": c[2], "items": c[3],
                         "ms": round(c[4], 1)} for c in classes],
        }
        if parity:
            line["parity"] = parity
        if configs:
            line["configs"] = configs
        if serve:
            line["serve"] = serve
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    eng.close()
    dist.close()


def _pt_run(m, temps, steps, interval, seed, device, warm=0, **kw):
    """Wall time of `steps` PT steps (engine::step with the exchange every
    `interval` steps) on a fresh handle with its state resident on the
    device; returns (seconds, engine)."""
    from ising_engine_b200.engine import Engine
    eng = Engine(m, num_temps=len(temps), seed=seed, exchange_interval=interval, device=device, **kw)
    eng.init_random()
    if warm:
        eng.step(temps, warm)
    t0 = time.perf_counter()
    eng.step(temps, steps)
    return time.perf_counter() - t0, eng


def _pt_parity(m, temps, steps, interval, seed, device, threads):
    """Spin words, energies, swap statistics and stream position after
    `steps` steps from the random init, against the oracle."""
    from oracle import oracle as O
    ref = O.run_schedule(m, np.tile(temps, (steps, 1)), seed, exchange_interval=interval, collect_stats=True,
                         threads=threads)
    _, eng = _pt_run(m, temps, steps, interval, seed, device)
    w, e = eng.spins(), eng.energies()
    att, acc = eng.swap_stats()
    out = {"steps": steps, "mismatched_cells": int((w != ref.words).any(axis=1).sum()),
           "energies_equal": bool(e.tobytes() == ref.energies.tobytes()),
           "stream_position_equal": eng.rng_state()[0] == ref.draws,
           "swap_stats_equal": bool((att == ref.swap_attempts).all() and (acc == ref.swap_accepts).all())
           if len(temps) > 1 else None}
    eng.close()
    return out


def run_config(cfg, device, args):
    """Configs 1, 2, 4 (seeded synthetic instances of their shapes); value =
    attempts/s of the PT steps on the level kernel (wall clock around
    ie_step, state resident on the device)."""
    from ising_engine_b200 import instances as I
    cores = os.cpu_count() or 1
    if cfg == 1:
        m = I.pm_j_lattice(32, 2, seed=2024)
        temps, steps, interval = np.ones(1), 1000, 1
        dt, eng = _pt_run(m, temps, steps, interval, 11, device, warm=20)
        eng.close()
        lane_dt, eng = _pt_run(m, temps, steps, interval, 11, device, warm=20, kernel_form=1)
        eng.close()
        return {"config": 1, "workload": "2D periodic +-J lattice L=32 (N=1024), one cell at beta=1, 1000 sweeps",
                "value": m.num_vars * 64.0 * steps / dt, "unit": UNIT, "s_per_1000_sweeps": dt,
                "per_lane_kernel_s_per_1000_sweeps": lane_dt,
                "parity": _pt_parity(m, temps, steps, interval, 11, device, cores)}
    if cfg == 2:
        m = I.maxcut_gnm(800, 19176, seed=3)
        temps, steps, interval = I.geometric_beta_ladder(32, 0.1, 3.0), 10000, 10
        dt, eng = _pt_run(m, temps, steps, interval, 12, device, warm=10)
        e = eng.energies()
        att, acc = eng.swap_stats()
        eng.close()
        return {"config": 2, "workload": "Max-Cut of G(800, 19176) as QUBO, 32 temperatures beta geometric "
                "0.1..3.0, 64 replicas each, exchange every 10 sweeps, 10^4 sweeps",
                "value": m.num_vars * 64.0 * len(temps) * steps / dt, "unit": UNIT, "seconds": dt,
                "best_cut": float(-e.min()), "mean_cut_coldest": float(-e[-1].mean()),
                "swap_acceptance_per_pair": [round(float(a) / max(int(b), 1), 4) for a, b in zip(acc, att)],
                "parity": _pt_parity(m, temps, 1000, interval, 12, device, cores)}
    m = I.pm_j_lattice(64, 3, seed=64)
    temps, interval = I.geometric_beta_ladder(64, 0.2, 2.0), 5
    steps = max(args.c4_steps, 10)
    dt, eng = _pt_run(m, temps, steps, interval, 99, device, warm=5)
    eng.close()
    pdt, eng = _pt_run(m, temps, 4, interval, 99, device, warm=1, pt_path=3)
    eng.close()
    att = m.num_vars * 64.0 * len(temps)
    return {"config": 4, "workload": "3D periodic +-J lattice L=64 (N=262144), 64 temperatures beta geometric "
            "0.2..2.0, 64 replicas each, exchange every 5 sweeps",
            "value": att * steps / dt, "unit": UNIT, "ms_per_step": dt / steps * 1e3,
            "timed": f"{steps} of the 5000 sweeps (attempts/s is per step; the full run scales linearly)",
            "plain": {"value": att * 4 / pdt, "ms_per_step": pdt / 4 * 1e3,
                      "form": "one launch (one CTA) per temperature cell per step, in sequence"},
            "batched_over_plain": (att * steps / dt) / (att * 4 / pdt),
            "parity": _pt_parity(m, temps, 6, interval, 99, device, cores)}


def run_serve(args, device):
    """Serving streams (config 5): Poisson arrivals of SA requests with N
    log-uniform in [100, 20000], degree 4..32, integer [-8, 8] or float32
    N(0, 1) couplings (half each), SA lengths uniform in [1000, 20000]
    sweeps, at each of the given rates; the pool admits by device-memory
    footprint and ticks until all are done. Latency = result taken - arrival,
    on the host clock. Offered load = rate x mean attempts per request."""
    from ising_engine_b200 import instances as I
    from ising_engine_b200.serve import ServeEngine, serve_stream
    lo, hi = args.serve_sweeps
    reqs = I.serve_requests(args.serve_count, args.seed + 5, sweeps_min=lo, sweeps_max=hi)
    reqs = [(m, s, I.sa_temps(sw)) for (m, s, sw) in reqs]
    attempts = sum(m.num_vars * 64.0 * len(t) for m, _, t in reqs)
    rows = []
    with ServeEngine(device=device, site_budget=args.serve_budget, tick_us=int(args.serve_tick_ms * 1e3)) as srv:
        m0, s0, t0 = reqs[0]
        srv.submit(m0, s0, t0[:2])
        srv.run_all()  # warm-up: kernels loaded, pools touched
        for k, rate in enumerate(args.serve_rates):
            arrivals = I.poisson_arrivals(len(reqs), rate, args.seed + 6 + k)
            tr = serve_stream(srv, reqs, arrivals, keep_results=False)
            s = tr.summary()
            rows.append({"rate_req_per_s": rate, "offered_attempts_per_s": rate * attempts / len(reqs),
                         "attempts_per_s": attempts / s["makespan_s"], "p50_ms": s["p50_ms"],
                         "p99_ms": s["p99_ms"], "mean_ms": s["mean_ms"], "makespan_s": s["makespan_s"],
                         "ticks": s["ticks"], "mean_tick_ms": s["mean_tick_ms"], "gpu_launches": tr.launches})
    cap = max(r["attempts_per_s"] for r in rows)
    return {"rates": rows, "requests": len(reqs), "site_budget": args.serve_budget, "tick_ms": args.serve_tick_ms,
            # the arrival rate the measured throughput sustains: above it the queue grows
            "saturation_req_per_s": cap / (attempts / len(reqs)),
            "mean_attempts_per_request": attempts / len(reqs),
            "stream": f"N log-uniform [100, 20000], degree 4..32, int [-8,8] / f32 N(0,1) half each, "
                      f"SA {lo}..{hi} sweeps (beta 0.1 -> 5.0), Poisson arrivals"}


def parity_sample(models):
    """Every 64th instance (64 of 4096): checked over the full schedule."""
    stride = max(1, len(models) // 64)
    return list(range(0, len(models), stride))


def strided_temps(temps):
    """CPU_SWEEPS sweeps taken at evenly spaced steps of the schedule, so the
    sample spans its whole temperature range."""
    idx = np.linspace(0, len(temps) - 1, min(CPU_SWEEPS, len(temps))).astype(int)
    return np.ascontiguousarray(temps[idx])


def cpu_sample_desc(models, temps):
    return (f"all {len(models)} instances, {min(CPU_SWEEPS, len(temps))} of the {len(temps)} sweeps "
            f"(every {max(1, len(temps) // CPU_SWEEPS)}th temperature of the schedule), parallel over "
            "instances; attempts/s = attempts of the sample / its time")


def cpu_baseline(models, seeds, temps):
    """The oracle (C++ restatement of the reference's Rayon path) on a bounded
    sample of the workload (every instance, a strided subset of the sweeps),
    dynamically scheduled over instances on every host core."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    ts = strided_temps(temps)
    t0 = time.perf_counter()
    O.run_sa_batch(models, seeds, ts, threads=cores, want_words=False)
    dt = time.perf_counter() - t0
    return {"value": attempts_of(models, len(ts)) / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": cpu_sample_desc(models, temps)}


def check_parity(models, seeds, temps, words, energies, offs):
    """The run's spins and energies against the oracle on every 64th instance
    over the full schedule: spin words bit for bit; energies equal to the
    oracle's FP64 recompute of the same words (the level kernel reports the
    recompute) and, for integer couplings, to the oracle's tracked sum; for
    f64 couplings the largest relative gap to the tracked sum."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    pick = parity_sample(models)
    sub = [models[i] for i in pick]
    t0 = time.perf_counter()
    wref, roff, eref = O.run_sa_batch(sub, seeds[pick], temps, threads=cores, want_words=True)
    dt = time.perf_counter() - t0
    bad_w = bad_e = 0
    max_rel = 0.0
    for j, i in enumerate(pick):
        m = models[i]
        w = words[offs[i]:offs[i + 1]]
        if not (w == wref[roff[j]:roff[j] + m.num_vars]).all():
            bad_w += 1
        e = energies[i]
        rec = O.replica_energies(m, w)[0]
        ok = e.tobytes() == rec.tobytes()
        if m.is_integral():
            ok = ok and e.tobytes() == eref[j].tobytes()
        else:
            max_rel = max(max_rel, float((np.abs(e - eref[j]) / np.maximum(np.abs(eref[j]), 1.0)).max()))
        bad_e += 0 if ok else 1
    return {"instances": len(pick), "sweeps": len(temps), "mismatched_words": bad_w,
            "mismatched_energies": bad_e, "max_rel_fp64": max_rel, "fp64_rel_tol": 1e-6,
            "oracle_s": dt, "sample": f"every {len(models) // len(pick)}th instance, full schedule"}


def run_reference(args):
    ws, rank, local = dist_setup()
    if rank != 0:
        return
    models, seeds, temps = make_workload(args.count, args.seed, args.sweeps)
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    # one step = every instance over a strided subset of the sweeps (a few
    # seconds of host work), so no single large instance sets the time
    ts = strided_temps(temps)
    for _ in range(args.warmup):
        O.run_sa_batch(models, seeds, ts, threads=cores, want_words=False)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.run_sa_batch(models, seeds, ts, threads=cores, want_words=False)
    dt = time.perf_counter() - t0
    value = attempts_of(models, len(ts)) * args.steps / dt
    sample = cpu_sample_desc(models, temps) + "; per step"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "i32+f64", "data": "synthetic (seeded)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "instances": len(models), "sweeps": args.sweeps,
                       "replicas": 64, "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.config != 3:
        ws, rank, local = dist_setup()
        if rank == 0:
            out = run_config(args.config, local, args)
            out.update({"metric": METRIC, "higher_is_better": True, "n_gpus": 1, "data": "synthetic (seeded)",
                        "dtype": "i32"})
            print(json.dumps(out))
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
