#!/usr/bin/env python
"""Benchmark of the gSQG RK4 hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload hires4096|forced4096|forced1024|ensemble96]
                    [--precision float32|float64]

Default workload ("hires4096"), the largest single-GPU configuration: gSQG
alpha = 0.5 at N = 4096 with RingForcing(kf=100, dk=2, eps=0.1) (host-drawn
phases, one row per step), CombinedDamping(mu=0.05, kf=100, nu=1e-20, p=8),
dt = 5e-5, a k^-3 random-phase initial field (seed 3, rms 1), and two
passive scalars (kappa = 1e-4) forced by a mean gradient G = (1, 0)
(S = -G.u), advanced after theta with the new velocity as the reference's
gSQGSolverWithScalars.step does.  The hyperviscous term is stiff for explicit
RK4 (nu k_max^8 dt >> 2.8), so the integrating-factor scheme is used.
One "step" = one RK4 step of theta and of both scalars; metric = RK4
steps/s.  "forced4096": the same without the scalars (theta alone);
"forced1024": forced-dissipative SQG (alpha = 1) at N = 1024, ring kf = 40,
mu = 0.1, nu = 1e-8, dt = 2e-4, k^4 exp(-(k/10)^2) initial field (seed 2).

Timing: CUDA events on the launching stream; each timed step is bracketed by
its own events and the L2 cache is flushed (a 256 MiB write) between steps
outside the events.  Per-pass durations: every launch site of one step
issues its pass 20 times back to back (programmatic dependent launch
between them, as between the passes of a step) inside one event pair, on a
copy of the state (plan buffers only; the next step recomputes them).
End to end ("e2e"): the same K steps through the public API, the ring
phases copied from pinned host memory and 1/2 <theta^2> read back to the
host every step; the K steps are run three times and the median run is
reported (a host thread stalled by another process shows up in one run).
Multi-GPU (torchrun): every rank runs an independent replica ("replicas
only": a single field does not shard); the elapsed time is the max over
ranks.
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

WORKLOADS = {
    "hires4096": dict(N=4096, alpha=0.5, kf=100.0, dk=2.0, eps=0.1, mu=0.05, kf_damp=100.0, nu=1e-20, p=8, dt=5e-5,
                      ic="kminus3", ic_seed=3, noise_seed=4, scalars=2),
    "forced4096": dict(N=4096, alpha=0.5, kf=100.0, dk=2.0, eps=0.1, mu=0.05, kf_damp=100.0, nu=1e-20, p=8, dt=5e-5,
                       ic="kminus3", ic_seed=3, noise_seed=4, scalars=0),
    "forced1024": dict(N=1024, alpha=1.0, kf=40.0, dk=2.0, eps=0.1, mu=0.1, kf_damp=40.0, nu=1e-8, p=8, dt=2e-4,
                       ic="k4exp", ic_seed=2, noise_seed=1, scalars=0),
}
SCALAR_KAPPA = 1e-4
MEAN_GRADIENT = (1.0, 0.0)
TIMING_REPS = 20


def workload_config(name, w, world):
    """The ``config`` object of the JSON line (identical in both arms)."""
    cfg = {"workload": name, "N": w["N"], "alpha": w["alpha"], "scheme": "ifrk4",
           "ring": [w["kf"], w["dk"], w["eps"]], "damping": [w["mu"], w["kf_damp"], w["nu"], w["p"]],
           "dt": w["dt"], "passive_scalars": w["scalars"], "parallelism": f"replicas x{world}",
           "l2": "flushed between timed steps (256 MiB write outside the step events)"}
    if w["scalars"]:
        cfg["scalar_kappa"] = SCALAR_KAPPA
        cfg["scalar_source"] = f"mean gradient G = {list(MEAN_GRADIENT)}"
    return cfg


def scalar_init(x, y, n):
    """Gaussian blobs of width 0.3 at (2 + i, 3)."""
    return {f"c{i}": np.exp(-((x - 2.0 - i) ** 2 + (y - 3.0) ** 2) / (2 * 0.3**2)) for i in range(n)}


def initial_field(O, g, w):
    if w["ic"] == "k4exp":
        return O.random_phase_field(g, lambda k: k**4 * np.exp(-((k / 10.0) ** 2)), w["ic_seed"])
    return O.random_phase_field(g, lambda k: k ** (-3.0), w["ic_seed"])


def ensemble_members(seed=7):
    """96 realisations: 48 x 128^2, 32 x 256^2, 16 x 512^2; alpha uniform in
    {0, 0.5, 1, 1.5}; 0-3 passive scalars (kappa 1e-4, Gaussian blobs of
    width 0.3 at seeded centres); theta random-phase with a spectrum peaked at
    k0 = 8, rms 1."""
    from pygsquig_b200.ensemble import Member
    from pygsquig_b200.utils.fields import random_phase_field

    rng = np.random.default_rng(seed)
    out = []
    for N, count in ((128, 48), (256, 32), (512, 16)):
        x = np.arange(N) * 2 * np.pi / N
        X, Y = np.meshgrid(x, x, indexing="ij")
        for _ in range(count):
            alpha = float(rng.choice([0.0, 0.5, 1.0, 1.5]))
            th0 = random_phase_field(N, 2 * np.pi, lambda k: (k / 8.0) ** 4 * np.exp(-2 * (k / 8.0) ** 2),
                                     int(rng.integers(1 << 30)))
            ns = int(rng.integers(0, 4))
            sc = []
            for _ in range(ns):
                cx, cy = rng.uniform(0, 2 * np.pi, 2)
                dx = np.angle(np.exp(1j * (X - cx)))
                dy = np.angle(np.exp(1j * (Y - cy)))
                sc.append(np.exp(-(dx**2 + dy**2) / (2 * 0.3**2)))
            out.append(Member(N, alpha, th0, sc, [1e-4] * ns))
    return out


def pass_bytes(N, w_bytes, n_scalars=0, n_src=0):
    """Algorithmic bytes per launch of each pass kind, averaged over the
    launch sites of one step (the kinds of sqg_timing_read).

    h = one half array, (N/2+1) x N complex = ~w N^2 bytes; f = one full
    spectrum, N x N complex = ~2 w N^2 bytes.
      row_inverse   theta in (f), u, v, theta_x, theta_y out (4h)
      row_stage     s=1: J^ rows (h), theta_n (f), acc out (f), 4h;
                    s=2,3: h, theta_n (f), acc in and out (2f), 4h
      row_last      s=4: h, acc in (f), theta_{n+1} out (f)
      col_theta     4h in, J^ (h) out
      row_vel       theta_{n+1} in (f), u, v out (2h), mean-gradient sources (h each)
      col_vel       2h in, u + i v out (f)
      row_scalar_inverse  s in (f), s_x, s_y out (2h)
      col_scalar    2h + u + i v (f) in, J^ (h) out
      row_scalar    s=1: h, s_n (f), acc out (f), 2h; s=2,3: h, f, 2f, 2h;
                    s=4: h, acc in (f), s_{n+1} out (f); plus its source (h)
    Ring-mode tables and phases are negligible.
    """
    h = (N // 2 + 1) * N * 2 * w_bytes
    f = N * N * 2 * w_bytes
    out = {
        "row_inverse": f + 4 * h,
        "row_stage": 5 * h + 8 * f / 3,
        "row_last": h + 2 * f,
        "col_theta": 5 * h,
    }
    if n_scalars:
        out.update({
            "row_vel": f + 2 * h + n_src * h,
            "col_vel": 2 * h + f,
            "row_scalar_inverse": f + 2 * h,
            "col_scalar": 3 * h + f,
            "row_scalar": 2.5 * h + 2.5 * f + (n_src / n_scalars) * h,
        })
    return out


def step_model_bytes(N, w_bytes, n_scalars):
    """The step model: 88 w N^2 for theta, 8 w N^2 once for u, v and 80 w N^2
    per passive scalar."""
    return (88 + (8 if n_scalars else 0) + 80 * n_scalars) * w_bytes * N * N


class ClockSampler:
    """nvidia-smi clocks/throttle sampling around the timed region.

    Started before the warm-up steps (a reader thread timestamps every
    sample); the caller keeps the same load running for about a second after
    the timed steps so that the samples bracket the timed region.
    """

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.p = None
        self.rows = []

    def start(self):
        import threading

        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
            return self

        def reader():
            for line in self.p.stdout:
                self.rows.append((time.time(), line.strip()))

        self.t = threading.Thread(target=reader, daemon=True)
        self.t.start()
        t0 = time.time()
        while not self.rows and time.time() - t0 < 5.0:
            time.sleep(0.05)
        return self

    def stop(self):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self, t_from, t_to):
        vals = []
        for t, line in self.rows:
            if not (t_from <= t <= t_to):
                continue
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                vals.append((float(parts[0]), float(parts[1]), float(parts[2]), parts[3:7]))
            except ValueError:
                continue
        if not vals:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for *_, r in vals for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(v[0] for v in vals), "sm_max_mhz": max(v[1] for v in vals),
                "power_w_max": max(v[2] for v in vals), "reasons": reasons, "samples": len(vals),
                "window": "timed steps plus 1 s of the same load after them"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


E2E_REPEATS = 3  # end-to-end runs of the timed steps; the median is reported


def ncu_traffic(workload, prec, kernel):
    p = os.path.join(ROOT, "profiles", "traffic_per_launch.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(f"{workload}/{prec}/{kernel}")


def _oracle_setup(w):
    """The workload on the float64 oracle: solver (with scalars), forcing,
    damping, initial state, phase generator."""
    from oracle import sqg_oracle as O

    g = O.make_grid(w["N"], 2 * np.pi)
    if w["scalars"]:
        sp = {f"c{i}": {"kappa": SCALAR_KAPPA, "source": O.MeanGradientSource(*MEAN_GRADIENT)}
              for i in range(w["scalars"])}
        s = O.gSQGSolverWithScalars(g, w["alpha"], 0.0, w["p"], passive_scalars=sp, scheme="ifrk4")
        st = s.initialize(theta0=initial_field(O, g, w), scalar_init=scalar_init(g.x, g.y, w["scalars"]))
    else:
        s = O.gSQGSolver(g, w["alpha"], 0.0, w["p"], scheme="ifrk4")
        st = s.initialize(theta0=initial_field(O, g, w))
    ring = O.RingForcing(w["kf"], w["dk"], w["eps"])
    damp = O.CombinedDamping(w["mu"], w["kf_damp"], w["nu"], w["p"])
    rng = np.random.default_rng(w["noise_seed"])
    n_ring = O.ring_mode_count(g, w["kf"], w["dk"])

    def step(st):
        return O.step_forced(s, st, w["dt"], ring, rng.uniform(0, 2 * np.pi, n_ring), damp)

    return st, step


def _oracle_label(w, n, cores):
    what = f"{n} IF-RK4 steps of the {w['N']}^2 workload"
    if w["scalars"]:
        what += f" with {w['scalars']} mean-gradient scalars"
    return what + f" (float64 oracle restatement of the reference algorithm, scipy.fft workers={cores})"


def cpu_baseline(w, seconds=12.0):
    """The float64 CPU restatement of the reference algorithm (9 complex
    FFTs per RHS, forcing rescale with 2 more, 5 per scalar stage), IF-RK4,
    scipy.fft threads = all host cores; a bounded number of steps (at least
    one)."""
    from oracle import sqg_oracle as O

    cores = len(os.sched_getaffinity(0))
    O.set_fft_workers(cores)
    st, step = _oracle_setup(w)
    if w["N"] <= 1024:
        st = step(st)  # warm the FFT plans
    n, t0 = 0, time.perf_counter()
    while True:
        st = step(st)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 200:
            break
    O.set_fft_workers(1)
    return {"value": n / el, "unit": "steps/s", "cores": cores, "kind": "port", "sample": _oracle_label(w, n, cores)}


def run_reference(args, w):
    """The reference arm: the float64 oracle port of the reference's CPU path
    on all host cores, on the same workload; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import sqg_oracle as O

    cores = len(os.sched_getaffinity(0))
    O.set_fft_workers(cores)
    st, step = _oracle_setup(w)
    t0 = time.perf_counter()
    nw = 1  # no JIT to warm: one step warms scipy's FFT plans
    for _ in range(nw):
        st = step(st)
    t_step = (time.perf_counter() - t0) / nw
    k = max(2, min(args.steps, int(90.0 / max(t_step, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(k):
        st = step(st)
    el = time.perf_counter() - t0
    v = k / el
    world = int(os.environ.get("WORLD_SIZE", "1"))
    line = {
        "impl": "reference", "metric": "RK4 steps/s", "value": v, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": k, "warmup": nw, "ms_per_step": 1e3 * el / k, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload, w, world),
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": _oracle_label(w, k, cores)},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hires4096", choices=sorted(WORKLOADS) + ["ensemble96"])
    ap.add_argument("--precision", default="float32", choices=["float32", "float64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variants", default="auto", help="extra measured variants: auto|none")
    ap.add_argument("--profile-range", action="store_true",
                    help="bracket the first timed step with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()
    w = WORKLOADS.get(args.workload, WORKLOADS["hires4096"])
    if args.impl == "reference":
        return run_reference(args, w)
    args.warmup = max(args.warmup, 3)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import pygsquig_b200 as P
    from pygsquig_b200 import replicas
    from pygsquig_b200.build import build
    from pygsquig_b200.utils.diagnostics import compute_total_energy
    from pygsquig_b200.utils.fields import random_phase_field

    if rank == 0:
        build()
    if world > 1:
        dist.barrier()

    def setup(workload, prec, total_steps):
        """Solver, forcing, damping, initial state and the per-step phases
        (host pinned and device copies) of a workload."""
        w = WORKLOADS[workload]
        N = w["N"]
        g = P.make_grid(N, 2 * np.pi)
        ring = P.RingForcing(w["kf"], w["dk"], w["eps"])
        damp = P.CombinedDamping(w["mu"], w["kf_damp"], w["nu"], w["p"])
        if w["ic"] == "k4exp":
            th0 = random_phase_field(N, 2 * np.pi, lambda k: k**4 * np.exp(-((k / 10.0) ** 2)), w["ic_seed"])
        else:
            th0 = random_phase_field(N, 2 * np.pi, lambda k: k ** (-3.0), w["ic_seed"])
        if w["scalars"]:
            sp = {f"c{i}": {"kappa": SCALAR_KAPPA, "source": P.MeanGradientSource(*MEAN_GRADIENT)}
                  for i in range(w["scalars"])}
            s = P.gSQGSolverWithScalars(g, w["alpha"], 0.0, w["p"], precision=prec, scheme="ifrk4",
                                        passive_scalars=sp)
            x = np.arange(N) * 2 * np.pi / N
            X, Y = np.meshgrid(x, x, indexing="ij")
            st = s.initialize(theta0=th0, scalar_init=scalar_init(X, Y, w["scalars"]))
        else:
            s = P.gSQGSolver(g, w["alpha"], 0.0, w["p"], precision=prec, scheme="ifrk4")
            st = s.initialize(theta0=th0)
        n_ring = ring.n_modes(g)
        rng = np.random.default_rng(w["noise_seed"] + 1000 * rank)
        noise_host = torch.from_numpy(rng.uniform(0, 2 * np.pi, size=(total_steps, n_ring))).pin_memory()
        noise_dev = noise_host.to("cuda")
        dt = w["dt"]

        def one(i, st, phases=None):
            ph = noise_dev[i] if phases is None else phases
            return s.step(st, dt, forcing=ring.bind(ph, dt, g), damping=damp)

        return w, g, s, st, one, noise_host, n_ring, ring, damp

    def copy_state(st):
        c = dict(st)
        c["theta_hat"] = st["theta_hat"].clone()
        if st.get("scalar_state") is not None:
            ss = st["scalar_state"]
            c["scalar_state"] = type(ss)(scalars={k: v.clone() for k, v in ss.scalars.items()}, time=ss.time,
                                         diagnostics={})
        return c

    def measure(workload, prec, steps, warmup, with_e2e, with_clocks, profile_range=False):
        w, g, s, st, one, noise_host, n_ring, ring, damp = setup(workload, prec, warmup + steps + 1)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream()
        sampler = ClockSampler(local).start() if with_clocks else None
        for i in range(warmup):
            st = one(i, st)
        torch.cuda.synchronize()
        pl = s.plan(damp, ring)
        # ---- device-resident timed region ----
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t_wall0 = time.time()
        launches = 0
        for k in range(steps):
            if profile_range and k == 0:
                torch.cuda.cudart().cudaProfilerStart()
            evs[k][0].record(stream)
            st = one(warmup + k, st)
            evs[k][1].record(stream)
            if profile_range and k == 0:
                torch.cuda.cudart().cudaProfilerStop()
            launches += pl.last_launch_count()
            flush.zero_()
        torch.cuda.synchronize()
        t_wall1 = time.time()
        if sampler:
            # same load for ~1 s more, so the clock samples bracket the timed steps
            stx = st
            while time.time() - t_wall1 < 1.0:
                for k in range(min(steps, 20)):
                    stx = one(warmup + k, stx)
                torch.cuda.synchronize()
            sampler.stop()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        ms = replicas.max_over_ranks(ms, "cuda")  # slowest rank
        if world > 1:
            dist.barrier()
        th = st["theta_hat"]
        finite = bool(torch.isfinite(torch.view_as_real(th)).all().item())
        res = {"ms": ms, "steps": steps, "launches": launches, "finite": finite, "launch_shape": pl.shape(),
               "clocks": sampler.summary(t_wall0 - 0.1, time.time()) if sampler else None}
        # ---- per-pass durations: each launch site of one step issues its pass
        # TIMING_REPS times back to back inside one event pair (on a copy of the
        # state; the copy's result is discarded) ----
        scratch = copy_state(st)
        flush.zero_()
        torch.cuda.synchronize()
        pl.set_timing(True, reps=TIMING_REPS)
        one(warmup, scratch)
        torch.cuda.synchronize()
        res["kernels"] = pl.timing_read()
        pl.set_timing(False)
        del scratch
        # ---- end to end through the public API with host buffers ----
        if with_e2e:
            # the host drives every step here (a blocking read per step), so a
            # stall of the host thread shows up in the figure: the K steps are
            # timed E2E_REPEATS times and the median run is reported
            out_host = torch.empty(1, dtype=torch.float64).pin_memory()
            runs = []
            for _ in range(E2E_REPEATS):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for k in range(steps):
                    ph = noise_host[warmup + k].to("cuda", non_blocking=True)  # H2D of this step's input
                    st = one(warmup + k, st, phases=ph)
                    half_theta2 = 0.5 * pl.inner(st["theta_hat"], st["theta_hat"])  # D2H of the step's metric
                    out_host[0] = half_theta2
                e1.record(stream)
                torch.cuda.synchronize()
                runs.append(replicas.max_over_ranks(e0.elapsed_time(e1), "cuda"))
            ems = sorted(runs)[len(runs) // 2]
            res["e2e"] = {"value": world * steps / (ems / 1e3), "unit": "steps/s",
                          "h2d_bytes_per_step": int(n_ring * 8), "d2h_bytes_per_step": 8,
                          "runs_steps_per_s": [round(world * steps / (r / 1e3), 2) for r in runs],
                          "reported": f"median of {E2E_REPEATS} runs of the timed steps"}
        del flush
        return res

    def kernel_table(kernels, N, wb, n_scalars, n_src, ms_per_step):
        """Per-pass rows: launches per step, average duration, algorithmic
        bytes and GB/s, share of the summed pass time."""
        bpl = pass_bytes(N, wb, n_scalars, n_src)
        kern = {}
        for name, (ms, cnt) in kernels.items():
            if cnt == 0:
                continue
            avg = ms / cnt
            e = {"launches_per_step": cnt // TIMING_REPS, "avg_us": 1e3 * avg,
                 "us_per_step": 1e3 * avg * (cnt // TIMING_REPS)}
            if name in bpl:
                e["algorithmic_bytes"] = bpl[name]
                e["achieved_gbs"] = bpl[name] / (avg / 1e3) / 1e9
            kern[name] = e
        tot = sum(v["us_per_step"] for v in kern.values())
        for v in kern.values():
            v["share"] = v["us_per_step"] / tot
        summary = {"method": f"each launch site of one step issues its pass {TIMING_REPS} times back to back "
                             "(programmatic dependent launch between them) inside one CUDA event pair",
                   "sum_us_per_step": tot, "ms_per_step_us": 1e3 * ms_per_step,
                   "sum_over_step": tot / (1e3 * ms_per_step),
                   # the passes' times must fit in the event-timed step (2 % for event jitter)
                   "sum_within_step": bool(tot <= 1.02e3 * ms_per_step)}
        return kern, summary

    def compare_precisions(workload, n_steps):
        """FP32 against FP64 on the GPU from the same initial state and phases
        (the FP64 path is checked against the float64 oracle by the tests):
        relative L2 of theta_hat, relative error of the energy and of each
        scalar's variance after n_steps."""
        out = {}
        for prec in ("float32", "float64"):
            w, g, s, st, one, _, _, ring, damp = setup(workload, prec, n_steps)
            for i in range(n_steps):
                st = one(i, st)
            torch.cuda.synchronize()
            pl = s.aux_plan()
            r = {"theta_hat": st["theta_hat"].to(torch.complex128),
                 "energy": compute_total_energy(st["theta_hat"], g, w["alpha"])}
            if st.get("scalar_state") is not None:
                r["scalar_variance"] = {k: pl.scalar_variance(v) for k, v in st["scalar_state"].scalars.items()}
            out[prec] = r
            del s, st
        a, b = out["float32"], out["float64"]
        res = {"steps": n_steps,
               "theta_hat_rel_l2": float(torch.linalg.vector_norm(a["theta_hat"] - b["theta_hat"]).item()
                                         / torch.linalg.vector_norm(b["theta_hat"]).item()),
               "energy_rel": abs(a["energy"] - b["energy"]) / abs(b["energy"]),
               "energy_fp64": b["energy"]}
        if "scalar_variance" in b:
            res["scalar_variance_rel"] = {k: abs(a["scalar_variance"][k] - v) / abs(v)
                                          for k, v in b["scalar_variance"].items()}
        res["reference"] = "FP64 path of this library (pinned to the float64 oracle by the -m gpu tests)"
        return res

    def measure_ensemble(steps, warmup):
        """Config-3 ensemble: every member advanced by graph-replayed multistep."""
        from pygsquig_b200.ensemble import EnsembleSolver

        members = ensemble_members()
        ens = EnsembleSolver(members, nu_p=1e-6, p=8, precision="float32", scheme="ifrk4")
        ens.multistep(warmup, 5e-4)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream()
        e0.record(stream)
        ens.multistep(steps, 5e-4)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ms = replicas.max_over_ranks(ms, "cuda")
        finite = all(bool(torch.isfinite(torch.view_as_real(t)).all().item()) for t in ens.theta)
        n_scal = sum(len(m.scalars0) for m in members)
        # the step model of every member (theta 88 w N^2, u, v 8 w N^2 once and
        # 80 w N^2 per scalar), summed over the members
        model = sum(step_model_bytes(m.N, 4, len(m.scalars0)) for m in members)
        peak, peak_kind = measured_peaks()
        gbs = model / (ms / steps / 1e3) / 1e9
        return {"value": world * steps / (ms / 1e3), "unit": "ensemble steps/s",
                "step_model": {"model_bytes_per_step": model, "model_gbs": gbs, "frac_of_peak": gbs / peak,
                               "peak_kind": peak_kind},
                "member_steps_per_s": world * len(members) * steps / (ms / 1e3), "ms_per_step": ms / steps,
                "members": len(members), "passive_scalars": n_scal, "steps": steps, "finite": finite,
                "gpu_launches_per_step": ens.launches_per_step(),
                "config": "48x128^2 + 32x256^2 + 16x512^2, alpha in {0,.5,1,1.5}, 0-3 scalars, FP32 IF-RK4, "
                          "nu=1e-6 p=8 dt=5e-4, one launch per pass of every RK stage over all sizes and "
                          "scalars (scalars one step behind theta), the step replayed from one CUDA graph, "
                          "no L2 flush (working set > L2)"}

    def measure_closure(steps=300, warmup=20):
        """Closure-vs-DNS GPU time per unit of simulated time: the coarse
        N = 256 FP32 solve with the CNN closure on every RK stage (graph
        replay, forcing split into DNS-sized sub-steps) against the N = 2048
        FP32 DNS step (graph multistep), both with ring forcing kf = 20 and
        CombinedDamping as in the closure experiment.  The spectral error is
        measured in the run: free-running coarse solves with and without the
        closure over 50 eddy times against the filtered DNS's time-mean E(k)
        that the experiment recorded (the DNS spectrum itself is not re-run:
        eight N = 2048 runs take far longer than a bench); the experiment
        report's own figure (windows restarted from the filtered DNS) is
        quoted beside it."""
        import math

        from pygsquig_b200.closure import experiment as X
        from pygsquig_b200.closure.cnn import ClosureCNN
        from pygsquig_b200.closure.model import ClosureSolver, SubgridClosure

        cfg = X.Config()
        here = os.path.join(ROOT, "pygsquig_b200", "closure", "trained")
        wpath = os.path.join(here, "closure_weights.npz")
        if os.path.exists(wpath):
            clo = SubgridClosure.load(wpath)
        else:
            clo = SubgridClosure(ClosureCNN(cfg.N_c, cfg.N_c, max_batch=1), cfg.N_c, 2 * math.pi, 1.0, 1e-3)
        m = int(round(cfg.dt_c / cfg.dt))
        rng = np.random.default_rng(11)
        out = {}
        # coarse closure solve
        g, s, damp, ring = X._solver(cfg, cfg.N_c, cfg.nu)
        runner = ClosureSolver(s, clo, damp, ring, forcing_substeps=m)
        st = s.initialize(theta0=rng.standard_normal((cfg.N_c, cfg.N_c)) * 0.3)
        noise = torch.as_tensor(rng.uniform(0, 2 * math.pi, ((warmup + steps) * m, ring.n_modes(g))), device="cuda")
        st = runner.multistep(st, warmup, cfg.dt_c, noise)
        torch.cuda.synchronize()
        tm = []
        runner.multistep(st, steps, cfg.dt_c, noise[warmup * m:], timer=tm)
        torch.cuda.synchronize()
        coarse_ms = sum(a.elapsed_time(b) for a, b in tm) / steps
        # DNS step
        gf, sf, dampf, ringf = X._solver(cfg, cfg.N_dns, cfg.nu)
        stf = sf.initialize(theta0=rng.standard_normal((cfg.N_dns, cfg.N_dns)) * 0.3)
        nf = 100
        noisef = torch.as_tensor(rng.uniform(0, 2 * math.pi, (nf + 10, ringf.n_modes(gf))), device="cuda")
        stf = sf.multistep(stf, 10, cfg.dt, forcing=ringf, damping=dampf, noise=noisef[:10])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sf.multistep(stf, nf, cfg.dt, forcing=ringf, damping=dampf, noise=noisef[10:])
        e1.record()
        torch.cuda.synchronize()
        dns_ms = e0.elapsed_time(e1) / nf
        out.update({"coarse_ms_per_step": coarse_ms, "coarse_dt": cfg.dt_c, "coarse_N": cfg.N_c,
                    "dns_ms_per_step": dns_ms, "dns_dt": cfg.dt, "dns_N": cfg.N_dns,
                    "gpu_time_ratio": (dns_ms / cfg.dt) / (coarse_ms / cfg.dt_c),
                    "forcing_substeps": m, "weights": "trained" if os.path.exists(wpath) else "random (timing only)"})
        rpath = os.path.join(here, "closure_report.json")
        if os.path.exists(rpath):
            rep = json.load(open(rpath))
            out["report_max_rel_err_E_k_le_kf"] = rep["models"]["closure"]["max_rel_err_E_k_le_kf"]
            out["report_source"] = ("pygsquig_b200/closure/trained/closure_report.json (coarse windows restarted "
                                    "from the filtered DNS every 2 time units)")
            # measured in this run: free-running coarse solves over 50 eddy times against the
            # filtered DNS's time-mean E(k) that the experiment recorded
            t_eddy = rep["eddy_time"]["value"]
            live = {"closure": X.free_running_errors(cfg, clo, rep["E_dns"], eddy_time=t_eddy),
                    "no_closure": X.free_running_errors(cfg, None, rep["E_dns"], eddy_time=t_eddy)}
            out["max_rel_err_E_k_le_kf"] = live["closure"]["max_rel_err_E_k_le_kf"]
            out["live_eval"] = {
                "protocol": "free-running N = 256 solves (dt_c = 1e-3, forcing in DNS-sized sub-steps) from a "
                            "seeded random-phase field with the DNS shell spectrum, 2 time units of spin-up, "
                            "time mean of E(k) over 50 eddy times, per-shell relative error for k <= kf against "
                            "the filtered N = 2048 DNS time mean",
                **{k: {kk: v[kk] for kk in ("max_rel_err_E_k_le_kf", "worst_shell", "rel_err_E", "finite",
                                            "t_avg", "steps")} for k, v in live.items()}}
        return out

    if args.workload == "ensemble96":
        r = measure_ensemble(args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"metric": "RK4 ensemble steps/s", "value": r["value"], "unit": r["unit"], "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                              "data": "synthetic", "config": {"workload": "ensemble96", "detail": r["config"]},
                              "ensemble": r}))
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    peak, peak_kind = measured_peaks()
    prec = args.precision
    main_res = measure(args.workload, prec, args.steps, args.warmup, True, True, args.profile_range)
    wb = 4 if prec == "float32" else 8
    N, ns = w["N"], w["scalars"]
    value = world * main_res["steps"] / (main_res["ms"] / 1e3)
    ms_per_step = main_res["ms"] / main_res["steps"]
    kern, ksum = kernel_table(main_res["kernels"], N, wb, ns, ns, ms_per_step)
    dom = max((k for k in kern if "achieved_gbs" in kern[k]), key=lambda k: kern[k]["share"])
    model_bytes = step_model_bytes(N, wb, ns)
    line = {
        "metric": "RK4 steps/s", "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if prec == "float32" else "f64",
        "data": "synthetic (seeded initial fields and host-drawn ring phases)",
        "config": workload_config(args.workload, w, world),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["achieved_gbs"], "peak": peak,
                     "unit": "GB/s", "frac": kern[dom]["achieved_gbs"] / peak, "peak_kind": peak_kind,
                     "traffic": ncu_traffic(args.workload, prec, dom)},
        "step_model": {"model_bytes_per_step": model_bytes,
                       "formula": "(88 + 8 [scalars > 0] + 80 n_scalars) w N^2",
                       "model_gbs": model_bytes / (ms_per_step / 1e3) / 1e9,
                       "frac_of_peak": model_bytes / (ms_per_step / 1e3) / 1e9 / peak},
        "kernels": kern,
        "kernel_timing": ksum,
        "launch_shape": main_res["launch_shape"],
        "gpu_launches": main_res["launches"],
        "clocks": main_res["clocks"],
        "e2e": main_res["e2e"],
        "finite": main_res["finite"],
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w)
    if args.variants == "auto":
        other = "float64" if prec == "float32" else "float32"
        v = measure(args.workload, other, max(10, args.steps // 2), 3, False, False)
        ow = 8 if other == "float64" else 4
        vms = v["ms"] / v["steps"]
        vk, vsum = kernel_table(v["kernels"], N, ow, ns, ns, vms)
        line["variant_" + other] = {"value": world * v["steps"] / (v["ms"] / 1e3), "unit": "steps/s",
                                    "ms_per_step": vms, "finite": v["finite"],
                                    "step_model_frac_of_peak":
                                        step_model_bytes(N, ow, ns) / (vms / 1e3) / 1e9 / peak,
                                    "kernels": vk, "kernel_timing": vsum}
        line["fp32_vs_fp64"] = compare_precisions(args.workload, 200)
    if args.variants == "auto" and args.workload == "hires4096":
        v = measure("forced4096", prec, args.steps, 3, False, False)
        vms = v["ms"] / v["steps"]
        vk, vsum = kernel_table(v["kernels"], 4096, wb, 0, 0, vms)
        line["variant_forced4096"] = {"value": world * v["steps"] / (v["ms"] / 1e3), "unit": "steps/s",
                                      "ms_per_step": vms, "finite": v["finite"],
                                      "step_model_frac_of_peak": step_model_bytes(4096, wb, 0) / (vms / 1e3) / 1e9 / peak,
                                      "kernels": vk, "kernel_timing": vsum}
    if args.variants == "auto":
        line["variant_ensemble96"] = measure_ensemble(200, 10)
    if args.variants == "auto":
        line["closure_vs_dns"] = measure_closure()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
