#!/usr/bin/env python
"""Benchmark of the MLS-MPM step (particle-steps/s) on B200.

Default workload: the two-material drop (128^3 grid, 2,097,152 particles:
neo-Hookean block + EOS fluid column, slip walls, dt 5e-5), seeded synthetic
inputs.  One bench "step" = one MPM time step of all particles.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload cfg2|cfg1|cfg3|cfg4|cfg3_adjoint]

Our arm prints ONE JSON line: value = whole-job particle-steps/s with state
resident in HBM (device time, CUDA events, max over ranks), e2e = the same
metric through the host-buffer C-ABI call pgmpm_advance_host (pinned host
memory in and out, copies inside the timed region), roofline of the dominant
kernel from live per-kernel CUDA events, and the reference's own CPU solver
timed on the host cores as cpu_baseline.  N > 1 runs independent replicas
(weak scaling; the MPM step of one scene does not shard).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PEAK_FALLBACK_GBS = 6650.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return PEAK_FALLBACK_GBS, "fallback"


# ----------------------------------------------------------------- workloads
def make_workload(name):
    from physgrad_b200 import workloads as W

    if name == "cfg1":
        return W.config1()
    if name == "cfg3" or name == "cfg3_adjoint":
        return W.config3()
    if name == "cfg4":
        return W.config4()
    if name == "cfg5":
        return W.config5()
    return W.config2()


def algorithmic_bytes(N, A, multi_mat):
    """Algorithmic HBM bytes per launch (FP32), in the unfused accounting the
    measurement contract states: P2G reads x, m, v, C, F (100 B per particle,
    +4 B for a material id) and writes 16 B per active node; the grid update
    moves 28 B per active node; G2P reads x and F (48 B) and the 27-node
    velocities (12 B per active node) and writes x, v, C, F (96 B); the whole
    step is 244 B per particle (+4) + 56 B per node, the sort left out."""
    mm = 4 if multi_mat else 0
    return {"p2g": (100 + mm) * N + 16 * A, "g2p": 144 * N + 12 * A, "grid": 28 * A,
            "step": (244 + mm) * N + 56 * A}


def fused_bytes(N, A, multi_mat):
    """The fused step (P2G variant 5): the G2P2G kernel's algorithmic bytes
    are the contract's fused minimum without the grid update, (196 [+4] B per
    particle: x, m, v, C, F read once, x, v, C, F written) + 28 B per active
    node (16 B written by the P2G half, 12 B read by the G2P half); the whole
    step's fused minimum is 196 [+4] B per particle + 56 B per node.  As
    built it moves the sorted order (4 B), x and F (48 B read, 48 B written),
    (m, V0) (8 B) [+ the material id, 4 B] and the next key (4 B) per
    particle; v and C are neither read (G2P recomputes them) nor stored
    between the steps of one call."""
    mm = 4 if multi_mat else 0
    return {"g2p2g": (196 + mm) * N + 28 * A, "step": (196 + mm) * N + 56 * A,
            "g2p2g_compulsory": (112 + mm) * N + 28 * A}


def compulsory_bytes(N, A, multi_mat):
    """What each kernel as split here must move: P2G reads the sorted order
    (4 B) and the payload G2P precomputed (64 B) per particle and adds 16 B
    per active node; G2P reads x, F, (m, V0) (+ material id), writes x, v,
    C, F, the next key and the next payload, and reads 12 B per node.  The
    per-kernel times are taken on single-step calls, whose G2P stores v and
    C; inside a multi-step call (the timed region) the steps before the last
    leave them unstored, 48 B per particle less."""
    mm = 4 if multi_mat else 0
    return {"p2g": 68 * N + 16 * A, "g2p": (220 + mm) * N + 12 * A, "grid": 28 * A}


# FP32 FMA peak of the part (148 SMs x 128 lanes x 2 FLOP x 1.965 GHz): no
# measured FP32 figure is recorded, so the nominal one is used and labelled.
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def kernel_launches_per_step(scenes, n_particles, fused=False):
    """Our kernels per step: the sort, then P2G, the grid update and G2P.
    The solver sorts with the bin sort (5 kernels: count, 2-kernel scan of
    the tile counts, cell offsets + node tiles, scatter) when the grids hold
    at most about 8 cells per particle, else with the radix sort (3 kernels
    per 8-bit pass + the tile marking).  With the fused kernel (bin sort
    only) a chained step is the sort, the grid update and G2P2G."""
    cells = sum(((int(s.n[0]) - 3) // 4 + 1) * ((int(s.n[1]) - 3) // 4 + 1) * ((int(s.n[2]) - 3) // 4 + 1)
                for s in scenes) * 64
    if cells <= 8 * max(n_particles, 1) + (1 << 20):
        return 5 + (2 if fused else 3)
    bits = max(1, int(np.ceil(np.log2(max(2, cells)))))
    passes = (bits + 7) // 8
    return 3 * passes + 1 + 3


# -------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        self.t0 = self.t1 = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            t_end = time.time() + 5.0  # wait for the first sample
            while time.time() < t_end and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(0.25)  # let the sampler record the tail of the window

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        import datetime

        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[1]), float(parts[2]), parts[4:8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        win = rows
        if self.t0 is not None and self.t1 is not None:
            # nvidia-smi timestamps are local wall-clock; compare in the same clock
            win = [r for r in rows if self.t0 - 0.05 <= r[0] <= self.t1 + 0.05]
            if not win:  # window shorter than the sampling period: nearest sample after start
                after = [r for r in rows if r[0] >= self.t0]
                win = after[:1] or rows[-1:]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, _, r in win for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[1] for r in win), "sm_max_mhz": max(r[2] for r in win),
                "reasons": reasons, "samples": len(win)}


# ------------------------------------------------------- reference CPU timing
def reference_cpu_rate(st, scene, total_steps, warmup=1, threads=None):
    """The reference's own CPU solver (physgrad::mpm::MPMSolver<float,64>,
    single-threaded by design) on `threads` host threads: each thread runs an
    independent instance of the whole workload (all particles, the full grid),
    and the `total_steps` timed steps are split over the instances, so the
    host's cores run the solver side by side.  Every instance first runs
    max(1, warmup / threads) untimed steps (first touch of its arrays).
    Returns (particle-steps/s, threads, description)."""
    import ctypes

    from oracle import pyoracle as O

    R = O.ref_lib()
    vp = ctypes.c_void_p
    R.ref_mpm_create.restype = vp
    R.ref_mpm_create.argtypes = [ctypes.c_int64, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float]
    R.ref_mpm_step.argtypes = [vp, ctypes.c_int]
    R.ref_mpm_destroy.argtypes = [vp]
    T = max(1, min(threads or min(os.cpu_count() or 1, 32), total_steps))
    N = st["x"].shape[0]
    x = np.ascontiguousarray(st["x"], np.float32)
    v = np.ascontiguousarray(st["v"], np.float32)
    m = np.ascontiguousarray(st["m"], np.float32)
    V0 = np.ascontiguousarray(st["V0"], np.float32)
    handles = []
    for t in range(T):
        h = R.ref_mpm_create(N, x.ctypes.data, v.ctypes.data, m.ctypes.data, V0.ctypes.data,
                             int(scene.n[0]), int(scene.n[1]), int(scene.n[2]), float(scene.dx), float(scene.dt),
                             float(scene.gravity[0]), float(scene.gravity[1]), float(scene.gravity[2]))
        if not h:
            raise RuntimeError("ref_mpm_create failed")
        handles.append(h)
    per = [total_steps // T + (1 if t < total_steps % T else 0) for t in range(T)]

    def par(ks):
        ths = [threading.Thread(target=R.ref_mpm_step, args=(h, k)) for h, k in zip(handles, ks)]
        t0 = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        return time.perf_counter() - t0

    wu = max(1, -(-warmup // T))
    par([wu] * T)
    dt = par(per)
    for h in handles:
        R.ref_mpm_destroy(h)
    rate = N * total_steps / dt
    desc = (f"{T} independent reference MPMSolver<float,64> instances (single-threaded each), each "
            f"the whole workload ({N} particles on the {scene.n[0]}^3 grid); {total_steps} timed steps "
            f"split over them ({min(per)}-{max(per)} each, after {wu} untimed), wall {dt:.2f} s")
    return rate, T, desc


# ---------------------------------------------------------------- our arm
def run_ours(args, rank, world, device):
    import torch

    import physgrad_b200 as pg
    from physgrad_b200 import _capi as C

    from physgrad_b200.distributed import max_over_ranks, shard_scenes, sum_over_ranks

    torch.cuda.set_device(device)
    scenes, counts, mats, st, meta = make_workload(args.workload)
    scaling = "weak"
    if world > 1 and len(scenes) > 1:
        # batched scenes: disjoint shards, no exchange (strong scaling)
        mine = shard_scenes(counts, world, rank)
        off = np.concatenate([[0], np.cumsum(counts)])
        idx = np.concatenate([np.arange(off[s], off[s + 1]) for s in mine])
        remap = {s: k for k, s in enumerate(mine)}
        st = {k: (None if a is None else a[idx]) for k, a in st.items()}
        st["mat"] = np.array([remap[int(m)] for m in st["mat"]], np.int32)
        scenes, counts, mats = [scenes[s] for s in mine], [counts[s] for s in mine], [mats[s] for s in mine]
        scaling = "strong"
    N = int(sum(counts))
    sim = pg.Simulator(scenes, counts, mats, device=device)
    Cm = st["C"].reshape(N, 9)
    Fm = st["F"].reshape(N, 9)
    sim.upload(st["x"], st["v"], Cm, Fm, st["m"], st["V0"], st["mat"])
    if args.autotune:
        sim.autotune(reps=3)
        sim.upload(st["x"], st["v"], Cm, Fm, st["m"], st["V0"], st["mat"])
    stream = torch.cuda.current_stream()
    # warm-up (also builds the CUDA graph)
    sim.step(args.warmup, stream=stream)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clk:
        torch.cuda.synchronize()
        clk.mark_start()
        ev0.record(stream)
        sim.step(args.steps, stream=stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        clk.mark_end()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, device=f"cuda:{device}")
    n_total = int(sum_over_ranks(N, device=f"cuda:{device}"))
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    flags = sim.status()
    clocks = clk.summary()
    # per-kernel device times: eager launches bracketed by events on the launching stream
    sim.set_profiling(True)
    prof_steps = max(5, min(args.steps, 50))
    sums = {"sort": 0.0, "p2g": 0.0, "grid": 0.0, "g2p": 0.0}
    for _ in range(prof_steps):
        sim.step(1, stream=stream)
        m = sim.metrics()
        sums["sort"] += m["sort_ms"]
        sums["p2g"] += m["p2g_ms"]
        sums["grid"] += m["grid_ms"]
        sums["g2p"] += m["g2p_ms"]
    sim.set_profiling(False)
    sim.status()
    A = sim.metrics()["active_nodes"]
    # the profiled steps ran the fused kernel: no P2G launch of their own
    fused = sim.metrics()["p2g_variant"] == 5 and sums["p2g"] <= 0.02 * max(sums["g2p"], 1e-9)
    kern_ms = {k: v / prof_steps for k, v in sums.items()}
    multi = len(mats) > 1
    alg = algorithmic_bytes(N, A, multi)
    comp = compulsory_bytes(N, A, multi)
    fb = fused_bytes(N, A, multi)
    hbm, peak_kind = peaks()
    prof = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            prof = json.load(f).get(args.workload, {})
    kernels = {}
    for k in (("g2p2g", "grid") if fused else ("p2g", "g2p", "grid")):
        ms_k = kern_ms["g2p"] if k == "g2p2g" else kern_ms[k]
        sec = ms_k * 1e-3
        a_k = fb["g2p2g"] if k == "g2p2g" else alg[k]
        c_k = fb["g2p2g_compulsory"] if k == "g2p2g" else comp[k]
        gbs = a_k / sec / 1e9
        kernels[k] = {"ms": round(ms_k, 5), "alg_bytes": a_k, "achieved_gbs": round(gbs, 1),
                      "frac": round(gbs / hbm, 4), "compulsory_bytes": c_k,
                      "compulsory_gbs": round(c_k / sec / 1e9, 1)}
        if k in prof:
            kernels[k]["dram_bytes_ncu"] = prof[k]["dram"]
            tf = prof[k]["flops"] / sec / 1e12
            kernels[k]["tflops"] = round(tf, 2)
            kernels[k]["tflops_frac_of_fp32_nominal"] = round(tf / FP32_NOMINAL_TFLOPS, 4)
    kernels["sort"] = {"ms": round(kern_ms["sort"], 5)}
    dom = "g2p2g" if fused else max(("p2g", "g2p"), key=lambda k: kern_ms[k])
    traffic = prof[dom]["dram"] if dom in prof else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": kernels[dom]["achieved_gbs"], "peak": hbm,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": kernels[dom]["frac"], "traffic": traffic}
    if "tflops" in kernels[dom]:
        roofline["flops"] = {"achieved": kernels[dom]["tflops"], "peak": round(FP32_NOMINAL_TFLOPS, 1),
                             "peak_kind": "nominal FP32", "unit": "TFLOP/s",
                             "frac": kernels[dom]["tflops_frac_of_fp32_nominal"]}
    step_sec = ms / args.steps * 1e-3
    if fused:
        step_gbs = fb["step"] * n_total / N / step_sec / 1e9
        step_roofline = {"bytes_per_step": fb["step"] * n_total // N, "achieved": round(step_gbs, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(step_gbs / hbm, 4),
                         "note": "whole step incl. the sort, fused-minimum algorithmic bytes 196 B/particle "
                                 "(+4 with material ids) + 56 B/node",
                         "unfused_accounting": {"bytes_per_step": alg["step"] * n_total // N,
                                                "frac": round(alg["step"] * n_total / N / step_sec / 1e9 / hbm, 4)}}
    else:
        step_gbs = alg["step"] * n_total / N / step_sec / 1e9
        step_roofline = {"bytes_per_step": alg["step"] * n_total // N, "achieved": round(step_gbs, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(step_gbs / hbm, 4),
                         "note": "whole step incl. the sort, unfused algorithmic bytes 244 B/particle + 56 B/node"}
    value = n_total * args.steps / (ms * 1e-3)
    launches_per_step = kernel_launches_per_step(scenes, N, fused)

    # e2e: host-buffer C-ABI call (pinned memory in/out), S steps per call
    S = min(args.steps, 100)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    hx, hv, hC, hF = pin(st["x"]), pin(st["v"]), pin(Cm), pin(Fm)
    hm, hV = pin(st["m"]), pin(st["V0"])
    hmat = pin(st["mat"]) if st["mat"] is not None else None
    ox, ov, oC, oF = (pin(np.empty_like(a)) for a in (hx, hv, hC, hF))
    L = pg.lib()
    import ctypes

    sh = ctypes.c_void_p(stream.cuda_stream)
    e2e_times = []
    for it in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        C.check(L.pgmpm_advance_host(sim.handle, hx.ctypes.data, hv.ctypes.data, hC.ctypes.data, hF.ctypes.data,
                                     hm.ctypes.data, hV.ctypes.data, hmat.ctypes.data if hmat is not None else None,
                                     S, ox.ctypes.data, ov.ctypes.data, oC.ctypes.data, oF.ctypes.data, sh))
        e2e_times.append(time.perf_counter() - t0)
    e2e_t = max_over_ranks(statistics.median(e2e_times[1:]), device=f"cuda:{device}")
    h2d = sum(a.nbytes for a in (hx, hv, hC, hF, hm, hV)) + (hmat.nbytes if hmat is not None else 0)
    d2h = sum(a.nbytes for a in (ox, ov, oC, oF))
    e2e = {"value": n_total * S / e2e_t, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d / S,
           "d2h_bytes_per_step": d2h / S, "steps_per_call": S,
           "call": "pgmpm_advance_host: state in from pinned host, S steps, state out to pinned host"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import pyoracle as O

        if O.ref_available():
            ncores = min(os.cpu_count() or 1, 32)
            # batched workloads: the first scene (the reference solves one scene at a time)
            n0 = int(counts[0])
            st0 = {k: st[k][:n0] for k in ("x", "v", "m", "V0")}
            rate, T, desc = reference_cpu_rate(st0, scenes[0], total_steps=2 * ncores, threads=ncores)
            cpu = {"value": rate, "unit": "particle-steps/s", "cores": T, "kind": "reference",
                   "sample": desc + "; physics = the reference CPU path (PIC, gravity, no stress)"}
    cfg = {"workload": meta.get("workload", args.workload), "n_particles": N, "n_scenes": len(scenes),
           "grid": [int(s.n[0]) for s in scenes][:8], "dt": float(scenes[0].dt), "physics": "MLS",
           "materials": meta.get("materials", "fixed-corotated"),
           "l2": f"inputs larger than L2: particle state {N * 104 / 1e6:.0f} MB + grid",
           "parallelism": ("scene shards" if scaling == "strong" else "replicas") if world > 1 else "single",
           "tuning": {k: sim.metrics()[k] for k in ("p2g_block", "p2g_ppt", "g2p_block", "graph_enabled")},
           "active_nodes": A}
    line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": scaling, "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded uniform positions of the configuration's shapes)", "config": cfg,
            "roofline": roofline, "step_roofline": step_roofline, "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps, "clocks": clocks, "device_flags": flags}
    sim.close()
    return line


def _events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_adjoint(args, device=0):
    """Config 3: forward+adjoint (checkpoint every 16) vs plain forward."""
    import torch

    import physgrad_b200 as pg

    torch.cuda.set_device(device)
    scenes, counts, mats, st, meta = make_workload("cfg3")
    N = int(sum(counts))
    steps, k = meta["steps"], 16
    sim = pg.Simulator(scenes, counts, mats, device=device)
    up = lambda s: s.upload(st["x"], st["v"], None, None, st["m"], st["V0"])
    up(sim)
    sim.step(args.warmup)
    e0, e1 = _events()

    def plain():
        up(sim)
        torch.cuda.synchronize()
        e0.record()
        sim.step(steps)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # each time is the median of 3 runs (both sides of the ratio alike)
    reps = 3
    t_plain = float(np.median([plain() for _ in range(reps)]))
    tgt = np.array([0.5, 0.3, 0.5])
    gx = torch.empty(N, 3, device="cuda")

    def fwd_adj():
        up(sim)
        torch.cuda.synchronize()
        e0.record()
        sim.forward_checkpointed(steps, k)
        out = {"x": torch.empty(N, 3, device="cuda"), "v": torch.empty(N, 3, device="cuda"),
               "C": torch.empty(N, 3, 3, device="cuda"), "F": torch.empty(N, 3, 3, device="cuda")}
        sim.download(out)
        com = out["x"].double().mean(0)
        gx.copy_((2 * (com - torch.tensor(tgt, device="cuda")) / N).float().expand(N, 3))
        g = sim.backward({"x": gx})
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), float(((com.cpu().numpy() - tgt) ** 2).sum()), g

    fwd_adj()  # warm-up (allocates the tape)
    runs = [fwd_adj() for _ in range(reps)]
    t_fa = float(np.median([r[0] for r in runs]))
    _, L, g = runs[-1]
    # FD along a uniform v0 shift in y (full size, FP32 forward)
    eps = 1e-3

    def loss_at(v0):
        s2 = pg.Simulator(scenes, counts, mats, device=device)
        s2.upload(st["x"], v0, None, None, st["m"], st["V0"])
        s2.step(steps)
        x = s2.download()["x"].astype(np.float64)
        s2.close()
        return float(((x.mean(0) - tgt) ** 2).sum())

    d = np.zeros_like(st["v"])
    d[:, 1] = 1.0
    fd = (loss_at(st["v"] + eps * d) - loss_at(st["v"] - eps * d)) / (2 * eps)
    ad = float(g["v"][:, 1].sum().item())
    line = {"metric": "particle-steps/s (forward+adjoint)", "value": N * steps / (t_fa * 1e-3),
            "unit": "particle-steps/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
            "ms_per_step": t_fa / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": "differentiable elastic cube (config 3)", "n_particles": N, "grid": 64,
                       "steps": steps, "checkpoint_every": k, "loss": "||COM - (0.5,0.3,0.5)||^2",
                       "timing": f"median of {reps} runs of each, inputs re-uploaded before each"},
            "plain_forward_ms": t_plain, "forward_adjoint_ms": t_fa, "ratio_vs_plain_forward": t_fa / t_plain,
            "loss": L, "grad_check": {"direction": "uniform v0_y shift", "fd": fd, "adjoint": ad,
                                      "rel_err": abs(fd - ad) / abs(fd)},
            "dL_dE": float(g["E"][0].item()),
            "note": "dL/dE of a centre-of-mass loss is ~0: momentum-conserving transfers, no wall contact",
            # the forward records every step's sort; a replayed step sorts
            # again only after a G2P that moved a particle into another cell
            # than the forward did (counted over all the runs above)
            "replays": {"sort_record": True, "replayed_steps_sorted_again": sim.replay_resorts()}}
    sim.close()
    return line


def run_sparse(args, device=0):
    """The two-material drop on a sparse grid (tile pool sized by the
    library's default, max(4096, particles / 32) tiles) against the dense
    grid: device ms per step of one call of K steps each, and the grid and
    sort memory the sparse pool holds against the dense grid's."""
    import torch

    import physgrad_b200 as pg

    torch.cuda.set_device(device)
    scenes, counts, mats, st, meta = make_workload("cfg2")
    N = int(sum(counts))
    res = {}
    for name, kw in (("dense", {}), ("sparse", {"sparse_tiles": 0})):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(device)[0]
        sim = pg.Simulator(scenes, counts, mats, device=device, **kw)
        sim.upload(st["x"], st["v"], st["C"].reshape(N, 9), st["F"].reshape(N, 9), st["m"], st["V0"], st["mat"])
        sim.step(args.warmup)
        torch.cuda.synchronize()
        used = free0 - torch.cuda.mem_get_info(device)[0]
        e0, e1 = _events()
        K = max(args.steps, 20)
        e0.record()
        sim.step(K)
        e1.record()
        torch.cuda.synchronize()
        res[name] = {"ms_per_step": e0.elapsed_time(e1) / K, "device_bytes": int(used), "flags": sim.status()}
        sim.close()
    return {"n_particles": N, "grid": 128, "steps": max(args.steps, 20),
            "dense_ms_per_step": round(res["dense"]["ms_per_step"], 5),
            "sparse_ms_per_step": round(res["sparse"]["ms_per_step"], 5),
            "ratio": round(res["sparse"]["ms_per_step"] / res["dense"]["ms_per_step"], 4),
            "dense_device_bytes": res["dense"]["device_bytes"], "sparse_device_bytes": res["sparse"]["device_bytes"],
            "flags": [res["dense"]["flags"], res["sparse"]["flags"]],
            "note": "device bytes = the solver's allocations (state, grid, sort), read from cudaMemGetInfo"}


def run_batched(args, device=0, adjoint=False, steps=None):
    """Config 4 (or 5 with adjoint): all scenes in one solver vs a loop of
    single-scene solvers (one launch sequence per scene per step).  steps:
    the configuration's own step count when None and --workload names it,
    else min(--steps, the configuration's)."""
    import torch

    import physgrad_b200 as pg

    torch.cuda.set_device(device)
    scenes, counts, mats, st, meta = make_workload("cfg5" if adjoint else "cfg4")
    N = int(sum(counts))
    steps = min(args.steps, meta["steps"]) if steps is None else int(steps)
    off = np.concatenate([[0], np.cumsum(counts)])
    sl = lambda a, s: None if a is None else a[off[s]:off[s + 1]]
    big = pg.Simulator(scenes, counts, mats, device=device)
    big.upload(st["x"], st["v"], None, None, st["m"], st["V0"], st["mat"])
    singles = []
    for s in range(len(scenes)):
        one = pg.Simulator([scenes[s]], [counts[s]], [mats[s]], device=device)
        one.upload(sl(st["x"], s), sl(st["v"], s), None, None, sl(st["m"], s), sl(st["V0"], s))
        singles.append(one)
    e0, e1 = _events()
    k = 8
    gxs = None
    if adjoint:
        gxb = torch.full((N, 3), 1.0 / N, device="cuda")

        def go_big():
            big.forward_checkpointed(steps, k)
            big.backward({"x": gxb})

        def go_loop():
            for s, one in enumerate(singles):
                one.forward_checkpointed(steps, k)
                one.backward({"x": gxb[off[s]:off[s + 1]]})
    else:
        def go_big():
            big.step(steps)

        def go_loop():
            for _ in range(steps):
                for one in singles:
                    one.step(1)

    # warm-up both (graphs, tapes)
    big.step(args.warmup)
    for one in singles:
        one.step(args.warmup)
    if adjoint:
        go_big()
        go_loop()
    torch.cuda.synchronize()
    e0.record()
    go_big()
    e1.record()
    torch.cuda.synchronize()
    t_big = e0.elapsed_time(e1)
    e0.record()
    go_loop()
    e1.record()
    torch.cuda.synchronize()
    t_loop = e0.elapsed_time(e1)
    name = "batched forward+adjoint (config 5)" if adjoint else "batched forward (config 4)"
    line = {"metric": "particle-steps/s" + (" (forward+adjoint)" if adjoint else ""),
            "value": N * steps / (t_big * 1e-3), "unit": "particle-steps/s", "n_gpus": 1, "steps": steps,
            "warmup": args.warmup, "ms_per_step": t_big / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": name, "n_scenes": len(scenes), "n_particles": N, "counts_min": int(min(counts)),
                       "counts_max": int(max(counts)), "grids": sorted(set(int(s.n[0]) for s in scenes)),
                       "checkpoint_every": k if adjoint else None},
            "loop_of_single_scene_value": N * steps / (t_loop * 1e-3), "batched_ms": t_big, "loop_ms": t_loop,
            "speedup_vs_loop": t_loop / t_big}
    big.close()
    for one in singles:
        one.close()
    return line


def run_targets(args, device=0):
    """The task's other targets, measured in the same run as the headline
    line: forward + adjoint of the differentiable elastic cube (262,144
    particles, 256 steps, checkpoints every 16) against its plain forward,
    with the gradient checked against a full-size central difference; the
    64-scene batched forward (500 steps) against a loop of single-scene
    solvers; the 32-scene batched forward + adjoint (128 steps, checkpoints
    every 8) against 32 sequential single-scene forward + adjoint solves.
    Every figure is a device time (CUDA events) at the configuration's own
    step count."""
    import torch

    sparse = run_sparse(args, device)
    torch.cuda.empty_cache()
    adj = run_adjoint(args, device)
    torch.cuda.empty_cache()
    b4 = run_batched(args, device, adjoint=False, steps=500)
    torch.cuda.empty_cache()
    b5 = run_batched(args, device, adjoint=True, steps=128)
    torch.cuda.empty_cache()
    return {
        "adjoint_ratio_vs_plain": round(adj["ratio_vs_plain_forward"], 4),
        "grad_fd_rel_err": adj["grad_check"]["rel_err"],
        "batched_speedup_vs_loop": round(b4["speedup_vs_loop"], 3),
        "batched_adjoint_speedup_vs_loop": round(b5["speedup_vs_loop"], 3),
        "sparse_vs_dense_step_ratio": sparse["ratio"],
        "targets": {
            "sparse_grid_two_material_drop": sparse,
            "differentiable_elastic_cube": {
                "n_particles": adj["config"]["n_particles"], "steps": adj["steps"], "checkpoint_every": 16,
                "plain_forward_ms": round(adj["plain_forward_ms"], 3),
                "forward_adjoint_ms": round(adj["forward_adjoint_ms"], 3),
                "ratio_vs_plain_forward": round(adj["ratio_vs_plain_forward"], 4), "target_ratio": 3.0,
                "timing": adj["config"]["timing"],
                "grad_check": adj["grad_check"],
                "replays": adj["replays"],
                "forward_adjoint_particle_steps_per_s": adj["value"]},
            "batched_forward_64_scenes": {
                "n_particles": b4["config"]["n_particles"], "steps": b4["steps"],
                "batched_ms": round(b4["batched_ms"], 3), "loop_ms": round(b4["loop_ms"], 3),
                "batched_particle_steps_per_s": b4["value"],
                "loop_particle_steps_per_s": b4["loop_of_single_scene_value"],
                "speedup_vs_loop": round(b4["speedup_vs_loop"], 3), "target_speedup": 1.5},
            "batched_forward_adjoint_32_scenes": {
                "n_particles": b5["config"]["n_particles"], "steps": b5["steps"], "checkpoint_every": 8,
                "batched_ms": round(b5["batched_ms"], 3), "loop_ms": round(b5["loop_ms"], 3),
                "batched_particle_steps_per_s": b5["value"],
                "loop_particle_steps_per_s": b5["loop_of_single_scene_value"],
                "speedup_vs_loop": round(b5["speedup_vs_loop"], 3)},
        },
    }


def run_reference(args):
    """Reference arm: the reference's own CPU MPM path on the host cores."""
    from oracle import pyoracle as O

    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libref_mpm.so not built (needs the reference tree)"}
    scenes, counts, mats, st, meta = make_workload(args.workload)
    N = int(sum(counts))
    rate_w, T, desc = None, None, None
    n0 = int(counts[0])  # batched workloads: the first scene (the reference solves one scene at a time)
    st0 = {k: st[k][:n0] for k in ("x", "v", "m", "V0")}
    rate, T, desc = reference_cpu_rate(st0, scenes[0], total_steps=args.steps, warmup=args.warmup)
    line = {"impl": "reference", "metric": "particle-steps/s", "value": rate, "unit": "particle-steps/s",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform, same workload)",
            "config": {"workload": meta.get("workload", args.workload), "n_particles": N,
                       "physics": "reference CPU path (PIC, gravity)"},
            "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": T, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def run_hashgrid(args, device=0):
    """Spatial hash grid (physgrad_b200.SpatialHashGrid over pgmpm_hashgrid_*):
    4,194,304 particles uniform in the unit cube, cell 1/160 (4,096,000 cells,
    not a power of two, so Morton buckets collide as in the reference), radius
    one cell (27 cells per query), every particle also a query.  Build and query
    timed with CUDA events over device arrays; the reference's own host class
    (oracle/_ref) timed on a 1/16 sample for the CPU baseline."""
    import ctypes

    import torch

    import physgrad_b200 as pg
    from physgrad_b200 import _capi as C

    torch.cuda.set_device(device)
    N, cs = 1 << 22, 1.0 / 160
    r = cs
    rng = np.random.default_rng(0)
    p = rng.random((N, 3), dtype=np.float32)
    grid = pg.SpatialHashGrid(cs, (0, 0, 0), (1, 1, 1), max_particles=N, device=device)
    L = C.lib()
    st = torch.cuda.current_stream()
    sh = ctypes.c_void_p(st.cuda_stream)
    pd = torch.tensor(p, device=f"cuda:{device}")
    off = torch.zeros(N + 1, dtype=torch.int64, device=f"cuda:{device}")
    tot = ctypes.c_int64()
    C.check(L.pgmpm_hashgrid_build(grid._h, pd.data_ptr(), N, C.PTR_DEVICE, sh))
    C.check(L.pgmpm_hashgrid_neighbors(grid._h, pd.data_ptr(), N, r, off.data_ptr(), None, 0, ctypes.byref(tot),
                                       C.PTR_DEVICE, sh))
    out = torch.empty(tot.value, dtype=torch.int32, device=f"cuda:{device}")

    def build():
        C.check(L.pgmpm_hashgrid_build(grid._h, pd.data_ptr(), N, C.PTR_DEVICE, sh))

    def query():
        C.check(L.pgmpm_hashgrid_neighbors(grid._h, pd.data_ptr(), N, r, off.data_ptr(), out.data_ptr(), tot.value,
                                           ctypes.byref(tot), C.PTR_DEVICE, sh))

    K = max(3, min(args.steps, 20))
    res = {}
    for name, fn in (("build", build), ("query", query)):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(K):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / K
    build_rate = N / (res["build"] * 1e-3)
    line = {"metric": "particles/s (spatial hash grid build)", "value": build_rate, "unit": "particles/s",
            "n_gpus": 1, "steps": K, "warmup": args.warmup, "ms_per_step": res["build"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/u32", "data": "synthetic (seeded uniform)",
            "config": {"workload": "spatial hash grid", "n_particles": N, "cell_size": cs, "cells": grid.total_cells,
                       "radius": r, "queries": N, "l2": "inputs + table + sort buffers ~ 200 MB > L2"},
            "query": {"ms": res["query"], "queries_per_s": N / (res["query"] * 1e-3),
                      "neighbors_per_query": tot.value / N, "neighbors_per_s": tot.value / (res["query"] * 1e-3)},
            "gpu_launches": {"build": 2 + 3 * 3, "query": 5}}
    # the reference's host class on a 1/16 sample (same density: a smaller cube)
    try:
        from oracle import hashgrid as H

        if not args.no_cpu_baseline and H.reference_available():
            import time

            n = N // 16
            side = float(np.float32((1.0 / 16) ** (1.0 / 3)))
            ps = (p[:n] * side).astype(np.float32)
            t0 = time.perf_counter()
            H.reference_build_and_query(ps, ps[: n // 8], r, cs, (0, 0, 0), (side, side, side))
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": n / dt, "unit": "particles/s (build + queries of 1/8 of them)",
                                    "cores": 1, "kind": "reference",
                                    "sample": f"{n} particles at the same density, {n // 8} queries, one thread"}
    except Exception as e:  # the baseline is optional
        line["cpu_baseline"] = {"unavailable": str(e)[:120]}
    return line


def run_coupling(args, device=0):
    """SPH-MPM contact coupling (pgmpm_sph_coupling, the reference's
    SPHMPMCouplingSystem pair search + forces, src/sph_mpm_coupling.h:453-575)
    and the FSI kinetic-energy monitor (pgmpm_kinetic_energy,
    src/fsi_coupling.h:837-858) on config 2's particles as the MPM side
    (2,097,152 particles, 128^3, uploaded state): 262,144 SPH particles seeded
    uniform in a slab across the elastic block's top face, [0.2, 0.5] x
    [0.49, 0.53] x [0.2, 0.5], contact radius 2 dx.  K calls timed with CUDA
    events on device arrays; e2e through host arrays (SPH state in, forces
    out).  CPU baseline: the reference's own class (oracle/_ref), whose pair
    search tests every SPH x MPM pair, on a sample of SPH particles against all
    MPM particles, one thread."""
    import time

    import torch

    import physgrad_b200 as pg

    torch.cuda.set_device(device)
    scenes, counts, mats, st, meta = make_workload("cfg2")
    N = int(sum(counts))
    sim = pg.Simulator(scenes, counts, mats, device=device)
    sim.upload(st["x"], st["v"], st["C"].reshape(N, 9), st["F"].reshape(N, 9), st["m"], st["V0"], st["mat"])
    n_sph, r = 1 << 18, 2.0 / 128
    rng = np.random.default_rng(11)
    lo, hi = np.array([0.2, 0.49, 0.2]), np.array([0.5, 0.53, 0.5])
    sx = (lo + (hi - lo) * rng.random((n_sph, 3))).astype(np.float32)
    sv = rng.normal(0.0, 0.05, (n_sph, 3)).astype(np.float32)
    dev = f"cuda:{device}"
    dsx, dsv = torch.tensor(sx, device=dev), torch.tensor(sv, device=dev)
    dsf = torch.zeros((n_sph, 3), dtype=torch.float32, device=dev)
    dmf = torch.zeros((N, 3), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    kw = dict(stiffness=1e5, damping=1e3, friction=0.3, radius=r, two_way=True)
    K = max(3, min(args.steps, 20))

    def call():
        dsf.zero_()
        return sim.sph_coupling(dsx, dsv, dsf, dmf, stream=stream, **kw)

    for _ in range(args.warmup):
        _, _, npairs, energy = call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    # kinetic energy monitor
    for _ in range(args.warmup):
        sim.kinetic_energy(stream=stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(K):
        sim.kinetic_energy(stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ke_ms = e0.elapsed_time(e1) / K
    # e2e: host SPH state in, host forces out
    hsf, hmf = np.zeros((n_sph, 3), np.float32), np.zeros((N, 3), np.float32)
    sim.sph_coupling(sx, sv, hsf, hmf, **kw)
    t = []
    for _ in range(3):
        hsf[:] = 0.0
        t0 = time.perf_counter()
        sim.sph_coupling(sx, sv, hsf, hmf, **kw)
        t.append(time.perf_counter() - t0)
    e2e_s = float(np.median(t))
    line = {"metric": "SPH particles/s (SPH-MPM contact coupling)", "value": n_sph / (ms * 1e-3),
            "unit": "SPH particles/s", "n_gpus": 1, "steps": K, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (energy f64)",
            "data": "synthetic (seeded uniform SPH slab over config 2's uploaded MPM state)",
            "config": {"workload": "SPH-MPM contact coupling", "mpm_particles": N, "sph_particles": n_sph,
                       "radius": r, "pairs": int(npairs), "grid": 128},
            "pairs_per_s": npairs / (ms * 1e-3), "energy": energy,
            "kinetic_energy_monitor": {"ms": ke_ms, "particles_per_s": N / (ke_ms * 1e-3)},
            "e2e": {"value": n_sph / e2e_s, "unit": "SPH particles/s", "h2d_bytes_per_step": 2 * sx.nbytes + hsf.nbytes,
                    "d2h_bytes_per_step": hsf.nbytes + hmf.nbytes,
                    "call": "Simulator.sph_coupling with host arrays (pinned staging inside the library)"}}
    try:
        from oracle import pyoracle as O

        if not args.no_cpu_baseline and O.ref_coupling_available():
            out = sim.download()
            # a sample of SPH particles that touch the block, against every MPM particle
            near = np.nonzero(sx[:, 1] < 0.5 + r)[0]
            ns = 256
            pick = near[rng.choice(len(near), ns, replace=False)]
            t0 = time.perf_counter()
            O.ref_sph_coupling(sx[pick], sv[pick], out["x"], out["v"], **kw)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": ns / dt, "unit": "SPH particles/s", "cores": 1, "kind": "reference",
                                    "sample": f"{ns} SPH particles that touch the block against all {N} MPM "
                                              f"particles (the reference tests every pair), wall {dt:.2f} s"}
    except Exception as e:  # the baseline is optional
        line["cpu_baseline"] = {"unavailable": str(e)[:120]}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5", "cfg3_adjoint", "hashgrid",
                                                       "coupling"])
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain", action="store_true", help="cfg4/cfg5: plain bench line instead of the batched comparison")
    ap.add_argument("--no-targets", action="store_true",
                    help="cfg2 at one GPU: leave out the adjoint and batched measurements added to the line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    try:
        if args.workload == "cfg3_adjoint" and world == 1:
            line = run_adjoint(args, local)
        elif args.workload == "hashgrid" and world == 1:
            line = run_hashgrid(args, local)
        elif args.workload == "coupling" and world == 1:
            line = run_coupling(args, local)
        elif args.workload in ("cfg4", "cfg5") and world == 1 and not args.plain:
            line = run_batched(args, local, adjoint=args.workload == "cfg5")
        else:
            line = run_ours(args, rank, world, local)
            if world == 1 and args.workload == "cfg2" and not args.no_targets:
                line.update(run_targets(args, local))
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
