#!/usr/bin/env python
"""Throughput of the CRKSPH particle step on B200: particle-steps/s.

Workload: the 2D Sedov-Taylor blast of the CRKSPH hot path -- 512 x 512 = 262,144
particles on the periodic unit square, rho = 1, p = 1e-6, gamma = 5/3, E = 1
deposited kernel-weighted at the centre, Wendland C4 with 32 neighbours,
Cullen-Dehnen switch, Heun RK2 with compatible energy, CFL 0.3 time step computed
on the device every step.  One "step" = one full integrator step (two right-hand
sides, neighbour search, finalize, dt).  Inputs are synthetic (seedless lattice).

Arms
  default            the GPU path (libwarpsph_b200) through the reference's API
  --impl reference   the reference's CPU implementation of the path -- here the C
                     oracle that restates it (the reference itself needs NVIDIA Warp
                     and two sibling packages that are not available), timed on the
                     host cores with all threads.
Multi-GPU (torchrun): the path does not shard (one simulation per GPU), so N ranks
run N independent replicas; value = total particle-steps/s, time = max over ranks.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s on 1 B200; DFSPH time-to-tolerance, learned warm-start vs plain"
UNIT = "particle-steps/s"
WORKLOAD = "Sedov 2D CRKSPH 512x512 (262,144 particles), Wendland C4, 32 neighbours, Cullen-Dehnen, RK2, compatible energy"


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--cpu-steps", type=int, default=8, help="steps of the CPU baseline sample (about 1 s each on 16 cores)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--eager", action="store_true",
                    help="time the step as issued from Python every step instead of as a replayed CUDA graph")
    ap.add_argument("--breakdown", action="store_true", help="print a per-kernel time breakdown to stderr")
    ap.add_argument("--no-dfsph", action="store_true", help="skip the DFSPH warm-start comparison")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched delta-SPH ensemble")
    ap.add_argument("--no-compsph", action="store_true", help="skip the CompSPH Sedov 2D throughput")
    ap.add_argument("--no-sedov3d", action="store_true", help="skip the CRKSPH Sedov 3D (128^3) throughput")
    ap.add_argument("--no-mlp", action="store_true", help="skip the warm-start MLP forward throughput")
    ap.add_argument("--mlp-samples", type=int, default=1 << 24, help="feature rows of the MLP forward section")
    ap.add_argument("--nx3d", type=int, default=128, help="lattice size of the CRKSPH Sedov 3D section (nx^3 particles)")
    ap.add_argument("--list-build-only", type=int, default=0, metavar="NX",
                    help="only time three neighbour-list builds of a periodic NX^3 lattice (128 neighbours) and exit")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 50 ms from start() to stop(); summarise() keeps the samples
    whose own timestamps fall inside a given wall-clock window (the timed region), so the
    process start-up happens before the window."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                                          "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def wait_ready(self, timeout: float = 5.0) -> None:
        """Returns once nvidia-smi has printed its first sample (its driver start-up done), so
        that the start-up does not overlap the timed region; gives up after `timeout` s."""
        t0 = time.perf_counter()
        while self.proc is not None and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summarise(self, t0: float, t1: float) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        from datetime import datetime
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[2]), float(parts[3]), parts[6:10]))
            except ValueError:
                continue
        inside = [r for r in rows if t0 - 0.06 <= r[0] <= t1 + 0.06]
        if not inside and rows:   # a window shorter than the sampling period: the nearest sample after its start
            after = [r for r in rows if r[0] >= t0]
            inside = after[:1] if after else rows[-1:]
        reasons = set()
        for r in inside:
            for nm, v in zip(names, r[3]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm = [r[1] for r in inside]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(r[2] for r in inside) if inside else None,
                "reasons": sorted(reasons), "samples": len(inside)}


# ---------------------------------------------------------------------------- byte model
def bytes_accel_dudt(d: int, K: float) -> float:
    """Algorithmic bytes per particle of the fused CRK accel + du/dt pass (FP32):
    per-particle inputs x, v, B, gradA (4d each), H, m, rho, V, A, c, P (+3 words of
    padding-free scalars) = 16d + 40, DvDx and gradB (4d^2 each) = 8d^2; outputs
    dv/dt (4d) and du/dt (4); per interacting pair a 4-byte index and the pairwise
    ap_ij, av_ij the reference's API returns (8d)."""
    return (16 * d + 40 + 8 * d * d) + 4 * d + 4 + K * (4 + 8 * d)


# DRAM bytes (read + write) of one accel pass on this bench's own workload (512^2), from an
# ncu capture of dram__bytes_read.sum + dram__bytes_write.sum: k_crk_accel_dudt 131.6 MB
# read + 132.5 MB written, and the k_crk_pack launch before it 23.1 MB read (its records
# stay in L2 for the accel launch).  Other sizes are scaled by particle count.
ACCEL_TRAFFIC_BYTES_PER_PARTICLE = (131.64e6 + 132.50e6 + 23.08e6) / 262144


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return dict(json.loads(p.read_text()), source="measured")
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


# ---------------------------------------------------------------------------- CPU arm
def cpu_setup(nx: int):
    """Sedov initial state built by the oracle on the host (never the GPU engine)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    from oracle.cases import sedov_state
    from oracle.steps import CRKSPHOracle, SWITCH_CULLEN
    import warpsph_b200 as ws
    cfg, _ = ws.buildConfig(dim=2, domain=ws.buildDomainDescription(1.0, 2, True, "cpu"), kernel=ws.KernelFunctions.Wendland4,
                            targetNeighbors=32, device="cpu")
    sch = ws.CRKSPHConfig()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    params = ws.make_params(cfg, sch)
    st = sedov_state(params, nx, 2, target_neighbors=32.0)
    orc = CRKSPHOracle(params, "f32", switch=SWITCH_CULLEN)
    dt = orc.o.cfl_dt(params, st["supports"], st["internalEnergies"])
    return orc, st, dt


def cpu_time_steps(orc, st, dt, steps: int):
    t0 = time.perf_counter()
    for _ in range(steps):
        st, _, _ = orc.step(st, dt, "rungeKutta2")
    return st, time.perf_counter() - t0


def cpu_baseline(nx: int, steps: int) -> dict:
    """The oracle (C restatement of the reference, all host threads) on a bounded
    sample: `steps` full RK2 steps of the same Sedov workload."""
    orc, st, dt = cpu_setup(nx)
    n = st["masses"].shape[0]
    st, sec = cpu_time_steps(orc, st, dt, steps)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": n * steps / sec, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} RK2 step(s) of the {nx}x{nx} Sedov CRKSPH workload ({n} particles), FP32 oracle, {sec:.2f} s"}


def reference_arm(args, rank: int):
    """Each step is one RK2 step of the full workload on the host cores."""
    if rank != 0:
        return 0
    t0 = time.perf_counter()
    orc, st, dt = cpu_setup(args.nx)
    n = st["masses"].shape[0]
    st, _ = cpu_time_steps(orc, st, dt, min(args.warmup, 1))
    per = []
    for _ in range(args.steps):
        st, sec = cpu_time_steps(orc, st, dt, 1)
        per.append(sec)
    total = sum(per)
    val = n * args.steps / total
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    cb = {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
          "sample": f"{args.steps} RK2 steps of the {args.nx}x{args.nx} Sedov CRKSPH workload ({n} particles), FP32 oracle"}
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD + " -- CPU oracle restating the reference", "particles": n},
            "cpu_baseline": cb, "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t0}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------- DFSPH warm start
def dfsph_dambreak_3d(dev, eval_dx: float = 0.005, train_dx: float = 0.025, train_steps: int = 30, eval_steps: int = 100,
                      samples: int = 200_000) -> dict:
    """DFSPH time-to-tolerance on the 3D dam break, learned warm start against the plain
    initial pressures.

    Case: a 0.5 x 1.0 x 0.5 m water column in the corner of a 1.6 x 1.2 x 0.6 m open tank
    lined with three layers of mDBC wall particles (one mirrored ghost point each),
    g = -9.81, the reference's DFSPH step order (divergence-free solve, explicit Euler,
    density solve in the finalize), rho0 = 1, dt = 0.1 dx s/m.  Training: 32 seeded random
    columns (0.3-0.7 m wide and deep, 0.6-1.0 m tall) at dx = train_dx for train_steps
    steps each, samples of fluid particles every third step, a seeded subset of `samples`
    rows per solve, 25 epochs.  Evaluation: the 0.5 x 1.0 x 0.5 m column at dx = eval_dx;
    every tenth step from step 10, both solves of the same state run from the plain guess
    (the reference's: 0.75 p_prev for the divergence-free solve, 0 for the density solve),
    from the network's, and, for reference, from the previous step's pressure as it is,
    to the 0.01 % density tolerance and the 0.1 %-per-step
    divergence tolerance (1e-3 rho0 / dt on the reference's density-rate residual).  Times
    are CUDA-event GPU ms per solve including the learned guess (features + network)."""
    import numpy as np
    import torch
    from warpsph_b200 import learned, ops
    t0 = time.perf_counter()
    rng = np.random.default_rng(0)
    geos = [(float(rng.uniform(0.3, 0.7)), float(rng.uniform(0.6, 1.0)), s) for s in range(32)]
    data = learned.generate_samples(geos, steps=train_steps, device=dev, dx=train_dx, dt=0.1 * train_dx,
                                    make_case=learned.dam_break_mdbc_3d, collect_every=3, max_samples=samples)
    t_data = time.perf_counter() - t0
    nets, fit = {}, {}
    for mode in (ops.DENSITY, ops.DIVERGENCE_FREE):
        f, tg = data[mode]
        net = learned.WarmStartMLP(dev, seed=mode)
        losses = net.fit(f, tg, epochs=25, batch=4096, lr=2e-3)
        q = torch.quantile(tg.abs().float(), torch.tensor([0.5, 0.99], device=tg.device)).tolist()
        fit[mode] = {"samples": int(f.shape[0]), "final_mse": losses[-1], "target_variance": float(tg.var()),
                     "target_abs_p50": q[0], "target_abs_p99": q[1]}
        nets[mode] = net
    t_fit = time.perf_counter() - t0 - t_data
    case = learned.DamBreakMDBC(dim=3, column=(0.5, 1.0, 0.5), dx=eval_dx, dt=0.1 * eval_dx, device=dev, seed=7)
    tot = learned.compare_warm_starts([(0.5, 1.0, 7)], steps=eval_steps, nets=(nets[ops.DENSITY], nets[ops.DIVERGENCE_FREE]),
                                      skip=10, compare_every=10, df_budget=None, max_iterations=3000, cases=[case], previous=True)
    out = {"case": (f"3D dam break, 0.5 x 1.0 x 0.5 m column at dx {eval_dx} m: {case.n_fluid:,} fluid + {case.n_wall:,} wall "
                    f"particles (+ {case.n_wall:,} ghost points) in a 1.6 x 1.2 x 0.6 m tank, 3 mDBC layers, dt {0.1 * eval_dx:g} s, "
                    f"{eval_steps} steps"),
           "particles": {"fluid": case.n_fluid, "walls": case.n_wall, "ghosts": case.n_wall, "spacing_m": eval_dx}}
    for name, mode in (("density_solve", ops.DENSITY), ("divergence_free_solve", ops.DIVERGENCE_FREE)):
        rows = [(k, arm, st) for (_, k, arm, st) in tot["solves"] if st.mode == mode]
        arms = {}
        for arm in ("plain", "learned", "previous"):
            r = [st for (_, a, st) in rows if a == arm]
            arms[arm] = {"solves": len(r), "iterations_per_solve": sum(st.iterations for st in r) / max(len(r), 1),
                         "ms_per_solve": sum(st.ms for st in r) / max(len(r), 1),
                         "missed_tolerance": sum(int(not st.converged) for st in r),
                         "per_solve": [(k, st.iterations, round(st.ms, 3)) for (k, a, st) in rows if a == arm]}
        out[name] = {"tolerance": ("1e-4 rho0 (reference error definition, one-sided)" if mode == ops.DENSITY
                                   else "1e-3 rho0 per step = 1e-3 rho0 / dt on the mean |residual| rate"),
                     "plain": arms["plain"], "learned": arms["learned"], "previous_pressure": arms["previous"],
                     "time_speedup": arms["plain"]["ms_per_solve"] / max(arms["learned"]["ms_per_solve"], 1e-9),
                     "time_speedup_vs_previous_pressure": arms["previous"]["ms_per_solve"] / max(arms["learned"]["ms_per_solve"], 1e-9),
                     "target_speedup": 2.0 if mode == ops.DENSITY else None}
    out["training"] = {"columns": len(geos), "spacing_m": train_dx, "steps_per_column": train_steps,
                       "density": fit[ops.DENSITY], "divergence_free": fit[ops.DIVERGENCE_FREE],
                       "data_s": round(t_data, 1), "fit_s": round(t_fit, 1)}
    out["wall_s"] = time.perf_counter() - t0
    return out


# ---------------------------------------------------------------------------- batched ensemble
def ensemble_throughput(dev, chunks: int = 6) -> dict:
    """The batched weakly compressible delta-SPH ensemble: 256 periodic 2D unit boxes with
    particle counts log-uniform in [4096, 65536] (seed 0), divergence-free E(k) ~ k^-5/3
    velocity fields at U_max = 1, stiff Tait EOS c0 = 10, delta = 0.1, nu = 1e-3, Wendland
    C2 with the reference's default 50 neighbours, Heun RK2 at the weakly compressible step
    rule per box (viscous and acoustic limits; the acoustic 0.3 h / c0 / k decides).
    One cooperative launch per step for all boxes, steps replayed from a CUDA graph,
    lists rebuilt when the Verlet skin requires it (included in the time)."""
    import torch
    from warpsph_b200.ensemble import Ensemble, build_boxes
    t0 = time.perf_counter()
    E = Ensemble(build_boxes(256, seed=0), dev)
    tune = E.autotune(steps=2)
    E.advance(1 + E.graph_steps)
    torch.cuda.synchronize()
    r0 = E.rebuilds
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    done = E.advance(chunks * E.graph_steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"workload": "256 periodic 2D delta-SPH boxes, N_b log-uniform [4096, 65536], RK2, CUDA graph",
            "particles": E.n, "boxes": len(E.sizes), "verlet_entries_per_particle": E.nnz / E.n,
            "steps": done, "ms_per_step": ms / done, "value": E.n * done / (ms / 1e3), "unit": "particle-steps/s",
            "launches_per_step": "1 cooperative step kernel (+ list rebuilds)", "rebuilds": E.rebuilds - r0,
            "tile": {"lanes": E.tile[0], "block": E.tile[1]},
            "autotune_ms_per_step": {f"{k[0]}x{k[1]}": round(v, 3) for k, v in tune.items()},
            "status": E.status(), "wall_s": time.perf_counter() - t0}


def mlp_forward_throughput(dev, n: int = 1 << 24, reps: int = 20) -> dict:
    """The warm-start network's forward pass on n feature rows (n x 32 B, larger than L2)
    through both tensor-core kernels, tcgen05 (TMEM accumulators) and mma.sync, and the
    training gradient on min(n, 2^22) rows through both."""
    import torch
    from warpsph_b200 import learned, ops
    peaks = load_peaks()
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    theta = learned.WarmStartMLP(dev, seed=7).theta
    feats = torch.randn((n, 8), device=dev, generator=g)
    flops = 2.0 * (8 * 64 + 2 * 64 * 64 + 64)     # per sample, without the K padding
    out = {"samples": n, "flop_per_sample": flops, "peak_bf16_tflops": peaks["bf16_tflops"], "peak_source": peaks["source"]}
    for tc in ("tcgen05", "mma"):
        for _ in range(3):
            ops.mlp_forward(theta, feats, tensor_cores=tc)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            ops.mlp_forward(theta, feats, tensor_cores=tc)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tf = n * flops / (ms * 1e-3) / 1e12
        out[tc] = {"ms": ms, "samples_per_s": n / (ms * 1e-3), "tflops": tf, "frac": tf / peaks["bf16_tflops"]}
    # the training gradient (forward with kept activations, then the backward GEMMs): per
    # sample the forward's FLOPs, the two data-gradient GEMMs (2 x 2 x 64 x 64) and the three
    # weight-gradient GEMMs (2 x (2 x 64 x 64 + 64 x 8))
    gflops = flops + 2 * (2 * 64 * 64) + 2 * (2 * 64 * 64 + 64 * 8)
    ng = min(n, 1 << 22)
    fg, tg = feats[:ng].contiguous(), torch.randn(ng, device=dev, generator=g)
    out["grad"] = {"samples": ng, "flop_per_sample": gflops}
    for tc in ("tcgen05", "mma"):
        for _ in range(3):
            ops.mlp_grad(theta, fg, tg, tensor_cores=tc)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            ops.mlp_grad(theta, fg, tg, tensor_cores=tc)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tf = ng * gflops / (ms * 1e-3) / 1e12
        out["grad"][tc] = {"ms": ms, "samples_per_s": ng / (ms * 1e-3), "tflops": tf, "frac": tf / peaks["bf16_tflops"]}
    st = int(ops.mlp_status(dev).item())
    if st:
        raise RuntimeError(f"tcgen05 MLP kernels reported status {st:#x}")
    return out


def scheme_throughput(dev, scheme: str, dim: int, nx: int, neighbours: int, steps: int, warmup: int, kahan: bool = False,
                      timed_kernel: str = None, bytes_per_particle: float = None, breakdown: bool = False,
                      graph: bool = True) -> dict:
    """particle-steps/s of one compressible scheme on the Sedov blast (device-resident,
    CUDA events, CFL dt on the device every step), the total-energy drift over the timed
    steps from the FP64 conservation sums, and the dominant pair kernel's average launch
    against the measured HBM peak."""
    import torch
    import warpsph_b200 as ws
    from warpsph_b200 import ops
    t0 = time.perf_counter()
    cfg, integ = ws.buildConfig(dim=dim, domain=ws.buildDomainDescription(1.0, dim, True, dev), kernel=ws.KernelFunctions.Wendland4,
                                targetNeighbors=neighbours, integrationScheme=ws.IntegrationSchemeType.rungeKutta2, cflFactor=0.3,
                                device=dev)
    System, State, Config, Update, step, *_ = ws.buildScheme(scheme)
    sch = Config()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    sch.compensatedSums = kahan
    system = ws.buildSedov(System, State, cfg, nx=nx, dim=dim, domainExtent=1.0, E0=1.0, p0=1e-6, gamma=5 / 3,
                           kernel=ws.KernelFunctions.Wendland4, targetNeighbors=neighbours, device=dev)
    params = ws.make_params(cfg, sch)
    n = system.state.masses.shape[0]
    box = {"system": system, "dt": torch.tensor([cfg.dt], device=dev, dtype=torch.float32)}

    def one_step():
        S = box["system"].state
        box["dt"] = ops.cfl_dt(params, S.supports, S.internalEnergies, dt_prev=box["dt"])
        box["system"] = integ.function(state=box["system"], f=step, dt=box["dt"], config=cfg, compParams=sch).state

    for _ in range(warmup):
        one_step()
    torch.cuda.synchronize()
    S = box["system"].state
    c0 = ops.conservation_sums(params, S.masses, S.velocities, S.internalEnergies).cpu().numpy()
    timer = ops.KernelTimer(names={timed_kernel, "neighbors_build"}) if timed_kernel else None
    ops.TIMER = timer
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    gc.collect()
    gc.disable()
    torch.cuda.reset_peak_memory_stats(dev)
    a0 = torch.cuda.memory_stats(dev)
    try:
        e0.record()
        for _ in range(steps):
            one_step()
        e1.record()
        torch.cuda.synchronize()
    finally:
        gc.enable()
    a1 = torch.cuda.memory_stats(dev)
    ops.TIMER = None
    ms = e0.elapsed_time(e1)
    S = box["system"].state
    c1 = ops.conservation_sums(params, S.masses, S.velocities, S.internalEnergies).cpu().numpy()
    out = {"particles": int(n), "neighbours": neighbours, "steps": steps, "ms_per_step": ms / steps,
           "value": n * steps / (ms / 1e3), "unit": UNIT, "compensated_sums": kahan,
           "energy_drift_timed_steps": float(abs(c1[3] - c0[3]) / c0[3]),
           "verlet_entries_per_particle": box["system"].adjacency.nnz / n,
           "allocator_in_timed_region": {key: int(a1.get(key, 0) - a0.get(key, 0)) for key in
                                         ("num_device_alloc", "num_device_free", "num_alloc_retries")}}
    if graph:
        # the same steps recorded once as a CUDA graph (device-decided lists), when the device
        # has room for a second step's worth of buffers (the graph keeps its own)
        torch.cuda.empty_cache()
        free, _ = torch.cuda.mem_get_info(dev)
        need = 2 * max(a1.get("allocated_bytes.all.peak", 0) - a0.get("allocated_bytes.all.current", 0), 1)
        if free < need:
            out["graph"] = {"skipped": f"{free / 2**30:.1f} GiB free, about {need / 2**30:.1f} GiB needed"}
        else:
            from warpsph_b200.stepgraph import StepGraph
            sg = StepGraph(box["system"], integ, step, cfg, sch, dt=box["dt"], warmup=3)
            sg.replay(2)
            torch.cuda.synchronize()
            gc.collect()
            gc.disable()
            try:
                rb0 = sg.rebuilds()
                g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                g0.record()
                sg.replay(steps)
                g1.record()
                torch.cuda.synchronize()
            finally:
                gc.enable()
            sg.check()
            gms = g0.elapsed_time(g1)
            out["eager_value"], out["eager_ms_per_step"] = out["value"], out["ms_per_step"]
            out["value"], out["ms_per_step"] = n * steps / (gms / 1e3), gms / steps
            out["graph"] = {"launches_per_step": sg.launches_per_step, "launches_per_list_rebuild": sg.launches_per_rebuild,
                            "list_rebuilds_timed": sg.rebuilds() - rb0}
            sg.release()
            del sg
            ops.release_device_lists()
            torch.cuda.empty_cache()
    if timer is not None:
        nb = timer.summary().get("neighbors_build")
        out["list_builds_timed"] = nb["launches"] if nb else 0
        k = timer.summary().get(timed_kernel)
        if k:
            peaks = load_peaks()
            ach = bytes_per_particle * n / (k["avg_ms"] / 1e3) / 1e9
            out["kernel"] = {"name": timed_kernel, "avg_launch_ms": k["avg_ms"], "launches": k["launches"],
                             "algorithmic_bytes_per_particle": bytes_per_particle, "achieved_gbs": ach,
                             "frac_of_measured_hbm": ach / peaks["hbm_gbs"]}
    if breakdown:
        # one more step with CUDA events around every library call (after the timed region)
        bt = ops.KernelTimer()
        ops.TIMER = bt
        one_step()
        torch.cuda.synchronize()
        ops.TIMER = None
        out["breakdown_ms_one_step"] = {k: round(v["total_ms"], 3) for k, v in sorted(bt.summary().items(), key=lambda kv: -kv[1]["total_ms"])}
    out["wall_s"] = time.perf_counter() - t0
    return out


# ---------------------------------------------------------------------------- GPU arm
def build_workload(nx, dev):
    import warpsph_b200 as ws
    cfg, integrator = ws.buildConfig(dim=2, domain=ws.buildDomainDescription(1.0, 2, True, dev), kernel=ws.KernelFunctions.Wendland4,
                                     targetNeighbors=32, integrationScheme=ws.IntegrationSchemeType.rungeKutta2, cflFactor=0.3,
                                     device=dev)
    System, State, Config, Update, step, *_ = ws.buildScheme("crkSPH")
    sch = Config()
    sch.gamma = 5 / 3
    sch.viscositySwitchParams.scheme = ws.ViscositySwitch.CullenDehnen2010
    system = ws.buildSedov(System, State, cfg, nx=nx, dim=2, domainExtent=1.0, E0=1.0, p0=1e-6, gamma=5 / 3,
                           kernel=ws.KernelFunctions.Wendland4, targetNeighbors=32, device=dev)
    return cfg, sch, integrator, step, system


E2E_FIELDS = ["positions", "velocities", "internalEnergies", "supports", "masses", "densities", "alpha0s", "alphas", "divergence"]


def e2e_graph(sg, steps: int, world: int, barrier) -> dict:
    """particle-steps/s through the recorded step with host buffers: every step copies the
    state it starts from (recorded beforehand from the same run) from pinned host memory
    into the graph's inputs, replays the step and copies the resulting state back to
    pinned host memory.  The uploads and downloads run on a copy stream, overlapped with
    the neighbouring steps; the time is the whole sequence on the device clock."""
    import torch
    import torch.distributed as dist
    dev = sg.device
    n = sg.n
    traj = []
    for _ in range(2 + steps):
        S = sg.inputs.state
        traj.append({f: getattr(S, f).detach().cpu().pin_memory() for f in E2E_FIELDS})
        sg.replay(1)
    torch.cuda.synchronize()
    h2d = sum(t.numel() * t.element_size() for t in traj[0].values())
    host_out = [{f: torch.empty_like(traj[0][f]).pin_memory() for f in E2E_FIELDS} for _ in range(2)]
    comp = torch.cuda.current_stream(dev)
    copy = torch.cuda.Stream(dev)
    d_in = [{f: torch.empty_like(getattr(sg.inputs.state, f)) for f in E2E_FIELDS} for _ in range(2)]
    d_out = [{f: torch.empty_like(getattr(sg.inputs.state, f)) for f in E2E_FIELDS} for _ in range(2)]

    def upload(k):
        with torch.cuda.stream(copy):
            for f in E2E_FIELDS:
                d_in[k % 2][f].copy_(traj[k][f], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(copy)
        return ev

    def run(k0, count):
        ev = upload(k0)
        for k in range(k0, k0 + count):
            comp.wait_event(ev)
            sg.load_state(d_in[k % 2])
            if k + 1 < k0 + count:
                ev = upload(k + 1)        # the next step's inputs cross while this step computes
            sg.replay(1)
            S = sg.system.state            # the result leaves the graph's buffers before the next replay
            torch._foreach_copy_([d_out[k % 2][f] for f in E2E_FIELDS], [getattr(S, f) for f in E2E_FIELDS], non_blocking=True)
            done = torch.cuda.Event()
            done.record(comp)
            copy.wait_event(done)
            with torch.cuda.stream(copy):   # and crosses to the host while the next step computes
                for f in E2E_FIELDS:
                    host_out[k % 2][f].copy_(d_out[k % 2][f], non_blocking=True)
        comp.wait_stream(copy)

    run(0, 2)
    barrier()
    torch.cuda.synchronize()
    gc.collect()
    gc.disable()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run(2, steps)
    e1.record()
    torch.cuda.synchronize()
    gc.enable()
    te = torch.tensor([e0.elapsed_time(e1)], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    return {"value": n * steps * world / (float(te.item()) / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": h2d, "steps": steps, "path": "recorded step (CUDA graph)",
            "inputs": "each step uploads the state it starts from, recorded from the same run beforehand"}


def gpu_arm(args, rank: int, world: int):
    import torch
    import torch.distributed as dist
    import warpsph_b200 as ws
    from warpsph_b200 import _capi, ops

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    cfg, sch, integ, step, system = build_workload(args.nx, dev)
    params = ws.make_params(cfg, sch)
    n = system.state.masses.shape[0]
    L = _capi.lib()

    state = {"system": system, "dt": torch.tensor([cfg.dt], device=dev, dtype=torch.float32)}

    def one_step():
        S = state["system"].state
        dt = ops.cfl_dt(params, S.supports, S.internalEnergies, dt_prev=state["dt"])
        state["dt"] = dt
        state["system"] = integ.function(state=state["system"], f=step, dt=dt, config=cfg, compParams=sch).state

    def barrier():
        if world > 1:
            dist.barrier()

    clocks = ClockSampler(dev.index)
    clocks.start()
    clocks.wait_ready()
    for _ in range(max(args.warmup, 0)):
        one_step()
    torch.cuda.synchronize()

    # ------------------------------------------------ the step issued from Python (eager)
    timer = ops.KernelTimer(names={"crk_accel_dudt"})
    barrier()
    torch.cuda.synchronize()
    # as timeit does: one collection before the timed region and none inside it, so a
    # generation-2 sweep of the interpreter heap does not land between two launches
    gc.collect()
    gc.disable()
    tw0 = time.time()
    mem0 = torch.cuda.memory_stats(dev)
    launches0 = L.sph_launch_count()
    ops.TIMER = timer
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        one_step()
    ev1.record()
    torch.cuda.synchronize()
    ops.TIMER = None
    launches = L.sph_launch_count() - launches0
    gc.enable()
    mem1 = torch.cuda.memory_stats(dev)
    # device allocations by torch's caching allocator inside the timed region (each one a
    # cudaMalloc / cudaFree, which synchronise the device)
    allocator = {k: int(mem1.get(k, 0) - mem0.get(k, 0)) for k in ("num_device_alloc", "num_device_free", "num_alloc_retries")}
    tw1 = time.time()

    # ------------------------------------------------ the step recorded once as a CUDA graph
    # (device-decided neighbour lists: no step reads the device; one graph launch per step)
    sg = None
    graph_info = None
    if not args.eager:
        from warpsph_b200.stepgraph import StepGraph
        t_cap = time.perf_counter()
        sg = StepGraph(state["system"], integ, step, cfg, sch, dt=state["dt"], warmup=3)
        torch.cuda.synchronize()
        t_cap = time.perf_counter() - t_cap
        sg.replay(max(args.warmup, 3))
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        gc.collect()
        gc.disable()
        rb0 = sg.rebuilds()
        gw0 = time.time()
        gmem0 = torch.cuda.memory_stats(dev)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        with torch.cuda.nvtx.range("recorded_steps"):    # lets a profiler select the timed replays
            sg.replay(args.steps)
        g1.record()
        torch.cuda.synchronize()
        gc.enable()
        gmem1 = torch.cuda.memory_stats(dev)
        gw1 = time.time()
        barrier()
        sg.check()
        g_ms = g0.elapsed_time(g1)
        rebuilds = sg.rebuilds() - rb0
        graph_info = {"ms": g_ms, "wall": (gw0, gw1),
                      "launches": sg.launches_per_step * args.steps + sg.launches_per_rebuild * rebuilds,
                      "launches_per_step": sg.launches_per_step, "launches_per_list_rebuild": sg.launches_per_rebuild,
                      "list_rebuilds_timed": rebuilds, "capture_s": round(t_cap, 3),
                      "list_capacity": sg.lists[0].capacity if sg.lists else None,
                      "allocator": {k: int(gmem1.get(k, 0) - gmem0.get(k, 0))
                                    for k in ("num_device_alloc", "num_device_free", "num_alloc_retries")}}

    barrier()
    clocks.stop()
    clock_info = clocks.summarise(tw0, graph_info["wall"][1] if graph_info else tw1)
    eager_ms = ev0.elapsed_time(ev1)
    t = torch.tensor([graph_info["ms"] if graph_info else eager_ms, eager_ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max, eager_ms_max = float(t[0].item()), float(t[1].item())
    value = n * args.steps * world / (ms_max / 1e3)
    eager = {"value": n * args.steps * world / (eager_ms_max / 1e3), "ms_per_step": eager_ms_max / args.steps,
             "launches_per_step": launches / max(args.steps, 1), "allocator_in_timed_region": allocator}
    if graph_info:
        launches = graph_info["launches"]
        allocator = graph_info["allocator"]
    ksum = timer.summary().get("crk_accel_dudt", {"launches": 0, "avg_ms": float("nan")})

    # roofline of the dominant kernel
    S = state["system"].state
    adj = state["system"].adjacency
    dvec = S.positions[adj.i] - S.positions[adj.j]
    r = torch.linalg.norm(dvec - torch.round(dvec), dim=1)   # unit periodic box: minimum image
    Hmax = torch.maximum(S.supports[adj.i], S.supports[adj.j])
    K_meas = float((r < Hmax).sum().item()) / n
    nnz_per = adj.nnz / n
    per_particle = bytes_accel_dudt(2, 32.0)
    peaks = load_peaks()
    achieved = per_particle * n / (ksum["avg_ms"] / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": ACCEL_TRAFFIC_BYTES_PER_PARTICLE * n / 1e9,
                "traffic_unit": "GB per launch of the pack + accel pass (ncu dram__bytes_read+write on this 512^2 workload)",
                "kernel": "k_crk_accel_dudt",
                "algorithmic_bytes_per_particle": per_particle, "model_K": 32, "measured_interacting_per_particle": K_meas,
                "verlet_entries_per_particle": nnz_per, "avg_launch_ms": ksum["avg_ms"], "launches_timed": ksum["launches"],
                "peak_source": peaks.get("source")}

    breakdown = None
    if args.breakdown:
        bt = ops.KernelTimer()
        ops.TIMER = bt
        for _ in range(3):
            one_step()
        torch.cuda.synchronize()
        ops.TIMER = None
        breakdown = bt.summary()

    # ------------------------------------------------ end-to-end through the API with host buffers
    e2e = None
    if not args.no_e2e and sg is not None:
        e2e = e2e_graph(sg, max(3, args.steps), world, barrier)
    elif not args.no_e2e:
        fields = E2E_FIELDS
        e2e_steps = max(3, args.steps // 2)
        # the inputs of 2 + e2e_steps consecutive steps of the run, recorded into pinned host
        # memory beforehand: every step of the end-to-end leg uploads the state that step
        # really starts from, so its neighbour lists are kept or rebuilt as in the
        # device-resident run
        traj = []
        for _ in range(2 + e2e_steps):
            S = state["system"].state
            traj.append({f: getattr(S, f).detach().cpu().pin_memory() for f in fields})
            one_step()
        torch.cuda.synchronize()
        S = state["system"].state
        host_in = traj[0]
        # two pinned result buffers: step k's download may still run while step k+1 computes
        host_out = [{f: torch.empty_like(host_in[f]).pin_memory() for f in fields} for _ in range(2)]
        h2d = sum(t.numel() * t.element_size() for t in host_in.values())
        d2h = h2d
        comp = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(dev)
        # two device input sets: step k+1's inputs land in one while step k reads the other
        d_in = [{f: torch.empty_like(getattr(S, f)) for f in fields} for _ in range(2)]

        def upload(k):
            """Copies step k's recorded inputs from pinned host memory on the copy stream."""
            with torch.cuda.stream(copy):
                for f in fields:
                    d_in[k % 2][f].copy_(traj[k][f], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(copy)
            return ev

        def run(k0, steps):
            ev = upload(k0)
            for k in range(k0, k0 + steps):
                comp.wait_event(ev)
                S = state["system"].state
                for f in fields:
                    setattr(S, f, d_in[k % 2][f])
                if k + 1 < k0 + steps:
                    ev = upload(k + 1)      # the next step's inputs cross while this step computes
                one_step()
                done = torch.cuda.Event()
                done.record(comp)
                copy.wait_event(done)
                S = state["system"].state
                with torch.cuda.stream(copy):   # this step's result crosses while the next step computes
                    for f in fields:
                        t = getattr(S, f)
                        t.record_stream(copy)
                        host_out[k % 2][f].copy_(t, non_blocking=True)
            comp.wait_stream(copy)

        run(0, 2)   # untimed: settles the allocator's pools for this pattern
        barrier()
        torch.cuda.synchronize()
        gc.collect()
        gc.disable()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run(2, e2e_steps)
        e1.record()
        torch.cuda.synchronize()
        gc.enable()
        ems = e0.elapsed_time(e1)
        te = torch.tensor([ems], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": n * e2e_steps * world / (float(te.item()) / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": e2e_steps,
               "inputs": "each step uploads the state it starts from, recorded from the same run beforehand"}

    dfsph = None
    if rank == 0 and world == 1 and not args.no_dfsph:
        dfsph = dfsph_dambreak_3d(dev)
    ens = None
    if rank == 0 and world == 1 and not args.no_ensemble:
        ens = ensemble_throughput(dev)

    mlp = None
    if rank == 0 and world == 1 and not args.no_mlp:
        mlp = mlp_forward_throughput(dev, n=args.mlp_samples)
    comp = None
    if rank == 0 and world == 1 and not args.no_compsph:
        d, K = 2, 32.0
        comp = scheme_throughput(dev, "compSPH", 2, args.nx, 32, steps=args.steps, warmup=args.warmup,
                                 timed_kernel="compsph_accel_dudt", bytes_per_particle=(8 * d + 28) + (4 * d + 8) + K * (4 + 8 * d))
        comp["workload"] = f"Sedov 2D CompSPH {args.nx}x{args.nx}, Wendland C4, 32 neighbours, Cullen-Dehnen, RK2, compatible energy"
    s3 = None
    if rank == 0 and world == 1 and not args.no_sedov3d:
        s3 = scheme_throughput(dev, "crkSPH", 3, args.nx3d, 128, steps=5, warmup=3, kahan=True, timed_kernel="crk_accel_dudt",
                               bytes_per_particle=bytes_accel_dudt(3, 128.0), breakdown=True)
        s3["workload"] = (f"Sedov 3D CRKSPH {args.nx3d}^3 ({args.nx3d ** 3:,} particles), Wendland C4, 128 neighbours, Cullen-Dehnen, RK2, "
                          "Kahan sums")

    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(args.nx, args.cpu_steps)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "particles": n, "nx": args.nx, "parallelism": f"replicas x{world}",
                           "l2": "working set larger than L2 (pair arrays ~0.7 GB per step), no flush needed"},
                "roofline": roofline, "cpu_baseline": cb, "e2e": e2e, "gpu_launches": int(launches), "clocks": clock_info,
                "allocator_in_timed_region": allocator,
                "step_path": ("one CUDA graph launch per step (StepGraph), device-decided neighbour lists" if graph_info
                              else "issued from Python every step"),
                "graph": ({k: v for k, v in graph_info.items() if k not in ("wall", "ms", "allocator")} if graph_info else None),
                "eager": eager,
                "dfsph_dambreak_3d": dfsph, "ensemble": ens, "compsph": comp, "sedov3d": s3, "mlp_forward": mlp}
        if breakdown is not None:
            line["breakdown_ms"] = {k: round(v["total_ms"] / 3, 4) for k, v in breakdown.items()}
        print(json.dumps(line), flush=True)
    return 0


def list_build_only(nx: int) -> int:
    """Three full neighbour-list builds (sph_neighbors_build through ops.buildVerletList)
    of a periodic nx^3 lattice with Wendland C4 supports for 128 neighbours; prints one JSON
    line with the wall time of each build."""
    import torch
    import warpsph_b200 as ws
    from warpsph_b200 import ops
    dev = torch.device("cuda")
    dom = ws.buildDomainDescription(1.0, 3, True, dev)
    cfg, _ = ws.buildConfig(dim=3, domain=dom, kernel=ws.KernelFunctions.Wendland4, targetNeighbors=128, device=dev)
    x, H, _, _ = ws.buildPointCloud(nx, dom, cfg.targetNeighbors, device=dev)
    p = ws.make_params(cfg)
    ms, entries = [], 0.0
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        adj = ops.buildVerletList(x, H, p, cfg.verletScale)
        torch.cuda.synchronize()
        ms.append(1e3 * (time.perf_counter() - t0))
        entries = adj.nnz / x.shape[0]
    print(json.dumps({"list_build": {"particles": int(x.shape[0]), "verlet_entries_per_particle": entries, "ms": ms}}), flush=True)
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.list_build_only:
        return list_build_only(args.list_build_only)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)
    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    try:
        return gpu_arm(args, rank, world)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
