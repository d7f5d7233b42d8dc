"""Benchmark: DOF-updates/s of the fused FP64 DGSEM tendency + RK3 path.

Workload (one "step"): CompressibleIdealGas2D on a periodic 128x128 quad mesh
of [0,1]^2 with interior nodes perturbed by 0.02*h*sin(2 pi x)sin(2 pi y),
N = 7 Legendre-Gauss (4 conservative variables, 4,194,304 DOF), gamma = 1.4,
rho = 1 + 0.1 sin(2 pi x) sin(2 pi y), (u, v) = (0.5, 0.3), p = 1, naive LLF
flux, Williamson RK3 at CFL 0.5 (dt from CovariantArcMin), 200 RK3 steps:
one full solve.  Inputs are seeded synthetic fields of this shape (the
reference ships no data for it).

Reported (one JSON line on rank 0):
  value     DOF-updates/s with the state resident in HBM, device-timed with
            CUDA events on the engine's stream, L2 flushed before every solve
  e2e       the same metric through the public API with host buffers: each
            step copies the initial state host->device from pinned memory,
            runs the solve, and copies the final state back
  roofline  algorithmic bytes per fused-stage launch / measured launch time
  cpu_baseline  the CPU oracle (C++ restatement of the reference CPU path,
            OpenMP over elements) on a bounded sample of the same workload

``--impl reference`` times the reference algorithm's CPU implementation (the
oracle port; the Fortran reference cannot be built in this image) on the same
workload, metric and unit.  Multi-GPU: the path runs as independent replicas
(one per rank, no data-path collective); value = all ranks' DOF-updates over
the slowest rank's time.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, N, STEPS_PER_SOLVE, CFL = 128, 7, 200, 0.5
NVAR, P = 4, N + 1
NEL = NX * NX
DOF = NVAR * P * P * NEL
GAMMA = 1.4
WORKLOAD = (f"CompressibleIdealGas2D periodic {NX}x{NX} perturbed(0.02h) N={N} Gauss, FP64, naive LLF, "
            f"Williamson RK3 CFL {CFL}, {STEPS_PER_SOLVE} steps per solve")


def algorithmic_bytes_per_element_stage():
    """Bytes one element must move per RK stage (8-byte words):
    state read+write and RK register read+write (4*nVar*P^2), own 9-field
    traces written + neighbour traces read (2*4*9*P), metric terms dsdx(4)+J(1)
    per node and nHat(2)+nScale(1) per face node, 80 B of sideInfo."""
    w = 8
    return w * (4 * NVAR * P * P + 2 * 4 * 9 * P) + w * (5 * P * P + 12 * P) + 80


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def recorded_traffic():
    """DRAM bytes per fused-stage launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "fused_stage_cig_c2.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def initial_state(x):
    X, Y = x[..., 0], x[..., 1]  # x: (nEl, 1, P, P, 2) device tensor
    rho = 1.0 + 0.1 * (2 * np.pi * X).sin() * (2 * np.pi * Y).sin()
    import torch
    q = torch.empty((NEL, 4, P, P), device=x.device, dtype=torch.float64)
    q[:, 0] = (rho * 0.5)[:, 0]
    q[:, 1] = (rho * 0.3)[:, 0]
    q[:, 2] = rho[:, 0]
    q[:, 3] = (1.0 / (GAMMA - 1.0) + 0.5 * rho * (0.5 ** 2 + 0.3 ** 2))[:, 0]
    return q


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc = index, None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(seconds=12.0, max_steps=STEPS_PER_SOLVE):
    """The CPU oracle on the full mesh, stepping until `seconds` of work."""
    from oracle import build as obuild
    obuild.build()
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores, fast=True)
    m = O.Mesh(NX, NX, periodic=(True, True), amp=0.02)
    mod = O.Model(O.CIG, N, m, fast=True)
    g = O.Geometry(N, m)
    X, Y = g.x[0, :, :, 0, :], g.x[1, :, :, 0, :]
    q = np.zeros((P, P, 4, NEL), order="F")
    rho = 1 + 0.1 * np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y)
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = rho * 0.5, rho * 0.3, rho
    q[:, :, 3] = 1 / (GAMMA - 1) + 0.5 * rho * 0.34
    mod.set("solution", q)
    dt = 1e-4
    mod.rk3(1, dt)  # warm-up
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps and time.perf_counter() - t0 < seconds:
        mod.rk3(1, dt)
        steps += 1
    el = time.perf_counter() - t0
    return {"value": DOF * steps / el, "unit": "DOF-updates/s", "cores": cores, "kind": "port",
            "sample": f"{steps} RK3 steps of the full {NX}x{NX} N={N} mesh ({steps}/{STEPS_PER_SOLVE} of a solve), "
                      f"{el:.1f} s, C++ restatement of the reference CPU branches, OpenMP over elements"}


def run_forms(steps=20, err_steps=500, n_instances=256):
    """The ensemble workload: 256 seeded nonlinear ShallowWater instances
    (nx, ny ~ U{8..64}, N ~ U{3,5,7}, 4-Gaussian topography, reflecting walls,
    per-instance CFL-0.5 time step), advanced (a) one FP64 handle per instance,
    (b) batched per degree in FP64, (c) batched per degree in the FP32-bulk form;
    DOF-updates/s over `steps` RK3 steps each, and the FP32-bulk error against
    the batched FP64 run after `err_steps` steps (the workload's length)."""
    import torch

    import self_b200 as S
    from self_b200 import ensemble as E
    inst = E.make_instances(n_instances, seed=0)
    e64 = E.ShallowWaterEnsemble(inst, form=S.FP64, autotune=True)
    e32 = E.ShallowWaterEnsemble(inst, form=S.FP32_BULK, autotune=True)
    un = E.UnbatchedShallowWater(inst)
    dof = sum(i.dof() for i in inst)
    out = {"workload": f"{n_instances} ShallowWater instances, nx,ny~U{{8..64}}, N~U{{3,5,7}}, FP32/FP64, "
                       f"per-instance CFL 0.5; rates over {steps} RK3 steps", "dof": dof}
    for name, runner in (("unbatched_fp64", un), ("batched_fp64", e64), ("batched_fp32_bulk", e32)):
        runner.reset()
        runner.ForwardStep(2)
        torch.cuda.synchronize()
        l0 = runner.launches() if hasattr(runner, "launches") else None
        t = E.time_it(lambda: runner.ForwardStep(steps))
        out[name] = {"value": dof * steps / t, "unit": "DOF-updates/s", "ms_per_rk3_step": 1e3 * t / steps}
    out["speedup_fp32_batched_vs_unbatched_fp64"] = out["batched_fp32_bulk"]["value"] / out["unbatched_fp64"]["value"]
    out["autotune"] = {f"N={k}": v for k, v in e32.tuning.items()}
    e64.reset()
    e32.reset()
    e64.ForwardStep(err_steps)
    e32.ForwardStep(err_steps)
    torch.cuda.synchronize()
    worst = 0.0
    for it in inst:
        a, b = e32.solution(it), e64.solution(it)
        worst = max(worst, float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)))
    out["fp32_bulk_rel_l2_err_vs_fp64_after_%d_steps" % err_steps] = worst
    return out


def _events_ms(fn):
    """Device time of fn() from CUDA events on the default (legacy) stream; the
    engine handles below use blocking streams, which are ordered with it."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _rel_l2(a, b):
    import torch
    d = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    return d if np.isfinite(d) else None


def shock_band(x, rng):
    """Smooth density wave (the C2 state) plus one seeded shock-tube band: in
    |y - y0| < 0.05 a Sod-like tube (rho, p) = (1, 1) | (0.125, 0.1) at rest,
    split at x = x0."""
    import torch
    X, Y = x[:, 0, :, :, 0], x[:, 0, :, :, 1]
    x0, y0 = rng.uniform(0.3, 0.7, size=2)
    rho = 1.0 + 0.1 * torch.sin(2 * np.pi * X) * torch.sin(2 * np.pi * Y)
    u = torch.full_like(X, 0.5)
    v = torch.full_like(X, 0.3)
    p = torch.ones_like(X)
    band = (Y - y0).abs() < 0.05
    left = X < x0
    rho = torch.where(band, torch.where(left, torch.ones_like(X), torch.full_like(X, 0.125)), rho)
    p = torch.where(band, torch.where(left, torch.ones_like(X), torch.full_like(X, 0.1)), p)
    u = torch.where(band, torch.zeros_like(X), u)
    v = torch.where(band, torch.zeros_like(X), v)
    q = torch.empty((X.shape[0], 4) + tuple(X.shape[1:]), device=X.device, dtype=torch.float64)
    q[:, 0], q[:, 1], q[:, 2] = rho * u, rho * v, rho
    q[:, 3] = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v)
    return q


def _closure_variant(mesh, geo, q0, form, mode, mlp, steps, dt, dof):
    """One timed run from q0: DOF-updates/s, the final state and closure statistics."""
    import self_b200 as S
    model = S.CompressibleIdealGas2D(mesh, geo, form=form)
    model.SetSolution(q0)
    if mode:
        model.SetClosure(mode, c=1.0, mlp=mlp)
    model.ForwardStep(2, dt)  # captures the RK-step graph
    model.Sync()
    p_, g_, us_ = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
    S.check(S.lib().selfgpu_model2d_autotune(model._h, ctypes.byref(p_), ctypes.byref(g_), ctypes.byref(us_)))
    model.ForwardStep(1, dt)  # recapture with the tuned launch
    model.Sync()
    model.SetSolution(q0)
    model.workSol.zero_()
    l0 = model.LaunchCount()
    if mode:
        model.ClosureState(reset=True)
    ms = _events_ms(lambda: model.ForwardStep(steps, dt))
    res = {"value": dof * steps / (ms / 1e3), "unit": "DOF-updates/s", "ms_per_rk3_step": ms / steps,
           "launches_per_rk3_step": (model.LaunchCount() - l0) / steps,
           "kernel": ("persistent, %d groups" % g_.value) if p_.value else "per-element"}
    if mode:
        nu, act, ind, (fb, evals) = model.ClosureState(reset=True)
        res["active_elements_last_stage"] = int((act > 0).sum())
        if mode == S.CLOSURE_MLP:
            res["mlp_evaluation_fraction"] = evals / (3.0 * steps * model.nElem)
            res["fallback_fraction_of_evaluations"] = fb / max(evals, 1)
            res["mean_abs_activation_diff_vs_indicator_last_stage"] = float((act - ind).abs().mean())
    sol = model.solution.clone()
    del model
    return res, sol


def run_closure_forms(n_problems=16, snapshots=4, c4_steps=50, c5_steps=100):
    """The learned shock closure (form 4) and the large single solve with all
    forms: training data from FP64 N=7 runs, training, the C4 workload
    (CIG 256x256 N=5 FP32, seeded four-quadrant Riemann problem) and the C5
    workload (CIG 512x512 N=7, smooth density wave + shock-tube band), plus
    the C2 solve in the FP32-bulk form."""
    import torch

    import self_b200 as S
    from self_b200 import closure as CL
    out = {}
    t0 = time.perf_counter()
    data = CL.harvest(N_run=7, nx=128, n_problems=n_problems, snapshots=snapshots, steps_between=20, seed=0,
                      N_sample=(5, 7))
    torch.cuda.synchronize()
    out["harvest"] = {"runs": f"{n_problems} seeded four-quadrant Riemann problems, CIG periodic 128x128 N=7 FP64 "
                              f"with the indicator closure, {snapshots} snapshots 20 RK3 steps apart; states "
                              f"interpolated to N=5 for the N=5 closure",
                      "seconds": time.perf_counter() - t0}
    mlps = {}
    for d, (f, l) in sorted(data.items()):
        m = CL.ClosureMLP(seed=d)
        t1 = time.perf_counter()
        loss = m.train(f, l, epochs=8, batch=8192, lr=2e-3, seed=d)
        tt = time.perf_counter() - t1
        pred = m.infer(f)
        mlps[d] = m
        out[f"training_N{d}"] = {"samples": int(f.shape[0]), "active_fraction": float((l > 0).float().mean()),
                                 "epochs": 8, "batch": 8192, "mse_first_last": [float(loss[0]), float(loss[-1])],
                                 "mean_abs_err_vs_indicator": float((pred - l).abs().mean()), "seconds": tt}
    del data

    # C4: 256 x 256, N = 5, FP32 bulk, seeded Riemann problem, learned closure
    N4 = 5
    interp = S.Lagrange(N4, S.GAUSS, N4, S.UNIFORM)
    mesh = S.Mesh2D(256, 256, periodic=(True, True))
    geo = S.SEMQuad(interp, mesh)
    rng = np.random.Generator(np.random.PCG64(100))
    q0 = CL.riemann_quadrants(geo.x, rng)
    dof4 = 4 * (N4 + 1) ** 2 * mesh.nElem
    probe = S.CompressibleIdealGas2D(mesh, geo)
    dt4 = CL.stable_dt(probe, q0)
    del probe
    c4 = {"workload": f"CIG periodic 256x256 N=5, seeded four-quadrant Riemann problem, {c4_steps} RK3 steps, "
                      f"dt={dt4:.3e}", "dof": dof4}
    ref4 = None
    for name, form, mode, mlp in (("fp64_indicator", S.FP64, S.CLOSURE_INDICATOR, None),
                                  ("fp32_learned", S.FP32_BULK, S.CLOSURE_MLP, mlps[5]),
                                  ("fp32_indicator", S.FP32_BULK, S.CLOSURE_INDICATOR, None),
                                  ("fp64_no_closure", S.FP64, S.CLOSURE_OFF, None)):
        res, sol = _closure_variant(mesh, geo, q0, form, mode, mlp, c4_steps, dt4, dof4)
        if ref4 is None:
            ref4 = sol
        else:
            res["rel_l2_vs_fp64_indicator"] = _rel_l2(sol, ref4)
        c4[name] = res
    c4["speedup_fp32_learned_vs_fp64_no_closure"] = c4["fp32_learned"]["value"] / c4["fp64_no_closure"]["value"]
    out["c4_learned_closure"] = c4
    del ref4, q0, geo, mesh

    # C5: 512 x 512, N = 7, all forms
    N5 = 7
    interp = S.Lagrange(N5, S.GAUSS, N5, S.UNIFORM)
    mesh = S.Mesh2D(512, 512, periodic=(True, True), perturbation=0.02)
    geo = S.SEMQuad(interp, mesh)
    rng = np.random.Generator(np.random.PCG64(200))
    q0 = shock_band(geo.x, rng)
    dof5 = 4 * (N5 + 1) ** 2 * mesh.nElem
    probe = S.CompressibleIdealGas2D(mesh, geo)
    dt5 = CL.stable_dt(probe, q0)
    del probe
    c5 = {"workload": f"CIG periodic 512x512 perturbed N=7, smooth density wave + shock-tube band, {c5_steps} RK3 "
                      f"steps, dt={dt5:.3e}", "dof": dof5}
    ref5 = None
    for name, form, mode, mlp in (("fp64_indicator", S.FP64, S.CLOSURE_INDICATOR, None),
                                  ("fp32_learned", S.FP32_BULK, S.CLOSURE_MLP, mlps[7]),
                                  ("fp32_indicator", S.FP32_BULK, S.CLOSURE_INDICATOR, None),
                                  ("fp64_no_closure", S.FP64, S.CLOSURE_OFF, None)):
        res, sol = _closure_variant(mesh, geo, q0, form, mode, mlp, c5_steps, dt5, dof5)
        if ref5 is None:
            ref5 = sol
        else:
            res["rel_l2_vs_fp64_indicator"] = _rel_l2(sol, ref5)
        c5[name] = res
    c5["speedup_fp32_learned_vs_fp64_no_closure"] = c5["fp32_learned"]["value"] / c5["fp64_no_closure"]["value"]
    out["c5_large_solve"] = c5
    del ref5, q0, geo, mesh

    # C2 in the FP32-bulk form (smooth: the closure stays off), error vs the FP64 engine
    interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
    mesh = S.Mesh2D(NX, NX, periodic=(True, True), perturbation=0.02)
    geo = S.SEMQuad(interp, mesh)
    q0 = initial_state(geo.x)
    c = (GAMMA * 1.0 / (q0[:, 2].min())).sqrt().item()
    dt = CFL * geo.CovariantArcMin() / (np.hypot(0.5, 0.3) + c)
    c2 = {}
    ref2 = None
    for name, form in (("fp64", S.FP64), ("fp32_bulk", S.FP32_BULK)):
        res, sol = _closure_variant(mesh, geo, q0, form, S.CLOSURE_OFF, None, STEPS_PER_SOLVE, dt, DOF)
        if ref2 is None:
            ref2 = sol
        else:
            res["rel_l2_vs_fp64"] = _rel_l2(sol, ref2)
        c2[name] = res
    c2["speedup_fp32_bulk_vs_fp64"] = c2["fp32_bulk"]["value"] / c2["fp64"]["value"]
    out["c2_forms"] = c2
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import build as obuild
    obuild.build()
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores, fast=True)
    m = O.Mesh(NX, NX, periodic=(True, True), amp=0.02)
    mod = O.Model(O.CIG, N, m, fast=True)
    g = O.Geometry(N, m)
    X, Y = g.x[0, :, :, 0, :], g.x[1, :, :, 0, :]
    q = np.zeros((P, P, 4, NEL), order="F")
    rho = 1 + 0.1 * np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y)
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = rho * 0.5, rho * 0.3, rho
    q[:, :, 3] = 1 / (GAMMA - 1) + 0.5 * rho * 0.34
    mod.set("solution", q)
    dt = 1e-4
    for _ in range(args.warmup):
        mod.rk3(1, dt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        mod.rk3(1, dt)
    el = time.perf_counter() - t0
    v = DOF * args.steps / el
    sample = (f"each step = 1 RK3 step of the full {NX}x{NX} N={N} mesh (1/{STEPS_PER_SOLVE} of a solve); "
              f"C++ restatement of the reference CPU path (the Fortran reference needs gfortran, hipfort, MPI and "
              f"HDF5, none of which exist in this image)")
    print(json.dumps({
        "impl": "reference", "metric": "DOF-updates/s", "value": v, "unit": "DOF-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "elements": NEL, "dof": DOF, "parallelism": "replicas"},
        "cpu_baseline": {"value": v, "unit": "DOF-updates/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_engine(args, rank, world, local_rank):
    import torch
    import self_b200 as S
    from self_b200 import replicas as R
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream(device=dev)
    interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
    mesh = S.Mesh2D(NX, NX, periodic=(True, True), perturbation=0.02)
    geo = S.SEMQuad(interp, mesh)
    model = S.CompressibleIdealGas2D(mesh, geo, stream=stream.cuda_stream)
    S.lib().selfgpu_model2d_set_kernel(model._h, 1 if args.kernel == "persistent" else 0)
    q0 = initial_state(geo.x)
    torch.cuda.synchronize()
    # CFL time step: dt = CFL * ArcMin / max(|u| + c)
    c = (GAMMA * 1.0 / (q0[:, 2].min())).sqrt().item()
    dt = CFL * geo.CovariantArcMin() / (np.hypot(0.5, 0.3) + c)
    flush = torch.empty(64 * 1024 * 1024, device=dev, dtype=torch.float32)  # 256 MB > 126 MB L2

    def solve():
        model.SetSolution(q0)
        model.workSol.zero_()
        model.ForwardStep(STEPS_PER_SOLVE, dt)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            solve()
    stream.synchronize()
    launches0 = model.LaunchCount()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    try:
        smi_id = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        smi_id = str(local_rank)
    clocks = Clocks(smi_id)
    R.barrier()
    torch.cuda.synchronize()
    with clocks, torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            solve()
            ends[k].record(stream)
        torch.cuda.synchronize()
    R.barrier()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    launches = model.LaunchCount() - launches0  # fused-stage launches (plus one trace prologue per solve)
    persistent = S.lib().selfgpu_model2d_persistent_launch_count(model._h)
    clk = clocks.summary()
    t_max = R.max_over_ranks(ms)
    value = R.aggregate_rate(DOF * STEPS_PER_SOLVE * args.steps, world, t_max / 1e3)
    stage_ms = ms / (args.steps * 3 * STEPS_PER_SOLVE)
    per_launch = algorithmic_bytes_per_element_stage() * NEL
    achieved = per_launch / (stage_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic = recorded_traffic()

    # ---- end to end through the public API with host buffers
    host_q = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True)
    host_q.copy_(q0.cpu())
    host_out = torch.empty_like(host_q).pin_memory()
    with torch.cuda.stream(stream):
        for _ in range(max(1, args.warmup // 2)):
            model.solution.copy_(host_q, non_blocking=True)
            model.workSol.zero_()
            S.lib().selfgpu_model2d_invalidate(model._h)
            model.ForwardStep(STEPS_PER_SOLVE, dt)
            host_out.copy_(model.solution, non_blocking=True)
        stream.synchronize()
        R.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            model.solution.copy_(host_q, non_blocking=True)
            model.workSol.zero_()
            S.lib().selfgpu_model2d_invalidate(model._h)
            model.ForwardStep(STEPS_PER_SOLVE, dt)
            host_out.copy_(model.solution, non_blocking=True)
        e1.record(stream)
        stream.synchronize()
    e2e_ms = R.max_over_ranks(e0.elapsed_time(e1))
    e2e = R.aggregate_rate(DOF * STEPS_PER_SOLVE * args.steps, world, e2e_ms / 1e3)
    model.CheckFinite()

    if rank != 0:
        return
    line = {
        "metric": "DOF-updates/s", "value": value, "unit": "DOF-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "elements": NEL, "dof": DOF, "rk3_steps_per_step": STEPS_PER_SOLVE,
                   "dt": dt, "parallelism": "replicas" if world > 1 else "single-gpu",
                   "l2": "flushed (256 MB write) before every timed solve; per-stage working set ~150 MB > L2"},
        "e2e": {"value": e2e, "unit": "DOF-updates/s", "h2d_bytes_per_step": int(host_q.numel() * 8),
                "d2h_bytes_per_step": int(host_out.numel() * 8)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "bytes_per_launch": per_launch, "launch_ms": stage_ms,
                     "kernel": ("k_fused_stage_tma<8,PhysCIG,double>" if persistent else
                                "k_fused_stage<8,PhysCIG,double>") + " (one RK stage over all elements)"},
        "clocks": clk,
    }
    if not args.no_forms:
        line["forms"] = run_forms()
        line["forms"].update(run_closure_forms())
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="selfgpu", choices=["selfgpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the ensemble / FP32-bulk form measurements")
    ap.add_argument("--kernel", default="persistent", choices=["persistent", "per-element"],
                    help="stage kernel: persistent bulk-copy kernel or one CTA per element group")
    args = ap.parse_args()
    from self_b200 import replicas as R
    rank, world, local_rank = R.init("gloo" if args.impl == "reference" else "nccl")
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_engine(args, rank, world, local_rank)
    finally:
        R.finalize()


if __name__ == "__main__":
    main()
