"""Benchmark: DOF-updates/s of the fused FP64 DGSEM tendency + RK3 path.

Workload (one "step"): CompressibleIdealGas2D on a periodic 128x128 quad mesh
of [0,1]^2 with interior nodes perturbed by 0.02*h*sin(2 pi x)sin(2 pi y),
N = 7 Legendre-Gauss (4 conservative variables, 4,194,304 DOF), gamma = 1.4,
rho = 1 + 0.1 sin(2 pi x) sin(2 pi y), (u, v) = (0.5, 0.3), p = 1, naive LLF
flux, Williamson RK3 at CFL 0.5 (dt from CovariantArcMin), 200 RK3 steps:
one full solve.  Inputs are seeded synthetic fields of this shape (the
reference ships no data for it).

Reported (one JSON line on rank 0), for the production FP64 form:
  value     DOF-updates/s with the state resident in HBM, device-timed with
            CUDA events on the engine's stream, L2 flushed before every solve
  e2e       the same metric through the C ABI a Fortran caller uses, with
            host buffers: each step copies the initial state from pinned host
            memory into hipMalloc'd device buffers (the library's HIP memory
            shim, as SELF's UpdateDevice does), runs the solve with
            selfgpu_model2d_rk3 on the engine's default stream, and copies
            the final state back with hipMemcpy (UpdateHost)
  roofline  algorithmic bytes per fused-stage launch / measured launch time
  cpu_baseline  the CPU oracle (C++ restatement of the reference CPU path,
            OpenMP over elements) on a bounded sample of the same workload

``--impl reference`` times the reference algorithm's CPU implementation (the
oracle port; the Fortran reference cannot be built in this image) on the same
workload, metric, unit, config and step definition (one 200-step solve).  Multi-GPU: the path runs as independent replicas
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


def cfl_dt(arcmin, rho_min):
    """dt = CFL * ArcMin / max(|u| + c) of the initial state, c = sqrt(gamma p / rho), p = 1."""
    return CFL * arcmin / (np.hypot(0.5, 0.3) + float(np.sqrt(GAMMA / rho_min)))


def config_dict(dt, world):
    """The config both arms print (same workload, same step definition)."""
    return {"workload": WORKLOAD, "elements": NEL, "dof": DOF, "rk3_steps_per_step": STEPS_PER_SOLVE,
            "dt": round(dt, 12), "parallelism": "replicas" if world > 1 else "single-gpu",
            "l2": "flushed (256 MB write) before every timed solve; per-stage working set ~150 MB > L2"}


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


def recorded_traffic(multistage):
    """DRAM bytes per RK stage of the C2 stage kernel from the committed ncu
    summary: of the multi-stage launch (all stages of a solve in one launch)
    or of the one-stage launch."""
    path = os.path.join(ROOT, "profiles", "fused_stage_cig_c2.txt")
    key = "traffic_bytes_per_stage_multistage:" if multistage else "traffic_bytes_per_launch:"
    try:
        for line in open(path):
            if line.startswith(key):
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
    """SM clocks and throttle reasons sampled during the timed region.

    An in-process NVML reader thread (every 10 ms, so that even a timed region
    of a few hundred milliseconds has samples); `nvidia-smi -lms 200` when NVML
    cannot be loaded.  Only reads the GPU's state."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index, self.proc, self.thread = index, None, None
        self.sm, self.mx, self.reasons = [], None, set()
        self.f = None

    def _nvml_loop(self, nv, h, bits):
        while not self.stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for nm, b in zip(self.NAMES, bits):
                    if r & b:
                        self.reasons.add(nm)
            except Exception:
                pass
            self.stop.wait(0.01)

    def __enter__(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            idx = str(self.index)
            h = nv.nvmlDeviceGetHandleByUUID(idx) if idx.startswith("GPU-") else nv.nvmlDeviceGetHandleByIndex(int(idx))
            self.mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h, bits), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread:
            self.stop.set()
            self.thread.join()
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if self.f is not None:
            self.f.flush()
            self.f.seek(0)
            for line in self.f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    self.sm.append(float(parts[1]))
                    self.mx = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(self.NAMES, parts[5:9]):
                    if v.lower() == "active":
                        self.reasons.add(nm)
            os.unlink(self.f.name)
            self.f = None
        sm = self.sm
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.mx,
                "reasons": sorted(self.reasons), "samples": len(sm),
                "source": "nvml" if self.thread is not None else "nvidia-smi"}


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


def _cpu_rate(make_model, dof, dt, steps, threads, reps=3):
    """Median over reps of DOF-updates/s of `steps` RK3 steps of the oracle."""
    from oracle import oracle as O
    O.set_threads(threads, fast=True)
    mod = make_model()
    mod.rk3(1, dt)  # warm-up
    rates = []
    for _ in range(reps):
        t0 = time.perf_counter()
        mod.rk3(steps, dt)
        rates.append(dof * steps / (time.perf_counter() - t0))
    return statistics.median(rates)


def run_cpu_table():
    """CPU baseline table for configs C1-C5 (the oracle port, FP64 plain, no
    closure): single thread and all host cores, median of 3 bounded samples."""
    from oracle import build as obuild
    obuild.build()
    from oracle import oracle as O
    cores = os.cpu_count() or 1

    def cig(nx, Nd, amp, ic):
        def make():
            m = O.Mesh(nx, nx, periodic=(True, True), amp=amp)
            mod = O.Model(O.CIG, Nd, m, fast=True)
            x = O.Geometry(Nd, m).x
            mod.set("solution", ic(x))
            return mod
        return make

    def smooth(x):
        X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
        q = np.zeros(X.shape[:2] + (4, X.shape[2]), order="F")
        rho = 1 + 0.1 * np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y)
        q[:, :, 0], q[:, :, 1], q[:, :, 2] = rho * 0.5, rho * 0.3, rho
        q[:, :, 3] = 1 / (GAMMA - 1) + 0.5 * rho * 0.34
        return q

    def lsw():
        m = O.Mesh(10, 10, bcid=O.BC_NONORMALFLOW)
        mod = O.Model(O.LSW, 7, m, fast=True)
        x = O.Geometry(7, m).x
        X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
        P7 = 8
        mod.set("H", np.ones((P7, P7, 1, 100), order="F"))
        mod.set("fCori", np.zeros((P7, P7, 1, 100), order="F"))
        q = np.zeros((P7, P7, 3, 100), order="F")
        q[:, :, 2] = 0.01 * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)
        mod.set("solution", q)
        return mod

    rows = {}
    specs = [
        ("C1", "LSW 10x10 N=7 walls (gravity-wave release), dt=1e-4", lsw, 3 * 64 * 100, 1e-4, (200, 1000), None),
        ("C2", "CIG periodic 128x128 perturbed N=7, density wave", cig(128, 7, 0.02, smooth), 4 * 64 * 16384, 1e-5,
         (1, 5), None),
        ("C4", "CIG periodic 256x256 N=5 (sampled on 128x128: the rate per DOF-update does not depend on the mesh "
               "size)", cig(128, 5, 0.0, smooth), 4 * 36 * 16384, 1e-5, (1, 8), None),
        ("C5", "CIG periodic 512x512 perturbed N=7 (sampled on 128x128, as C2)", cig(128, 7, 0.02, smooth),
         4 * 64 * 16384, 1e-5, (1, 5), None),
    ]
    for name, desc, make, dof, dt, (s1, sN), _ in specs:
        rows[name] = {"workload": desc, "one_thread": _cpu_rate(make, dof, dt, s1, 1),
                      "all_cores": _cpu_rate(make, dof, dt, sN, cores), "cores": cores}
    # C3: the ensemble instances, advanced one by one (a sample of the 256)
    from self_b200 import ensemble as E
    inst = E.make_instances(256, seed=0)[:12]

    def ens_rate(threads):
        O.set_threads(threads, fast=True)
        tot_dof, tot_t = 0, 0.0
        for it in inst:
            om = O.Mesh(it.nx, it.ny, bcid=O.BC_NONORMALFLOW)
            mod = O.Model(O.SW, it.N, om, fast=True)
            x = O.Geometry(it.N, om).x
            X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
            Pn = it.N + 1
            mod.set("topography", E.topography(it, X, Y).reshape(Pn, Pn, 1, -1, order="F"))
            q = np.zeros((Pn, Pn, 3, it.nElem), order="F")
            q[:, :, 2] = E.thickness(it, X, Y)
            mod.set("solution", q)
            mod.rk3(1, 1e-4)
            t0 = time.perf_counter()
            mod.rk3(3, 1e-4)
            tot_t += time.perf_counter() - t0
            tot_dof += it.dof() * 3
        return tot_dof / tot_t

    rows["C3"] = {"workload": "256 SW instances (sample: the first 12, advanced one by one)",
                  "one_thread": statistics.median([ens_rate(1) for _ in range(3)]),
                  "all_cores": statistics.median([ens_rate(cores) for _ in range(3)]), "cores": cores}
    return rows


def run_forms(steps=500, err_steps=500, n_instances=256):
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
    # the same FP64 kernels, each degree's handle replaying its own graph on its stream
    e64s = E.ShallowWaterEnsemble(inst, form=S.FP64, autotune=False, one_graph=False)
    for N, tun in e64.tuning.items():
        S.lib().selfgpu_model2d_set_launch(e64s.handles[N]["model"]._h, tun["persistent"], tun["groups"])
    un = E.UnbatchedShallowWater(inst)
    dof = sum(i.dof() for i in inst)
    out = {"workload": f"{n_instances} ShallowWater instances, nx,ny~U{{8..64}}, N~U{{3,5,7}}, FP32/FP64, "
                       f"per-instance CFL 0.5; rates over {steps} RK3 steps", "dof": dof,
           "batched_launch": "one CUDA graph launch per RK3 step for all degrees (one branch per degree)"}
    for name, runner in (("unbatched_fp64", un), ("batched_fp64", e64), ("batched_fp32_bulk", e32),
                         ("batched_fp64_per_degree_streams", e64s)):
        runner.reset()
        runner.ForwardStep(2)
        torch.cuda.synchronize()
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


def _closure_variant(mesh, geo, q0, form, mode, mlp, steps, dt, dof, nvtx=None):
    """One timed run from q0: DOF-updates/s, the final state and closure statistics
    (the timed steps inside an NVTX range named nvtx, for profilers)."""
    import torch

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
    if nvtx:
        torch.cuda.nvtx.range_push(nvtx)
    ms = _events_ms(lambda: model.ForwardStep(steps, dt))
    if nvtx:
        torch.cuda.nvtx.range_pop()
    res = {"value": dof * steps / (ms / 1e3), "unit": "DOF-updates/s", "ms_per_rk3_step": ms / steps,
           "launches_per_rk3_step": (model.LaunchCount() - l0) / steps,
           "kernel": ("persistent, %d groups" % g_.value) if p_.value else "per-element"}
    if mode:
        nu, act, ind, (fb, evals) = model.ClosureState(reset=True)
        res["active_elements_last_step"] = int((act > 0).sum())
        if mode == S.CLOSURE_MLP:  # the viscosity is formed once per RK step
            res["mlp_evaluation_fraction"] = evals / (float(steps) * model.nElem)
            res["fallback_fraction_of_evaluations"] = fb / max(evals, 1)
            res["mean_abs_activation_diff_vs_indicator_last_stage"] = float((act - ind).abs().mean())
    sol = model.solution.clone()
    del model
    return res, sol


def train_closures(n_problems=16, snapshots=4):
    """Training data from FP64 N=7 indicator-closure runs and the two closure
    MLPs (N=5 from states interpolated to N=5, N=7)."""
    import torch

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
    return out, mlps


def _closure_workload(tag, mesh, geo, q0, dt, dof, steps, mlp, desc):
    import self_b200 as S
    res = {"workload": desc, "dof": dof}
    ref = None
    for name, form, mode, m in (("fp64_indicator", S.FP64, S.CLOSURE_INDICATOR, None),
                                ("fp32_learned", S.FP32_BULK, S.CLOSURE_MLP, mlp),
                                ("fp32_indicator", S.FP32_BULK, S.CLOSURE_INDICATOR, None),
                                ("fp64_no_closure", S.FP64, S.CLOSURE_OFF, None)):
        r, sol = _closure_variant(mesh, geo, q0, form, mode, m, steps, dt, dof, nvtx=f"{tag}_{name}")
        if ref is None:
            ref = sol
        else:
            r["rel_l2_vs_fp64_indicator"] = _rel_l2(sol, ref)
        res[name] = r
    res["speedup_fp32_learned_vs_fp64_no_closure"] = res["fp32_learned"]["value"] / res["fp64_no_closure"]["value"]
    return res


def measure_c4(mlp5, steps=50):
    """C4: CIG periodic 256x256 N=5, seeded four-quadrant Riemann problem."""
    import self_b200 as S
    from self_b200 import closure as CL
    interp = S.Lagrange(5, S.GAUSS, 5, S.UNIFORM)
    mesh = S.Mesh2D(256, 256, periodic=(True, True))
    geo = S.SEMQuad(interp, mesh)
    q0 = CL.riemann_quadrants(geo.x, np.random.Generator(np.random.PCG64(100)))
    dt = CL.stable_dt(S.CompressibleIdealGas2D(mesh, geo), q0)
    return _closure_workload("c4", mesh, geo, q0, dt, 4 * 36 * mesh.nElem, steps, mlp5,
                             f"CIG periodic 256x256 N=5, seeded four-quadrant Riemann problem, {steps} RK3 steps, "
                             f"dt={dt:.3e}")


def measure_c5(mlp7, steps=100):
    """C5: CIG periodic 512x512 perturbed N=7, smooth density wave + shock-tube band."""
    import self_b200 as S
    from self_b200 import closure as CL
    interp = S.Lagrange(7, S.GAUSS, 7, S.UNIFORM)
    mesh = S.Mesh2D(512, 512, periodic=(True, True), perturbation=0.02)
    geo = S.SEMQuad(interp, mesh)
    q0 = CL.shock_band(geo.x, np.random.Generator(np.random.PCG64(200)), gamma=GAMMA)
    dt = CL.stable_dt(S.CompressibleIdealGas2D(mesh, geo), q0)
    return _closure_workload("c5", mesh, geo, q0, dt, 4 * 64 * mesh.nElem, steps, mlp7,
                             f"CIG periodic 512x512 perturbed N=7, smooth density wave + shock-tube band, {steps} RK3 "
                             f"steps, dt={dt:.3e}")


def measure_c2_forms():
    """C2 in the production FP64, reference-rounding FP64 and FP32-bulk forms
    (smooth: no closure); relative L2 differences against the production FP64 run."""
    import self_b200 as S
    interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
    mesh = S.Mesh2D(NX, NX, periodic=(True, True), perturbation=0.02)
    geo = S.SEMQuad(interp, mesh)
    q0 = initial_state(geo.x)
    dt = cfl_dt(geo.CovariantArcMin(), q0[:, 2].min().item())
    c2 = {}
    ref2 = None
    for name, form in (("fp64", S.FP64), ("fp64_ref", S.FP64_REF), ("fp32_bulk", S.FP32_BULK)):
        res, sol = _closure_variant(mesh, geo, q0, form, S.CLOSURE_OFF, None, STEPS_PER_SOLVE, dt, DOF,
                                    nvtx=f"c2_{name}")
        if ref2 is None:
            ref2 = sol
        else:
            res["rel_l2_vs_fp64"] = _rel_l2(sol, ref2)
        c2[name] = res
    c2["speedup_fp32_bulk_vs_fp64"] = c2["fp32_bulk"]["value"] / c2["fp64"]["value"]
    c2["speedup_fp64_vs_fp64_ref"] = c2["fp64"]["value"] / c2["fp64_ref"]["value"]
    return c2


def measure_c1():
    """C1: LinearShallowWater gravity-wave release, 10x10 walls, N=7, 1000 steps of dt = 1e-4."""
    import torch

    import self_b200 as S
    interp = S.Lagrange(7, S.GAUSS, 7, S.UNIFORM)
    mesh = S.Mesh2D(10, 10, bcid=S.BC_NONORMALFLOW)
    geo = S.SEMQuad(interp, mesh)
    lsw = S.LinearShallowWater(mesh, geo)
    X, Y = geo.x[:, 0, :, :, 0], geo.x[:, 0, :, :, 1]
    q1 = torch.zeros((mesh.nElem, 3, 8, 8), device="cuda", dtype=torch.float64)
    q1[:, 2] = 0.01 * torch.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)
    lsw.SetSolution(q1)
    lsw.ForwardStep(10, 1e-4)
    lsw.Sync()
    lsw.SetSolution(q1)
    lsw.workSol.zero_()
    ms = _events_ms(lambda: lsw.ForwardStep(1000, 1e-4))
    lsw.CheckFinite()
    out = {"workload": "LinearShallowWater 10x10 walls N=7, gravity-wave release, 1000 RK3 steps, dt=1e-4, FP64 "
                       "(19,200 DOF: launch-latency bound)",
           "graph_replayed": {"value": 19200 * 1000 / (ms / 1e3), "unit": "DOF-updates/s",
                              "ms_per_rk3_step": ms / 1000, "launches_per_solve": 3000}}
    # all 3000 RK stages in one cooperative launch (selfgpu_model2d_set_multistep)
    S.check(S.lib().selfgpu_model2d_set_multistep(lsw._h, 1))
    lsw.SetSolution(q1)
    lsw.workSol.zero_()
    lsw.ForwardStep(10, 1e-4)
    lsw.Sync()
    lsw.SetSolution(q1)
    lsw.workSol.zero_()
    l0 = lsw.LaunchCount()
    ms1 = _events_ms(lambda: lsw.ForwardStep(1000, 1e-4))
    lsw.CheckFinite()
    out["one_launch"] = {"value": 19200 * 1000 / (ms1 / 1e3), "unit": "DOF-updates/s",
                         "ms_per_rk3_step": ms1 / 1000, "launches_per_solve": lsw.LaunchCount() - l0}
    out["speedup_one_launch_vs_graph"] = ms / ms1
    return out


def measure_gas_ensemble(mlps, steps=100, n_instances=256):
    """The batched FP32-bulk + learned-closure form on an ensemble of uneven
    CompressibleIdealGas2D instances (nx, ny ~ U{8..64}, N ~ U{5, 7}, periodic,
    perturbed, smooth density waves, a seeded quarter with a shock-tube band),
    against the plain FP64 GPU form on the same instances (one handle per
    instance, and batched), with the FP64 indicator-closure run as the judge on
    shocked members.  Rates over `steps` RK3 steps; errors after them."""
    import torch

    import self_b200 as S
    from self_b200 import ensemble as E
    inst = E.make_gas_instances(n_instances, seed=0)
    variants = [("batched_fp32_learned", dict(form=S.FP32_BULK, closure=S.CLOSURE_MLP, mlps=mlps)),
                ("batched_fp32_indicator", dict(form=S.FP32_BULK, closure=S.CLOSURE_INDICATOR)),
                ("batched_fp64_indicator", dict(form=S.FP64, closure=S.CLOSURE_INDICATOR)),
                ("batched_fp64_plain", dict(form=S.FP64))]
    runners = {name: E.CompressibleGasEnsemble(inst, autotune=True, **kw) for name, kw in variants}
    runners["unbatched_fp64_plain"] = E.UnbatchedGas(inst)
    dof = sum(i.dof() for i in inst)
    n_smooth = sum(1 for i in inst if i.smooth)
    out = {"workload": f"{n_instances} CompressibleIdealGas2D instances, nx,ny~U{{8..64}}, N~U{{5,7}}, periodic "
                       f"perturbed 0.02h, smooth density waves ({n_smooth} smooth, {n_instances - n_smooth} with a "
                       f"shock-tube band), per-instance CFL/viscous step; rates over {steps} RK3 steps",
           "dof": dof}
    for name, r in runners.items():
        r.reset()
        r.ForwardStep(2)
        torch.cuda.synchronize()
        r.reset()
        torch.cuda.nvtx.range_push(f"gas_{name}")  # the timed steps, for profilers
        t = E.time_it(lambda: r.ForwardStep(steps))
        torch.cuda.nvtx.range_pop()
        out[name] = {"value": dof * steps / t, "unit": "DOF-updates/s", "ms_per_rk3_step": 1e3 * t / steps}
        if hasattr(r, "tuning"):
            out[name]["autotune"] = {f"N={k}": v for k, v in r.tuning.items()}
    lead = out["batched_fp32_learned"]["value"]
    out["speedup_fp32_learned_batched_vs_unbatched_fp64_plain"] = lead / out["unbatched_fp64_plain"]["value"]
    out["speedup_fp32_learned_batched_vs_batched_fp64_plain"] = lead / out["batched_fp64_plain"]["value"]
    # errors after `steps`: smooth members against the plain FP64 run, shocked
    # members against the FP64 indicator-closure run
    worst_smooth, worst_shock = 0.0, 0.0
    L, P64, I64 = runners["batched_fp32_learned"], runners["batched_fp64_plain"], runners["batched_fp64_indicator"]
    for it in inst:
        a = L.solution(it)
        b = (P64 if it.smooth else I64).solution(it)
        e = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        if it.smooth:
            worst_smooth = max(worst_smooth, e)
        else:
            worst_shock = max(worst_shock, e)
    out[f"fp32_learned_worst_rel_l2_vs_fp64_plain_smooth_members_after_{steps}_steps"] = worst_smooth
    out[f"fp32_learned_worst_rel_l2_vs_fp64_indicator_shocked_members_after_{steps}_steps"] = worst_shock
    out["all_finite"] = bool(all(torch.isfinite(L.solution(it)).all() for it in inst))
    del runners
    torch.cuda.empty_cache()
    return out


def run_closure_forms():
    """The learned shock closure (form 4), the large single solve with all
    forms, the batched learned-closure ensemble, C2 in the FP32-bulk form and C1."""
    out, mlps = train_closures()
    out["c4_learned_closure"] = measure_c4(mlps[5])
    out["c5_large_solve"] = measure_c5(mlps[7])
    out["gas_ensemble_fp32_learned"] = measure_gas_ensemble(mlps)
    out["c2_forms"] = measure_c2_forms()
    out["c1_lsw"] = measure_c1()
    return out


def measure_kernel(model, Nd, nx, form, steps, kernel="persistent"):
    """Diagnostic single-model run for profiling one stage kernel: a periodic
    nx x nx mesh (perturbed 0.02 h) at degree Nd, a smooth state, `steps` RK3
    steps after a warm-up; device time per RK stage and the algorithmic
    bandwidth (the same byte count as the roofline)."""
    import torch

    import self_b200 as S
    interp = S.Lagrange(Nd, S.GAUSS, Nd, S.UNIFORM)
    mesh = S.Mesh2D(nx, nx, periodic=(True, True), perturbation=0.02)
    geo = S.SEMQuad(interp, mesh)
    cls = {"LSW": S.LinearShallowWater, "SW": S.ShallowWater, "CIG": S.CompressibleIdealGas2D}[model]
    m = cls(mesh, geo, form={"fp64": S.FP64, "fp64_ref": S.FP64_REF, "fp32": S.FP32_BULK}[form])
    S.lib().selfgpu_model2d_set_kernel(m._h, 0 if kernel == "per-element" else 1)
    S.lib().selfgpu_model2d_set_multistage(m._h, 1 if kernel == "multistage" else 0)
    X, Y = geo.x[:, 0, :, :, 0], geo.x[:, 0, :, :, 1]
    Pd = Nd + 1
    nv = 4 if model == "CIG" else 3
    q = torch.zeros((mesh.nElem, nv, Pd, Pd), device="cuda", dtype=torch.float64)
    bump = 0.01 * torch.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.05)
    if model == "CIG":
        rho = 1.0 + 0.1 * torch.sin(2 * np.pi * X) * torch.sin(2 * np.pi * Y)
        q[:, 0], q[:, 1], q[:, 2], q[:, 3] = rho * 0.5, rho * 0.3, rho, 2.5 + 0.17 * rho
    elif model == "SW":
        q[:, 2] = 1.0 + bump
    else:
        q[:, 2] = bump
    m.SetSolution(q)
    m.ForwardStep(2, 1e-5)
    m.Sync()
    ms = _events_ms(lambda: m.ForwardStep(steps, 1e-5))
    m.CheckFinite()
    NT = 9 if model == "CIG" else 3
    A = {"CIG": 0, "SW": 8 * (2 * Pd * Pd + 4 * Pd), "LSW": 8 * (2 * Pd * Pd + 4 * Pd)}[model]
    w = 4 if form == "fp32" else 8
    b = w * (4 * nv * Pd * Pd + 8 * NT * Pd) + 8 * (5 * Pd * Pd + 12 * Pd) + A + 80
    if form == "fp32":  # FP64 solution, FP32 RK register and traces
        b = 8 * 2 * nv * Pd * Pd + 4 * 2 * nv * Pd * Pd + 4 * 8 * NT * Pd + 8 * (5 * Pd * Pd + 12 * Pd) + A + 80
    us = 1e3 * ms / (3 * steps)
    return {"workload": f"{model} periodic {nx}x{nx} N={Nd} {form}, {kernel} kernel, {steps} RK3 steps",
            "us_per_stage": us, "bytes_per_element_stage": b, "elements": mesh.nElem,
            "algorithmic_GBps": b * mesh.nElem / us / 1e3,
            "dof_updates_per_s": nv * Pd * Pd * mesh.nElem * steps / (ms / 1e3)}


def run_one_form(name, args=None):
    if name == "kernel":
        return measure_kernel(args.model, args.N, args.nx, args.fp, args.kernel_steps, args.kernel)
    if name == "ensemble":
        return run_forms()
    if name == "gas_ensemble":
        out, mlps = train_closures()
        out["gas_ensemble_fp32_learned"] = measure_gas_ensemble(mlps)
        return out
    if name == "c1":
        return measure_c1()
    if name == "c2":
        return measure_c2_forms()
    out, mlps = train_closures()
    out[name] = measure_c4(mlps[5]) if name == "c4" else measure_c5(mlps[7])
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
    dt = cfl_dt(g.arcmin, float(rho.min()))

    def solve():  # one step: the same full 200-step solve the GPU arm times
        mod.set("solution", q)
        mod.rk3(STEPS_PER_SOLVE, dt)

    for _ in range(args.warmup):
        solve()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        solve()
    el = time.perf_counter() - t0
    v = DOF * STEPS_PER_SOLVE * args.steps / el
    sample = (f"each step = one full {STEPS_PER_SOLVE}-step RK3 solve of the {NX}x{NX} N={N} mesh, as on the GPU "
              f"arm; C++ restatement of the reference CPU path, OpenMP over elements on {cores} host threads (the "
              f"Fortran reference needs gfortran, hipfort, MPI and HDF5, none of which exist in this image)")
    print(json.dumps({
        "impl": "reference", "metric": "DOF-updates/s", "value": v, "unit": "DOF-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(dt, world),
        "cpu_baseline": {"value": v, "unit": "DOF-updates/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "DOF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def e2e_through_c_abi(S, mesh, geo, q0, dt, args):
    """The solve as a Fortran caller runs it through the C ABI: device state
    from the library's hipMalloc, UpdateDevice (hipMemcpy from pinned host
    memory), selfgpu_model2d_rk3 on the handle's default (blocking) stream,
    UpdateHost (hipMemcpy back).  Returns the device time of args.steps such
    solves (CUDA events on the legacy default stream, which the copies and the
    engine's blocking stream are ordered with) and the bytes copied per step."""
    import torch
    L = S.lib()
    interp = geo.interp
    h = ctypes.c_void_p()
    S.check(L.selfgpu_model2d_create(ctypes.byref(h), S.MODEL_CIG, N, NEL, S.FP64, None))
    S.check(L.selfgpu_model2d_set_kernel(h, 0 if args.kernel == "per-element" else 1))
    S.check(L.selfgpu_model2d_set_multistage(h, 1 if args.kernel == "multistage" else 0))
    mats = [np.asfortranarray(m) for m in (interp.dgMatrix, interp.bMatrix, interp.qWeights)]
    S.check(L.selfgpu_model2d_set_interp(h, *[m.ctypes.data_as(ctypes.c_void_p) for m in mats]))
    si = np.asfortranarray(mesh.sideInfo)
    dp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    S.check(L.selfgpu_model2d_set_geometry(h, dp(geo.dsdx), dp(geo.J), dp(geo.nHat), dp(geo.nScale),
                                           dp(mesh.sideInfo_d), si.ctypes.data_as(ctypes.c_void_p)))
    S.check(L.selfgpu_model2d_set_params(h, 1.0, 0.0, GAMMA, 1.0))
    host_q = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True)
    host_q.copy_(q0.cpu())
    host_out = torch.empty_like(host_q).pin_memory()
    nbytes = host_q.numel() * 8
    d_q, d_g = ctypes.c_void_p(), ctypes.c_void_p()
    if L.hipMalloc(ctypes.byref(d_q), nbytes) or L.hipMalloc(ctypes.byref(d_g), nbytes):
        raise RuntimeError("hipMalloc failed")
    zero = torch.zeros_like(host_q).pin_memory()
    L.hipMemcpy(d_g, ctypes.c_void_p(zero.data_ptr()), nbytes, 1)  # the RK register starts at zero (H21)
    S.check(L.selfgpu_model2d_set_state(h, d_q, d_g))

    def solve():
        if L.hipMemcpy(d_q, ctypes.c_void_p(host_q.data_ptr()), nbytes, 1):
            raise RuntimeError("hipMemcpy H2D failed")
        S.check(L.selfgpu_model2d_invalidate(h))
        S.check(L.selfgpu_model2d_rk3(h, dt, STEPS_PER_SOLVE))
        if L.hipMemcpy(ctypes.c_void_p(host_out.data_ptr()), d_q, nbytes, 2):
            raise RuntimeError("hipMemcpy D2H failed")

    for _ in range(max(1, args.warmup)):
        solve()
    S.check(L.selfgpu_model2d_sync(h))
    from self_b200 import replicas as R
    R.barrier()
    leg = torch.cuda.default_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(leg)
    for _ in range(args.steps):
        solve()
    e1.record(leg)
    torch.cuda.synchronize()
    S.check(L.selfgpu_model2d_check_finite(h))
    S.check(L.selfgpu_model2d_destroy(h))
    L.hipFree(d_q)
    L.hipFree(d_g)
    return e0.elapsed_time(e1), int(nbytes), int(nbytes)


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
    S.lib().selfgpu_model2d_set_kernel(model._h, 0 if args.kernel == "per-element" else 1)
    S.lib().selfgpu_model2d_set_multistage(model._h, 1 if args.kernel == "multistage" else 0)
    q0 = initial_state(geo.x)
    torch.cuda.synchronize()
    dt = cfl_dt(geo.CovariantArcMin(), q0[:, 2].min().item())
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
    persistent0 = S.lib().selfgpu_model2d_persistent_launch_count(model._h)
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
        while not ends[-1].query():  # poll with the GIL released, so the clock sampler runs
            time.sleep(0.002)
        torch.cuda.synchronize()
    R.barrier()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    launches = model.LaunchCount() - launches0  # stage-kernel launches (plus one trace prologue per solve)
    persistent = S.lib().selfgpu_model2d_persistent_launch_count(model._h) - persistent0
    # RK stages per launch of the persistent kernel: 1, or all 3 x 200 of a
    # solve when the multi-stage launch applies (the default for this form)
    stages_per_launch = max(1, round(3 * STEPS_PER_SOLVE * args.steps / persistent)) if persistent else 1
    clk = clocks.summary()
    t_max = R.max_over_ranks(ms)
    value = R.aggregate_rate(DOF * STEPS_PER_SOLVE * args.steps, world, t_max / 1e3)
    stage_ms = ms / (args.steps * 3 * STEPS_PER_SOLVE)
    per_stage = algorithmic_bytes_per_element_stage() * NEL
    per_launch = per_stage * stages_per_launch
    launch_ms = stage_ms * stages_per_launch
    achieved = per_launch / (launch_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic = recorded_traffic(stages_per_launch > 1)
    if traffic is not None:
        traffic *= stages_per_launch

    model.CheckFinite()
    e2e_ms, h2d, d2h = e2e_through_c_abi(S, mesh, geo, q0, dt, args)
    e2e_ms = R.max_over_ranks(e2e_ms)
    e2e = R.aggregate_rate(DOF * STEPS_PER_SOLVE * args.steps, world, e2e_ms / 1e3)

    if rank != 0:
        return
    line = {
        "metric": "DOF-updates/s", "value": value, "unit": "DOF-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(dt, world),
        "form": "SELFGPU_FP64 (production FP64: multiply-add contraction, reciprocal products)",
        "e2e": {"value": e2e, "unit": "DOF-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "hipMemcpy (HIP shim) H2D from pinned host -> selfgpu_model2d_rk3 (C ABI, default "
                        "stream) -> hipMemcpy D2H"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "bytes_per_launch": per_launch, "launch_ms": launch_ms, "stages_per_launch": stages_per_launch,
                     "kernel": ("k_fused_stage_tma<8,PhysCIG,double,true> (all RK stages of a 200-step solve in "
                                "one launch)" if stages_per_launch > 1 else
                                ("k_fused_stage_tma<8,PhysCIG,double>" if persistent else
                                 "k_fused_stage<8,PhysCIG,double>") + " (one RK stage over all elements)")},
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
    ap.add_argument("--model", default="CIG", choices=["LSW", "SW", "CIG"], help="--form kernel: model")
    ap.add_argument("--N", type=int, default=7, help="--form kernel: degree")
    ap.add_argument("--nx", type=int, default=128, help="--form kernel: elements per direction")
    ap.add_argument("--fp", default="fp64", choices=["fp64", "fp64_ref", "fp32"], help="--form kernel: form")
    ap.add_argument("--kernel-steps", type=int, default=5, help="--form kernel: timed RK3 steps")
    ap.add_argument("--form", choices=["c1", "c2", "c4", "c5", "ensemble", "gas_ensemble", "kernel"], default=None,
                    help="run only this form's measurement and print its JSON (diagnostic mode)")
    ap.add_argument("--cpu-table", action="store_true",
                    help="print the CPU-baseline table of configs C1-C5 (oracle port) and exit")
    ap.add_argument("--kernel", default="multistage", choices=["persistent", "multistage", "per-element"],
                    help="stage kernel: persistent bulk-copy kernel (one launch per RK stage, or, multistage, "
                         "all stages of a call in one launch where that applies) or one CTA per element group")
    args = ap.parse_args()
    if args.cpu_table:
        print(json.dumps(run_cpu_table()), flush=True)
        return
    if args.form:
        print(json.dumps(run_one_form(args.form, args)), flush=True)
        return
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
