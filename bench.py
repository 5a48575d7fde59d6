#!/usr/bin/env python
"""Benchmark of the B200 smoke step: Mcell-steps/s on the 128^3 plume.

Workload (the configuration the headline metric is quoted on): a 128^3 MAC
grid, seed-0 velocity noise in [-0.01, 0.01], a sphere source at
(64, 12.8, 64) with radius 10 cells assigning density = temperature = 1 each
step, alpha 0.08, beta 0.4, eps 0.3, dt = 0.5 h, 200 steps.  A "step" is one
FluidSolver3D::step (advection of u, v, w; source; confinement + buoyancy;
projection with the pressure solve; advection of density and temperature;
telemetry).

Forms measured in one run:
  fp64_cg   (headline `value`)  the plain f64 drop-in, CG to 1e-6 (max 200): the
                               same arithmetic as the f64 reference arm
  mixed_cg                     f32 stencils/SpMV, f64 dots, f64 refinement to 1e-6
                               (in `variants`, with its speed-up over fp64_cg and
                               its relative L2 difference from it)
  fp64_sor / mixed_sor         red-black SOR omega = 1.7, 80 sweeps per step
Each form runs W untimed warm-up steps, is re-initialised (outside the timed
region) and then times exactly K steps from the initial state on the device
(CUDA events on the solver's stream, barrier + synchronize on both sides, max
over ranks).  `e2e` repeats the headline form through the public API with
host buffers: the initial fields are uploaded from pinned host memory, every
step returns its telemetry to the host (as FluidSolver3D::step does), and the
final density/temperature hand-off (FluidMedium::from_solver) is downloaded.

`--impl reference` times the CPU oracle (a C++ restatement of the reference's
single-threaded Rust solver; the Rust crate cannot be built in this image) on
a bounded sample of the same workload in f64.

Multi-GPU: the single simulation does not shard; N ranks run N independent
replicas (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "aether-core-engine_b200"))

METRIC = ("Mcell-steps/s 128³: FP32+FP64-refine vs FP64 GPU @1e-5 err; "
          "adjoint/fwd ratio")
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128, help="grid edge (default 128)")
    ap.add_argument("--seed", type=int, default=0, help="velocity-noise seed (default 0)")
    ap.add_argument("--poisson-kernel", type=int, default=0,
                    help="CG kernel: 0 auto, 1 streaming, 2 on-chip resident")
    ap.add_argument("--forms", default="fp64_cg,mixed_cg,fp64_sor,mixed_sor")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the 48-plume batched-ensemble measurement")
    ap.add_argument("--ensemble-steps", type=int, default=100)
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 256^3 x 100-step mixed/FP64 measurement")
    ap.add_argument("--no-medium", action="store_true",
                    help="skip the device medium-query measurement")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the reverse-mode (adjoint) measurement")
    ap.add_argument("--adjoint-directions", type=int, default=16,
                    help="finite-difference directions checked against the adjoint")
    ap.add_argument("--cpu-seconds", type=float, default=20.0,
                    help="target length of the bounded CPU sample")
    ap.add_argument("--reference-seconds", type=float, default=150.0,
                    help="time bound of the reference arm's timed steps")
    return ap.parse_args()


SEED = 0
POISSON_KERNEL = 0


def plume_for(form: str, n: int, seed: int | None = None):
    from aether_fluid.plume import Plume
    seed = SEED if seed is None else seed
    if form.endswith("sor"):
        return Plume(n, n, n, 200, seed=seed, solver="sor", iters=80)
    return Plume(n, n, n, 200, seed=seed)


def bench_config(form: str, n: int, world: int) -> dict:
    """The `config` object of a bench line; both arms print the same one."""
    p = plume_for(form, n)
    c = ",".join(f"{x:g}" for x in p.center)
    workload = (f"smoke plume {n}x{n}x{n}, sphere source r={p.radius:g} at ({c}), "
                f"seed {p.seed}, dt=0.5h")
    return {"workload": workload, "form": form, "grid": [n] * 3,
            "solver": "CG rel 1e-6 max 200" if "cg" in form else "RB-SOR omega 1.7 x 80",
            "parallelism": f"replicas x{world}",
            "l2": "state larger than L2 (no flush between steps)"}


# ---------------------------------------------------------------- clocks -----
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    QUERY = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus_id = (bus_id or "").lower()
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        rows = self.rows
        if self.bus_id:
            mine = [r for r in rows if r[0].lower().startswith(self.bus_id)]
            rows = mine or rows
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------ byte model -----
def poisson_bytes(n_cells: int, form: str, infos) -> float:
    """Algorithmic bytes of the Poisson kernel over the given solves: per cell,
    f64 CG 32 (init) + 88 per iteration; mixed CG 52 per refinement pass + 44
    per inner iteration; SOR 24 per sweep (f64) / 12 (f32) plus, for the mixed
    form, 52 for its one f64 residual/correction pass."""
    total = 0.0
    for inf in infos:
        if form == "fp64_cg":
            total += 32 + 88 * inf.iterations
        elif form == "mixed_cg":
            total += 52 * max(inf.refinements, 1) + 44 * inf.iterations
        elif form == "fp64_sor":
            total += 24 * inf.iterations
        else:
            total += 52 + 12 * inf.iterations
    return total * n_cells


def step_bytes(n_cells: int, form: str, infos) -> float:
    """Whole-step algorithmic bytes: f64 CG 336 + 88*N_it, f64 SOR 304 + 24*S,
    mixed CG 160 + 52*R + 44*N_in, mixed SOR 160 + 52 + 12*S."""
    total = 0.0
    for inf in infos:
        if form == "fp64_cg":
            total += 336 + 88 * inf.iterations
        elif form == "fp64_sor":
            total += 304 + 24 * inf.iterations
        elif form == "mixed_cg":
            total += 160 + 52 * max(inf.refinements, 1) + 44 * inf.iterations
        else:
            total += 160 + 52 + 12 * inf.iterations
    return total * n_cells


# Algorithmic bytes per cell of each timed stage (each stage reads each distinct
# input array once and writes each output once, at its stored precision;
# intermediates count 0): advect = u, v, w, density and temperature;
# forces = confinement + buoyancy + wall BC; telemetry is counted as fused
# into the scalar advection (0 bytes of its own).
STAGE_BYTES = {"fp64": {"advect": 96 + 56, "forces": 64, "divergence": 32, "project": 56},
               "mixed": {"advect": 48 + 28, "forces": 32, "divergence": 20, "project": 32}}


def stage_fractions(form: str, cells: int, r: dict, peak: float) -> dict:
    """Per stage: algorithmic GB/s over the stage's event-timed duration, as a
    fraction of the measured HBM peak; the Poisson stage uses the solver
    reports' iteration counts."""
    kind = "mixed" if form.startswith("mixed") else "fp64"
    steps = len(r["infos"])
    out = {}
    for stage, per_cell in STAGE_BYTES[kind].items():
        ms = r["stages"][stage][0]
        if ms > 0:
            out[stage] = per_cell * cells * steps / (ms / 1e3) / 1e9 / peak
    pms = r["stages"]["poisson"][0]
    if pms > 0:
        out["poisson"] = poisson_bytes(cells, form, r["infos"]) / (pms / 1e3) / 1e9 / peak
    return out


def time_large(torch, n: int = 256, steps: int = 100, seed: int = 1) -> dict:
    """The 256^3 x 100-step plume (seed 1, source (128, 25.6, 128) r = 20) in
    the mixed and FP64 CG forms: throughput, whole-step and per-stage fractions
    of the measured HBM peak (state far larger than L2), and the mixed/FP64
    ratio."""
    peak, _ = measured_peak()
    out = {"grid": [n, n, n], "steps": steps, "seed": seed}
    for form in ("mixed_cg", "fp64_cg"):
        r = time_form(form, n, steps, 3, None, torch, 0, seed=seed)
        cells = r["cells"]
        its = [i.iterations for i in r["infos"]]
        out[form] = {"value": cells * steps / (r["ms"] / 1e3) / 1e6,
                     "ms_per_step": r["ms"] / steps,
                     "mean_solver_iters": sum(its) / len(its),
                     "step_roofline_frac": step_bytes(cells, form, r["infos"]) / (r["ms"] / 1e3)
                     / 1e9 / peak,
                     "stage_roofline_frac": stage_fractions(form, cells, r, peak),
                     "stage_ms": {k: round(v[0], 3) for k, v in r["stages"].items()},
                     "poisson_plan": r["plan"]}
    out["mixed_over_fp64"] = out["mixed_cg"]["value"] / out["fp64_cg"]["value"]
    return out


# DRAM bytes per launch of the Poisson kernel: dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu capture of that kernel on the same workload
# (one solve of the plume at that grid edge).  Keyed by (kernel, grid edge);
# any other kernel or workload reports null.  A capture is not taken inside
# this script: ncu replays each launch many times, so its figure is recorded
# here beside the kernel it belongs to.
NCU_TRAFFIC = {("k_cg_res_f64", 128): 59.88e6 + 2362.94e6,
               ("k_cg_res_mixed", 128): 40.0e6 + 2.8e6,
               ("k_cg_stream_f64", 256): 119.02e9 + 80.63e9,
               ("k_cg_stream_mixed", 256): 52.4e9 + 40.9e9}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------- our arm ----
def time_form(form: str, n: int, steps: int, warmup: int, dist, torch, rank: int,
              seed: int | None = None):
    """K steps of one form from the initial state, timed on the solver's
    stream with CUDA events (barrier + synchronize on both sides).  A second,
    identical pass with per-stage CUDA events gives the stage breakdown and the
    Poisson kernel's time for the roofline; it is kept out of the headline
    because the extra events cost a few per cent of a step."""
    import aether_fluid as af
    p = plume_for(form, n, seed)
    s = p.build(precision=af.Precision.MIXED if form.startswith("mixed") else af.Precision.FP64)
    s.set_params(poisson_kernel=POISSON_KERNEL)
    if warmup > 0:
        s.run(warmup, p.dt, 0.0, p.dt)
    s.init_velocity_noise(p.seed)  # back to the initial state, outside the timed region
    stream = torch.cuda.ExternalStream(s.stream)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    plan = s.poisson_plan()
    launches0 = s.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start.record(stream)
    tel, infos = s.run(steps, p.dt, 0.0, p.dt)
    end.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(end)
    launches = s.launch_count() - launches0
    fields = {f: s.get_field(f) for f in ("u", "v", "w", "density", "temperature")}
    # the stage breakdown: the same K steps again, with per-stage events
    s.init_velocity_noise(p.seed)
    s.set_stage_timing(True)
    torch.cuda.synchronize()
    s.run(steps, p.dt, 0.0, p.dt)
    torch.cuda.synchronize()
    stages = s.stage_timing()
    s.set_stage_timing(False)
    s.close()
    return {"ms": ms, "infos": infos, "tel": tel, "stages": stages, "launches": launches,
            "fields": fields, "cells": p.cells, "plan": plan}


def time_e2e(form: str, n: int, steps: int, warmup: int, dist, torch):
    """Headline form through the public API with host buffers."""
    import aether_fluid as af
    from aether_fluid import _lib
    p = plume_for(form, n)
    s = p.build(precision=af.Precision.MIXED if form.startswith("mixed") else af.Precision.FP64)
    # The initial condition, generated once on the host into pinned memory.
    s.init_velocity_noise(p.seed)
    init = {f: torch.empty(p.cells, dtype=torch.float64, pin_memory=True)
            for f in ("u", "v", "w")}
    for f, t in init.items():
        t.numpy()[:] = s.get_field(f)
    out_d = torch.empty(p.cells, dtype=torch.float64, pin_memory=True)
    out_t = torch.empty(p.cells, dtype=torch.float64, pin_memory=True)
    lib = _lib.load()
    dp = ctypes.POINTER(ctypes.c_double)

    def one_run(k):
        # host -> device: the step inputs (initial velocity) from pinned memory
        for fid, f in enumerate(("u", "v", "w")):
            _lib.check(lib.afl_upload_field(s._h, fid, ctypes.cast(init[f].data_ptr(), dp),
                                            p.cells))
        tel = [s.step(p.dt, step * p.dt) for step in range(k)]  # telemetry per step
        mx = ctypes.c_double()
        _lib.check(lib.afl_medium_handoff(s._h, ctypes.cast(out_d.data_ptr(), dp),
                                          ctypes.cast(out_t.data_ptr(), dp), p.cells,
                                          ctypes.byref(mx)))
        return tel

    one_run(warmup)                      # warm-up pass
    s.init_velocity_noise(p.seed)        # reset density/temperature/pressure (untimed)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    one_run(steps)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    if dist:
        t = torch.tensor([el], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el = float(t.item())
    s.close()
    h2d = 3 * p.cells * 8
    d2h = steps * 64 + 2 * p.cells * 8 + 8
    return {"seconds": el, "h2d_per_step": h2d / steps, "d2h_per_step": d2h / steps}


def time_ensemble(steps: int, torch, dist=None):
    """The 48-plume ensemble (mixed CG to 1e-6) through the sharded-ensemble
    API: each rank advances a cell-balanced share of the instances as one
    batched, graph-captured ensemble on its GPU in the default step form (one
    persistent launch per step; no data-path collective; a host-side gather
    returns the results to rank 0).  Whole-job time is the slowest rank's.  At
    one GPU the same 48 plumes also run in the other step form (per-stage
    launches) and one at a time through single-grid solvers, for comparison."""
    import aether_fluid as af
    from aether_fluid.ensemble import plume48
    from aether_fluid.sharding import run_sharded
    specs = plume48()
    cells = sum(s.cells for s in specs)
    if dist:
        dist.barrier()
    res = run_sharded(specs, steps, dist=dist, precision=af.Precision.MIXED)
    world = dist.get_world_size() if dist else 1
    if res is None:                      # ranks other than 0
        return None
    _, infos, parts = res
    batched = max(p.get("run_seconds", 0.0) for p in parts)
    its = [i.iterations for row in infos for i in row]
    out = {"instances": len(specs), "cells": cells, "steps": steps, "ranks": world,
           "batched_mcell_steps_per_s": cells * steps / batched / 1e6,
           "batched_s": batched, "mean_solver_iters": float(sum(its) / len(its)),
           "per_rank": [{"rank": p["rank"], "instances": len(p["indices"]),
                         "cells": p.get("cells", 0), "run_s": p.get("run_seconds"),
                         "graph": p.get("info", {}).get("graph"),
                         "persistent_step": p.get("info", {}).get("persistent"),
                         "solver_ctas": p.get("info", {}).get("solver_ctas"),
                         "tile_depth": p.get("info", {}).get("tile_depth"),
                         "autotune_choice": p.get("autotune_choice")} for p in parts]}
    if world == 1:
        single_s = 0.0
        for sp in specs:
            s = af.FluidSolver3D(sp.nx, sp.ny, sp.nz, precision=af.Precision.MIXED)
            s.set_params(vorticity_eps=sp.eps, buoyancy_beta=sp.beta, gravity_alpha=sp.alpha,
                         solver_kind=0, solver_iters=200, cg_rel_tol=1e-6)
            s.init_velocity_noise(sp.seed, -sp.noise, sp.noise)
            s.set_sphere_source(sp.center, sp.radius)
            s.run(1, sp.dt)                 # warm the kernels (untimed)
            s.init_velocity_noise(sp.seed, -sp.noise, sp.noise)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.run(steps, sp.dt, 0.0, sp.dt)
            torch.cuda.synchronize()
            single_s += time.perf_counter() - t0
            s.close()
        out["one_at_a_time_mcell_steps_per_s"] = cells * steps / single_s / 1e6
        out["one_at_a_time_s"] = single_s
        out["speedup"] = single_s / batched
        # the other step form: the graph of per-stage launches (the default is
        # one persistent launch per step), autotuned the same way
        from aether_fluid.ensemble import Ensemble
        ens = Ensemble(specs, precision=af.Precision.MIXED)
        ens.set_persistent(False)
        choice = ens.autotune()
        t0 = time.perf_counter()
        ens.run(steps)
        graph_s = time.perf_counter() - t0
        info = ens.info()
        ens.close()
        out["stage_graph"] = {"mcell_steps_per_s": cells * steps / graph_s / 1e6,
                              "s": graph_s, "solver_ctas": info["solver_ctas"],
                              "tile_depth": info["tile_depth"],
                              "autotune_choice": choice,
                              "default_over_stage_graph": graph_s / batched}
    return out


def time_adjoint(ndir: int, torch, n: int = 96, steps: int = 64, every: int = 8):
    """Reverse mode through the FP64 step on the 96^3 adjoint workload:
    controls are the initial velocity (seed-0 noise in [-0.01, 0.01], wall BC)
    and the source's temperature amplitude map (seed 2, uniform in [0.5, 1.5]);
    L = 0.5*|rho_final - rho_target|^2 after `steps` steps, the target being
    the density of a run whose source sits 8 cells further in x; a checkpoint
    every `every` steps; pressure solves to 1e-12 so that the discrete forward
    is the one the adjoint differentiates.  Reports device times of one
    forward and one backward (recompute + adjoint) after a warm-up pair, and
    central differences along `ndir` seeded unit directions of the control
    space (velocity parts wall-masked) at eps 1e-4, 1e-6 and 1e-7 against the
    adjoint's directional derivative: the step is piecewise smooth (limiter
    switches), so the difference error falls with eps until round-off."""
    import numpy as np
    from aether_fluid.adjoint import Adjoint
    from aether_fluid.ensemble import rng_f64
    cells = n ** 3
    noise = rng_f64(0, 0, 3 * cells)
    dt = 0.5 / n
    center, radius = (n / 2, 0.1 * n, n / 2), 5.0 * n / 64.0

    def make(c):
        return Adjoint(n, n, n, center=c, radius=radius, checkpoint_every=every,
                       cg_rel_tol=1e-12, solver_iters=4000)

    tgt_solver = make((center[0] + 8.0, center[1], center[2]))
    adj = make(center)
    u, v, w = adj.wall_masked(*(-0.01 + 0.02 * noise[a * cells:(a + 1) * cells]
                                for a in range(3)))
    ctl = (u, v, w, 0.5 + rng_f64(2, 0, cells))
    tgt = tgt_solver.forward(*ctl, steps, dt)
    tgt_solver.close()
    rho = adj.forward(*ctl, steps, dt)           # warm-up pair
    adj.backward(rho - tgt)
    torch.cuda.synchronize()
    rho = adj.forward(*ctl, steps, dt)
    grads = adj.backward(rho - tgt)
    st = adj.stats()
    gnorm = float(np.sqrt(sum(float(np.dot(g, g)) for g in grads)))
    rng = np.random.default_rng(11)

    def loss(xx):
        return 0.5 * float(np.sum((adj.forward(*xx, steps, dt) - tgt) ** 2))

    rel = {1e-4: [], 1e-6: [], 1e-7: []}
    for _ in range(ndir):
        d = [rng.standard_normal(cells) for _ in range(4)]
        d[0], d[1], d[2] = adj.wall_masked(d[0], d[1], d[2])
        nrm = np.sqrt(sum(float(np.dot(a, a)) for a in d))
        d = [a / nrm for a in d]
        ad = sum(float(np.dot(a, b)) for a, b in zip(grads, d))
        for eps, out in rel.items():
            fd = (loss([a + eps * b for a, b in zip(ctl, d)]) -
                  loss([a - eps * b for a, b in zip(ctl, d)])) / (2 * eps)
            out.append(abs(fd - ad) / abs(ad) if ad != 0 else float("inf"))
    adj.close()
    fd = {f"eps_{eps:.0e}": {"rel_err_max": max(r), "rel_err_median": float(np.median(r))}
          for eps, r in rel.items() if r}
    return {"grid": [n, n, n], "steps": steps, "checkpoint_every": every,
            "forward_ms": st["forward_ms"], "backward_ms": st["backward_ms"],
            "adjoint_fwd_ratio": st["backward_ms"] / st["forward_ms"],
            "forward_cg_iters": st["forward_cg_iters"], "adjoint_cg_iters": st["adjoint_cg_iters"],
            "gradient_norm": gnorm, "fd_directions": ndir, "fd": fd}


def time_medium(torch, n_rays: int = 1 << 20, cpu_rays: int = 4000) -> dict:
    """The renderer's medium queries (FluidMedium::transmittance and
    ::sample_interaction, src/fluid.rs:792-874) on the device: a 128^3 plume
    after 100 FP64 steps, the medium bounds and scales of the reference scene
    (src/main.rs:109: Aabb (-2.25, 0.22, -2.15)-(2.25, 5.15, 1.45), sigma_t
    scale 1.42, g 0.34), 2^20 rays from a camera-like origin towards uniform
    points of the box.  Rays/s through the public API with host buffers
    (copies included), next to the CPU oracle on a bounded sample of the same
    rays (1 core)."""
    import numpy as np
    import aether_fluid as af
    from aether_fluid.plume import Plume
    p = Plume(128, 128, 128, 100, seed=0)
    s = p.build()
    s.run(p.steps, p.dt, 0.0, p.dt)
    lo, hi = (-2.25, 0.22, -2.15), (2.25, 5.15, 1.45)
    m = af.DeviceMedium.from_solver(s, af.Aabb(lo, hi), 1.42, 0.34)
    rng = np.random.default_rng(0)
    o = np.tile([0.0, 2.4, 9.0], (n_rays, 1))
    target = rng.uniform(lo, hi, size=(n_rays, 3))
    rays = np.column_stack([o, target - o, np.full(n_rays, 1e-4), np.full(n_rays, 20.0)])
    m.transmittance(rays, 1)                 # warm-up at full size: staging buffers grown
    m.sample_interaction(rays, 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tr = m.transmittance(rays, 7)
    t_tr = time.perf_counter() - t0
    t0 = time.perf_counter()
    hit = m.sample_interaction(rays, 8)[0]
    t_int = time.perf_counter() - t0
    out = {"rays": n_rays, "grid": [128, 128, 128], "steps": p.steps,
           "transmittance_rays_per_s": n_rays / t_tr, "interaction_rays_per_s": n_rays / t_int,
           "mean_transmittance": float(tr.mean()), "interaction_fraction": float(hit.mean()),
           "h2d_bytes": int(rays.nbytes), "unit": "rays/s (host buffers, copies included)"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    d, q = s.get_field("density"), s.get_field("temperature")
    t0 = time.perf_counter()
    O.medium_transmittance(d, q, (128, 128, 128), lo, hi, 1.42, rays[:cpu_rays], 7)
    t_cpu = time.perf_counter() - t0
    out["cpu_oracle_transmittance_rays_per_s"] = cpu_rays / t_cpu
    out["cpu_sample"] = f"first {cpu_rays} rays, 1 core"
    m.close()
    s.close()
    return out


def cpu_sample(n: int, seconds: float):
    """The oracle (f64, 1 thread) on the first steps of the same plume until
    `seconds` of CPU time have been spent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    p = plume_for("fp64_cg", n)
    s = O.OracleSolver(p.nx, p.ny, p.nz)
    s.set_params(vorticity_eps=p.eps, buoyancy_beta=p.beta, gravity_alpha=p.alpha,
                 solver_kind=O.CG, solver_iters=p.iters, cg_rel_tol=p.rel_tol)
    s.init_velocity_noise(p.seed)
    s.set_sphere_source(p.center, p.radius)
    t0 = time.perf_counter()
    steps, iters = 0, []
    while True:
        s.step(p.dt, steps * p.dt)
        iters.append(s.last_cg_iters())
        steps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    return {"value": p.cells * steps / el / 1e6, "steps": steps, "seconds": el,
            "cg_iters": iters}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def summary(variants, large, ensemble, adjoint) -> dict:
    """The figures a reader looks for first, in a few short keys at the end of
    the line (the full sections come before it)."""
    r3 = lambda x: round(x, 3) if isinstance(x, (int, float)) else x  # noqa: E731
    out = {f"{k}_mcells": r3(v["value"]) for k, v in variants.items()}
    if "mixed_cg" in variants and "fp64_cg" in variants:
        out["mixed_over_fp64_128"] = r3(variants["mixed_cg"]["speedup_vs_fp64_cg"])
        out["mixed_rel_l2_vs_fp64"] = {f: float(f"{e:.2e}") for f, e in
                                       variants["mixed_cg"]["rel_l2_vs_fp64_cg"].items()}
    if large and "mixed_cg" in large:
        out["large_256"] = {
            "mixed_mcells": r3(large["mixed_cg"]["value"]),
            "fp64_mcells": r3(large["fp64_cg"]["value"]),
            "mixed_over_fp64": r3(large["mixed_over_fp64"]),
            "stage_frac_fp64": {k: r3(v) for k, v in
                                large["fp64_cg"]["stage_roofline_frac"].items()},
            "stage_frac_mixed": {k: r3(v) for k, v in
                                 large["mixed_cg"]["stage_roofline_frac"].items()}}
    if ensemble and "speedup" in ensemble:
        out["ensemble_mcells"] = r3(ensemble["batched_mcell_steps_per_s"])
        out["ensemble_speedup"] = r3(ensemble["speedup"])
        if "stage_graph" in ensemble:
            out["ensemble_stage_graph_mcells"] = r3(ensemble["stage_graph"]["mcell_steps_per_s"])
    if adjoint and "adjoint_fwd_ratio" in adjoint:
        out["adjoint_fwd_ratio"] = r3(adjoint["adjoint_fwd_ratio"])
        out["adjoint_fd_eps1e-7_max"] = adjoint["fd"].get("eps_1e-07", {}).get("rel_err_max")
    return out


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist
    else:
        torch.cuda.set_device(local)
    import aether_fluid as af
    af.load()

    forms = [f for f in args.forms.split(",") if f]
    headline = forms[0]
    props = torch.cuda.get_device_properties(local)
    try:
        bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}"
    except AttributeError:
        bus = None
    results = {}
    clocks = None
    for form in forms:
        sampler = ClockSampler(bus) if form == headline else None
        if sampler:
            sampler.start()
        r = time_form(form, args.n, args.steps, args.warmup, dist, torch, rank)
        if sampler:
            clocks = sampler.stop()
        ms = r["ms"]
        if dist:
            t = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        r["ms_max"] = ms
        results[form] = r

    e2e = None
    if not args.no_e2e:
        e2e = time_e2e(headline, args.n, args.steps, args.warmup, dist, torch)

    ensemble = None
    if not args.no_ensemble:
        try:
            ensemble = time_ensemble(args.ensemble_steps, torch, dist)
        except Exception as exc:  # reported, never hides the headline
            ensemble = {"error": str(exc)}

    large = None
    if not args.no_large and rank == 0:
        try:
            large = time_large(torch)
        except Exception as exc:  # reported, never hides the headline
            large = {"error": str(exc)}

    medium = None
    if not args.no_medium and rank == 0:
        try:
            medium = time_medium(torch)
        except Exception as exc:  # reported, never hides the headline
            medium = {"error": str(exc)}

    adjoint = None
    if not args.no_adjoint:
        try:
            adjoint = time_adjoint(args.adjoint_directions, torch)
        except Exception as exc:  # reported, never hides the headline
            adjoint = {"error": str(exc)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(args.n, args.cpu_seconds)

    if rank == 0:
        import numpy as np
        head = results[headline]
        cells = head["cells"]
        value = cells * args.steps * world / (head["ms_max"] / 1e3) / 1e6
        peak, peak_kind = measured_peak()
        pois_ms, pois_calls = head["stages"]["poisson"]
        pois_bytes = poisson_bytes(cells, headline, head["infos"])
        achieved = pois_bytes / pois_calls / (pois_ms / pois_calls / 1e3) / 1e9
        pois_kernel = {"mixed_cg": ("k_cg_res_mixed", "k_cg_stream_mixed"),
                       "fp64_cg": ("k_cg_res_f64", "k_cg_stream_f64"),
                       "fp64_sor": ("k_rbsor_f64",) * 2,
                       "mixed_sor": ("k_rbsor_mixed",) * 2}[headline][
                           0 if head["plan"]["resident"] else 1]
        variants = {}
        for form, r in results.items():
            its = [i.iterations for i in r["infos"]]
            sb = step_bytes(cells, form, r["infos"])
            variants[form] = {
                "value": cells * args.steps * world / (r["ms_max"] / 1e3) / 1e6,
                "ms_per_step": r["ms_max"] / args.steps,
                "mean_solver_iters": float(np.mean(its)),
                "max_solver_iters": int(np.max(its)),
                "converged_steps": int(sum(i.converged for i in r["infos"])),
                "step_roofline_frac": sb / (r["ms"] / 1e3) / 1e9 / peak,
                "stage_roofline_frac": stage_fractions(form, cells, r, peak),
                "stage_ms": {k: round(v[0], 3) for k, v in r["stages"].items()},
                "poisson_plan": r["plan"] if "cg" in form else None,
            }
        # accuracy of the mixed forms against the f64 GPU forms after K steps
        for mixed, ref in (("mixed_cg", "fp64_cg"), ("mixed_sor", "fp64_sor")):
            if mixed in results and ref in results:
                errs = {}
                for f, a in results[mixed]["fields"].items():
                    b = results[ref]["fields"][f]
                    den = float(np.linalg.norm(b))
                    errs[f] = float(np.linalg.norm(a - b) / den) if den > 0 else 0.0
                variants[mixed]["rel_l2_vs_" + ref] = errs
        if "mixed_cg" in variants and "fp64_cg" in variants:
            variants["mixed_cg"]["speedup_vs_fp64_cg"] = (
                variants["mixed_cg"]["value"] / variants["fp64_cg"]["value"])
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": head["ms_max"] / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64" if headline.startswith("mixed") else "f64",
            "data": "synthetic (seeded velocity noise, sphere source)",
            "config": bench_config(headline, args.n, world),
            "gpu_launches": int(head["launches"]),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": NCU_TRAFFIC.get((pois_kernel, args.n)),
                         "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                            "of one capture of this kernel on this workload"
                                            if (pois_kernel, args.n) in NCU_TRAFFIC else None),
                         "algorithmic_bytes_per_launch": pois_bytes / pois_calls,
                         "kernel": pois_kernel,
                         "note": ("on-chip resident solve: achieved is the algorithmic bytes a "
                                  "streaming CG would move over kernel time, an effective "
                                  "bandwidth that exceeds the HBM peak because r, d and the "
                                  "pressure stay on chip (TMEM, shared memory) and q in L2; "
                                  "traffic is "
                                  "the measured DRAM figure" if head["plan"]["resident"] else
                                  "streaming solve through HBM"),
                         "peak_source": peak_kind},
            "variants": variants,
            "large_256": large,
            "medium": medium,
            "ensemble": ensemble,
            "adjoint_fwd_ratio": adjoint.get("adjoint_fwd_ratio") if adjoint else None,
            "adjoint": adjoint,
        }
        if e2e:
            line["e2e"] = {"value": cells * args.steps * world / e2e["seconds"] / 1e6,
                           "unit": UNIT, "h2d_bytes_per_step": e2e["h2d_per_step"],
                           "d2h_bytes_per_step": e2e["d2h_per_step"]}
        if cpu:
            line["cpu_baseline"] = {
                "value": cpu["value"], "unit": UNIT, "cores": 1, "kind": "port",
                "sample": (f"first {cpu['steps']} steps of the same plume in f64 "
                           f"(CG iters {cpu['cg_iters']}), {cpu['seconds']:.1f} s on "
                           f"{cpu_model()}")}
        line["clocks"] = clocks
        line["summary"] = summary(variants, large, ensemble, adjoint)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """The reference arm: the CPU oracle (a C++ restatement of the reference's
    single-threaded Rust solver, which has no toolchain in this image) on the
    same workload, form and config as our arm, on one host core.  It runs W
    untimed warm-up steps, re-initialises the plume (untimed) and times
    exactly K steps from the initial state, as our arm does; a step is one
    full f64 plume step (about 3 s at 128^3).  Should K steps exceed the time
    bound, it stops early and reports the steps it timed."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    bound = max(args.reference_seconds, 10.0)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    p = plume_for("fp64_cg", args.n)
    s = O.OracleSolver(p.nx, p.ny, p.nz)
    s.set_params(vorticity_eps=p.eps, buoyancy_beta=p.beta, gravity_alpha=p.alpha,
                 solver_kind=O.CG, solver_iters=p.iters, cg_rel_tol=p.rel_tol)
    s.set_sphere_source(p.center, p.radius)
    s.init_velocity_noise(p.seed)
    t0 = time.perf_counter()
    warm = 0
    while warm < args.warmup and time.perf_counter() - t0 < bound / 4:
        s.step(p.dt, warm * p.dt)
        warm += 1
    s.init_velocity_noise(p.seed)  # back to the initial state (untimed)
    t0 = time.perf_counter()
    steps, iters = 0, []
    while steps < args.steps:
        s.step(p.dt, steps * p.dt)
        iters.append(s.last_cg_iters())
        steps += 1
        if time.perf_counter() - t0 >= bound:
            break
    el = time.perf_counter() - t0
    value = p.cells * steps / el / 1e6
    sample = (f"steps 0..{steps - 1} of the {args.n}^3 plume in f64 on 1 core "
              f"(CG iters {iters}); C++ restatement of the reference's single-threaded "
              f"Rust solver (no Rust toolchain here), {cpu_model()}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus,  # the launch's GPU count; the timed work ran on 1 CPU core
        "steps": steps, "warmup": warm, "ms_per_step": el * 1e3 / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded velocity noise, sphere source)",
        "config": bench_config("fp64_cg", args.n, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    global SEED, POISSON_KERNEL
    args = parse()
    SEED = args.seed
    POISSON_KERNEL = args.poisson_kernel
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
