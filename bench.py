"""Throughput of the fixed-background GRHD operator on B200.

Workload (default): Kerr-Schild torus, M = 1, spin 0.9, 256^3 cells on
[-40, 40]^3, ideal gas Gamma = 5/3, constant-ell torus (inner edge 6M,
pressure maximum at 12M, rho_peak 1) with a seeded 1e-3 relative density
perturbation, atmosphere rho_floor 1e-10 / pressure_floor 1e-12 /
v^2 cap 0.8, MUSCL-MC (theta 2) + HLLE, excision r < 1.5, classic RK4,
CFL 0.25, FP64.  A step is one RK4 step of the whole grid (4 RHS
evaluations, 4 stage combinations with post-stage con2prim/atmosphere, the
CFL reduction).  Metric: cell-updates/s (interior cells x steps / time).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank advances its own
replica of the grid (no data-path collective); value = all ranks' cell
updates / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELLS = 256
HALF_WIDTH = 40.0
SPIN = 0.9
GAMMA = 5.0 / 3.0
CFL = 0.25
SEED = 20261203 + 1
BYTES_PER_CELL_UPDATE = 720   # RK4, FP64 state: 440 B read + 280 B write
BYTES_PER_RHS_CELL = 80       # one RHS: 5 doubles read + 5 written
METRIC = "GRHD cell-updates/s (RK4 step, KS torus a=0.9, 256^3, FP64)"


def workload_config(n, precision="fp64"):
    return {
        "workload": f"kerr_schild_torus_a0.9_{n}^3_rk4_{precision}",
        "precision": precision,
        "grid": [n, n, n], "domain": [-HALF_WIDTH, HALF_WIDTH],
        "background": "KerrSchild M=1 a=0.9", "eos_gamma": GAMMA,
        "torus": {"inner_radius": 6.0, "pressure_max_radius": 12.0,
                  "rho_peak": 1.0, "density_perturbation": 1e-3,
                  "seed": SEED},
        "atmosphere": {"rho_floor": 1e-10, "pressure_floor": 1e-12,
                       "max_velocity_squared": 0.8},
        "recovery": {"max_iterations": 80, "pressure_floor": 1e-12,
                     "max_velocity_squared": 0.9},
        "reconstruction": "MUSCL-MC theta=2", "riemann": "HLLE",
        "integrator": "RK4", "cfl": CFL, "excision_radius": 1.5,
        "l2": "inputs larger than L2 (state 1.5 GB per grid)",
    }


# ----------------------------------------------------------------- GPU arm


def build_state(n, precision, device):
    """The torus workload (grdzhadzha_b200.workloads.kerr_schild_torus):
    operator and level with the seeded initial data on the device."""
    from grdzhadzha_b200 import workloads as W
    return W.kerr_schild_torus(n, spin=SPIN, half_width=HALF_WIDTH,
                               gamma=GAMMA, seed=SEED, precision=precision,
                               device=device)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "200"], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path:
            return None
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm = float(parts[1].split()[0])
                smax = float(parts[2].split()[0])
            except ValueError:
                continue
            rows.append((sm, smax, parts[5:9]))
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows
                          for i in range(4) if r[i].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


def run_ours(args, rank, world, local_rank):
    import torch

    device = f"cuda:{local_rank}"
    torch.cuda.set_device(local_rank)
    n = args.n
    op, lv = build_state(n, args.precision, device)
    cells = lv.num_cells
    dist = world > 1
    if dist:
        import torch.distributed as tdist

    # One step = the CFL speed of the current state + one RK4 step; the
    # speed is computed inside the previous step's last stage (the first
    # step computes it from the state).
    cfl_state = {"mi": 0.0}

    def step(t):
        dt, cfl_state["mi"], _ = op.advance_rk4_cfl(
            lv, CFL, time=t, max_inverse_dt=cfl_state["mi"])
        return t + dt

    t = 0.0
    for _ in range(args.warmup):
        t = step(t)
    torch.cuda.synchronize()
    if dist:
        tdist.barrier()
    op.profile(True)
    op.profile_read()
    launches0 = op.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # the timed steps run as one multi-step call (the driver pattern of
    # several steps between looks at the state); each step is the same
    # CFL speed + RK4 step as above
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        ev0.record()
        t, cfl_state["mi"], _ = op.advance_rk4_cfl_steps(
            lv, CFL, args.steps, time=t, max_inverse_dt=cfl_state["mi"])
        ev1.record()
        torch.cuda.synchronize()
    if dist:
        tdist.barrier()
    ms = ev0.elapsed_time(ev1)
    launches = op.launch_count() - launches0
    prof = op.profile_read()
    op.profile(False)
    if dist:
        x = torch.tensor([ms], dtype=torch.float64, device=device)
        tdist.all_reduce(x, op=tdist.ReduceOp.MAX)
        ms = float(x.item())
    value = cells * args.steps * world / (ms / 1e3)

    # ---- end to end through the API with host buffers: each step is one
    # grhd_advance_rk4_cfl_host call on a state in pinned host memory (its
    # inputs copied host -> device, the whole new state device -> host,
    # inside the call) ----
    host = torch.empty_like(lv.state, device="cpu").pin_memory()
    host.copy_(lv.state)
    e2e_steps = max(1, min(args.steps, 5))
    mi = cfl_state["mi"]
    # untimed: the first call allocates the context's device copy
    dt, mi, _, _, _ = op.advance_rk4_cfl_host(host, lv, CFL, time=t,
                                              max_inverse_dt=mi)
    t += dt
    torch.cuda.synchronize()
    if dist:
        tdist.barrier()
    ev0.record()
    for _ in range(e2e_steps):
        dt, mi, _, h2d, d2h = op.advance_rk4_cfl_host(host, lv, CFL, time=t,
                                                      max_inverse_dt=mi)
        t += dt
    ev1.record()
    torch.cuda.synchronize()
    e2e_ms = ev0.elapsed_time(ev1)
    if dist:
        x = torch.tensor([e2e_ms], dtype=torch.float64, device=device)
        tdist.all_reduce(x, op=tdist.ReduceOp.MAX)
        e2e_ms = float(x.item())
        tdist.barrier()
    e2e = {"value": cells * e2e_steps * world / (e2e_ms / 1e3),
           "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "steps": e2e_steps,
           "api": "grhd_advance_rk4_cfl_host (pinned host state)"}

    # ---- roofline of the dominant kernel ----
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom = max(prof, key=lambda k: prof[k][0])
    dom_ms, dom_n = prof[dom]
    per_launch_cells = {"faces": cells, "cells": cells, "ghosts": cells,
                        "stage": cells, "cfl": cells}[dom]
    per_cell_bytes = {"faces": BYTES_PER_RHS_CELL,
                      "cells": BYTES_PER_RHS_CELL,
                      "ghosts": BYTES_PER_RHS_CELL,
                      "stage": 200, "cfl": 40}[dom]
    alg_bytes = per_launch_cells * per_cell_bytes
    achieved = alg_bytes / (dom_ms / max(dom_n, 1) / 1e3) / 1e9
    # DRAM traffic per launch from the committed ncu capture of the same
    # kernel; a capture on a smaller grid is scaled by the cell count
    traffic, traffic_note, fp64_pipe = None, None, None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        if tr.get("kernel_class") == dom:
            g = int(tr["grid"])
            traffic = tr["dram_bytes_per_launch"] * (n / g) ** 3
            traffic_note = (f"ncu capture at {g}^3 scaled by cells"
                            if g != n else "ncu capture")
            if "fp64_pipe_active_pct" in tr:
                fp64_pipe = tr["fp64_pipe_active_pct"] / 100.0
    except (OSError, ValueError, KeyError):
        pass
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved,
                "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": traffic,
                "traffic_source": traffic_note, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": alg_bytes,
                "avg_launch_ms": dom_ms / max(dom_n, 1),
                # the pipe that binds this kernel (ncu, committed capture):
                # FP64 arithmetic, not HBM
                "fp64_pipe_active_frac_ncu": fp64_pipe,
                "step_frac_of_hbm_roofline":
                    value / world * BYTES_PER_CELL_UPDATE / 1e9 / hbm_peak}
    kernel_ms = {k: {"ms_total": v[0], "launches": v[1]}
                 for k, v in prof.items()}
    return {"value": value, "ms": ms, "e2e": e2e, "roofline": roofline,
            "clocks": clk.summary(), "launches": launches,
            "kernel_ms": kernel_ms, "state": lv, "op": op}


# ------------------------------------------------------ batched ensemble


def run_ensemble(count, steps, warmup, hbm_peak):
    """The batched ensemble (Michel + Kerr-Schild tori of sizes 32..128^3,
    one persistent launch per call, replayed from a CUDA graph, launch
    shape from the autotuner), timed in FP64 and in mixed precision.

    Both runs take the same step sizes, dt = min(CFL dt, 0.5 x the FP64
    CFL dt of the initial state) per member (the cap binds throughout), so
    that the mixed run's accretion rates are compared with the FP64 ones
    at the same times; the CFL speed is still computed in the launch every
    step."""
    import torch
    import grdzhadzha_b200 as G
    from grdzhadzha_b200 import workloads as W

    out = {}
    caps = None
    for prec in ("fp64", "mixed"):
        members, specs = W.batched_ensemble(count=count, precision=prec)
        cells = sum(lv.num_cells for _, lv in members)
        if caps is None:
            probe = G.Ensemble(members, cfl=CFL)
            probe.advance(0, use_graph=False)
            caps = [0.5 * CFL / probe.member_info(i)["max_inverse_dt"]
                    for i in range(len(members))]
            del probe
        ens = G.Ensemble(members, cfl=CFL, max_dt=caps)
        tune = ens.autotune(trial_steps=1)
        ens.advance(warmup, use_graph=False)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        l0 = ens.launch_count()
        with ClockSampler(torch.cuda.current_device()) as clk:
            torch.cuda.synchronize()
            ev0.record()
            ens.advance(steps, use_graph=True)
            ev1.record()
            torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        infos = [ens.member_info(i) for i in range(len(members))]
        value = cells * steps / (ms / 1e3)
        out[prec] = {
            "value": value, "unit": "cell-updates/s", "ms": ms,
            "steps": steps, "warmup": warmup, "members": len(members),
            "cells": cells, "tuning": tune, "clocks": clk.summary(),
            "gpu_launches": ens.launch_count() - l0,
            "step_frac_of_hbm_roofline":
                value * BYTES_PER_CELL_UPDATE / 1e9 / hbm_peak,
            "_info": infos, "_kind": [sp["kind"] for sp in specs],
            "sizes": sorted({sp["n"] for sp in specs}),
        }
        del ens, members
        torch.cuda.empty_cache()

    def rel(a, b):
        return abs(a - b) / abs(b) if b != 0.0 else None

    errs = {}
    a, b = out["mixed"].pop("_info"), out["fp64"].pop("_info")
    kinds = out["mixed"].pop("_kind")
    out["fp64"].pop("_kind")
    for kind in ("michel", "torus"):
        sel = [i for i, k in enumerate(kinds) if k == kind]
        for key in ("mdot", "mdot_integral"):
            e = [rel(a[i][key], b[i][key]) for i in sel]
            e = [x for x in e if x is not None]
            errs[f"{kind}_{key}_max_rel_err"] = max(e) if e else None
        errs[f"{kind}_time_max_rel_err"] = max(
            rel(a[i]["time"], b[i]["time"]) for i in sel)
        errs[f"{kind}_max_abs_mdot_fp64"] = max(abs(b[i]["mdot"])
                                                for i in sel)
    errs["note"] = ("Michel: Mdot through r = 4 of the transonic inflow; "
                    "torus: Mdot through r = 2.5, atmosphere inflow only "
                    "(the tori do not reach r = 2.5 within the run)")
    out["mixed"]["mdot_error_vs_fp64"] = errs
    return out


# ------------------------------------------------------ discrete adjoint


def run_adjoint(n, steps, every, fd_steps, hbm_peak):
    """The adjoint workload (Kerr-Schild torus a = 0.7, n^3 on [-20, 20]^3,
    J = integral of the accretion rate through r = 2.5 over `steps` RK4
    steps, checkpoint every `every`): forward and backward sweep timed with
    CUDA events, their ratio, the gradient; then, on a run of `fd_steps`
    steps with the sphere r = 5 inside the torus body (within the horizon
    over which J is smooth at the 1e-6 scale), the gradient against central
    differences with h = 1e-6 and 1e-7 relative (their spread shows how
    smooth J is at that scale)."""
    import torch
    from grdzhadzha_b200 import workloads as W
    from grdzhadzha_b200.adjoint import THETA_NAMES
    out = {"config": {"workload": f"adjoint_kerr_schild_torus_a0.7_{n}^3",
                      "steps": steps, "checkpoint_every": every,
                      "domain": [-20.0, 20.0], "accretion_radius": 2.5,
                      "torus": {"inner_radius": 3.5,
                                "pressure_max_radius": 6.0},
                      "parameters": list(THETA_NAMES), "dtype": "f64"}}
    op, adj = W.adjoint_torus(n=n, steps=steps, checkpoint_every=every)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    adj.forward()  # warm-up (allocation-free afterwards)
    torch.cuda.synchronize()
    l0 = adj.launch_count()
    ev[0].record()
    J = adj.forward()
    ev[1].record()
    grad = adj.backward()
    ev[2].record()
    torch.cuda.synchronize()
    fwd, bwd = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    cells = n ** 3
    out.update({
        "J": J, "gradient": dict(zip(THETA_NAMES, grad)), "dt": adj.dt,
        "forward_ms": fwd, "backward_ms": bwd,
        "backward_over_forward": bwd / fwd,
        "forward_cell_updates_per_s": cells * steps / (fwd / 1e3),
        "gpu_launches": adj.launch_count() - l0})
    # the adjoint checked without differences: the tangent-linear sweep
    # along the same steps and branches gives dJ.v, which must equal
    # <gradient, v>; over the whole run for a random direction (relative
    # to sum_k |g_k v_k|), and per parameter over the first 25 steps
    import numpy as np
    rng = np.random.default_rng(20261203)
    checks = []
    v = list(rng.uniform(-1.0, 1.0, 8))
    ev[0].record()
    _, dJ = adj.tangent(v)
    ev[1].record()
    torch.cuda.synchronize()
    out["tangent_sweep_ms"] = ev[0].elapsed_time(ev[1])
    want = float(np.dot(grad, v))
    scale = float(np.abs(np.asarray(grad) * np.asarray(v)).sum())
    checks.append({"steps": steps, "direction": "random",
                   "tangent": dJ, "adjoint": want,
                   "rel_err": abs(dJ - want) / scale})
    del adj, op
    torch.cuda.empty_cache()
    short = min(25, steps)
    for R in (2.5, 5.0):
        op, adj = W.adjoint_torus(n=n, steps=short, checkpoint_every=short,
                                  accretion_radius=R)
        adj.forward()
        g = adj.backward()
        for k, name in enumerate(THETA_NAMES):
            e = [0.0] * 8
            e[k] = 1.0
            _, dJ = adj.tangent(e)
            checks.append({"steps": short, "accretion_radius": R,
                           "direction": name, "tangent": dJ,
                           "adjoint": g[k],
                           "rel_err": abs(dJ - g[k]) / max(abs(g[k]), 1e-300),
                           "rel_err_of_norm": abs(dJ - g[k]) / max(
                               float(np.linalg.norm(g)), 1e-300)})
        del adj, op
        torch.cuda.empty_cache()
    out["tlm_check"] = checks
    if fd_steps > 0:
        op, adj = W.adjoint_torus(n=n, steps=fd_steps,
                                  checkpoint_every=min(every, fd_steps),
                                  accretion_radius=5.0)
        adj.forward()
        g = adj.backward()
        base = adj.theta()
        rows = {}
        for k, name in enumerate(THETA_NAMES):
            fds = []
            for rel in (1e-6, 1e-7):
                h = rel * max(abs(base[k]), 0.1)
                tp, tm = list(base), list(base)
                tp[k] += h
                tm[k] -= h
                fds.append((adj.forward(tp) - adj.forward(tm)) / (2 * h))
            rows[name] = {"adjoint": g[k], "central_difference": fds,
                          "rel_err": [abs(g[k] - f) / max(abs(f), 1e-300)
                                      for f in fds]}
        out["fd_check"] = {"steps": fd_steps, "accretion_radius": 5.0,
                           "h_rel": [1e-6, 1e-7], "rows": rows}
        del adj, op
        torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------ CPU oracle


class CpuBaseline:
    """The reference's algorithm on the host cores, on a bounded sample of
    the same workload: the central 128 x 128 columns of the 256^3 torus
    grid over nz mid-plane z planes, as one box stepped as z-slab boxes,
    one thread each (the reference's per-box loops, its MPI ranks standing
    as threads).  One sample is one complete step as the GPU arm's: the
    CFL bound of the current state, then one RK4 step (4 RHS evaluations,
    the stage combinations, the post-stage recoveries).

    kind "reference" (where oracle/_ref was built): GRDzhadzha's own
    operator, its headers compiled unmodified at -O3 -march=x86-64-v3
    against oracle/shim (oracle/ref_capi.cpp: the RK4 step from the
    operator's compute_rhs and update_conserved, slab ghosts exchanged
    between the RHS evaluations, slabs of 8 planes).  The reference has no
    excision: the sample runs without it (the cells inside the horizon
    near the hole then fail their recovery and are reset to the
    atmosphere, as the reference does).
    kind "port" (otherwise): the oracle's timing build
    (oracle/liborc_grhd_fast.so, -O3 with AVX2 + FMA), slabs of 16 planes,
    with the workload's excision.

    The sample's state is built by the oracle (torus + numpy-seeded 1e-3
    perturbation + recovery)."""

    PORT_BUILD = "gcc -O3 -march=x86-64-v3 -ffp-contract=fast"
    REF_BUILD = ("g++ -O3 -march=x86-64-v3 (GRDzhadzha's headers, "
                 "unmodified, against oracle/shim)")

    def __init__(self, threads):
        import ctypes as C
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import numpy as np
        import oracle_lib as O

        self.O, self.C = O, C
        self.threads = threads
        self.kind = "reference" if O.have_ref() else "port"
        self.build = self.REF_BUILD if self.kind == "reference" \
            else self.PORT_BUILD
        planes = 8 if self.kind == "reference" else 16
        O.set_threads(threads)
        n = N_CELLS
        dx = 2.0 * HALF_WIDTH / n
        c = 0.5 * n * dx
        p = O.default_params(background=O.BG_KERR_SCHILD, ks_mass=1.0,
                             ks_spin=SPIN, gamma=GAMMA, dx=dx,
                             center=(c, c, c), atmo_rho_floor=1e-10,
                             atmo_pressure_floor=1e-12,
                             atmo_max_velocity_squared=0.8,
                             rec_max_iterations=80,
                             rec_max_velocity_squared=0.9, limiter_theta=2.0,
                             excision_radius=(0.0 if self.kind == "reference"
                                              else 1.5))
        nxy = 128
        nz = min(n, planes * threads)
        box = O.Box()
        x0, z0 = n // 2 - nxy // 2, n // 2 - nz // 2
        for d, (lo, hi) in enumerate(((x0, x0 + nxy - 1),
                                      (x0, x0 + nxy - 1),
                                      (z0, z0 + nz - 1))):
            box.lo[d], box.hi[d] = lo, hi
            box.glo[d], box.ghi[d] = lo - 2, hi + 2
            box.dlo[d], box.dhi[d] = 0, n - 1
        box.comp_stride = (nxy + 4) * (nxy + 4) * (nz + 4)
        s = O.new_state(box)
        cfg = O.torus_config(total_mass=1.0, inner_radius=6.0,
                             pressure_max_radius=12.0, rho_peak=1.0,
                             max_velocity_squared=0.8)
        tp = O.make_torus(p, cfg, box, 0.0)
        O.fill_torus(p, cfg, tp, box, s, 0.0)
        rng = np.random.default_rng(SEED)
        V = O.state_view(box, s)
        V[O.RHO] *= 1.0 + 1e-3 * rng.uniform(-1, 1, V[O.RHO].shape)
        V[O.EPS] = V[O.PRESS] / ((GAMMA - 1.0) * V[O.RHO])
        O.fill_conserved_from_primitives(p, box, s)
        O.recover_primitives(p, box, s)
        O.set_threads(1)
        self.ranks = min(threads, nz // 2)
        if self.kind == "port":
            self.L = O.fast_lib()
            self.L.orc_set_threads(threads)
        self.p, self.box, self.s = p, box, s
        self.inv = np.array([1.0 / dx] * 3)
        self.t = 0.0
        self.cells = nxy * nxy * nz
        what = ("GRDzhadzha's own operator" if self.kind == "reference"
                else "the oracle's timing build")
        self.desc = (f"one RK4 step with its CFL bound (4 RHS evaluations, "
                     f"stage combinations, post-stage recoveries) of "
                     f"{what} ({self.build}; z-slab boxes of "
                     f"{nz // self.ranks}+ planes, one thread each"
                     + ("; no excision: the reference has none"
                        if self.kind == "reference" else "")
                     + f") over the central {nxy}x{nxy}x{nz} cells of the "
                     f"{n}^3 grid")

    def sample(self):
        """(cell-updates/s, seconds) of one step of the sample."""
        O, C = self.O, self.C
        if self.kind == "reference":
            t0 = time.perf_counter()
            dt, _, _ = O.ref_advance_rk4_cfl(self.p, self.box, self.s,
                                             self.t, CFL, ranks=self.ranks,
                                             fast=True)
            el = time.perf_counter() - t0
            self.t += dt
            return self.cells / el, el
        L = self.L
        err = O.Error()
        diag = O.Diag()
        mi = C.c_double()
        t0 = time.perf_counter()
        st = L.orc_compute_max_inverse_dt(C.byref(self.p), C.byref(self.box),
                                          O._dp(self.s), O._dp(self.inv),
                                          self.t, C.byref(mi), C.byref(err))
        if st:
            raise RuntimeError(f"oracle CFL bound failed ({st})")
        dt = CFL / max(mi.value, 1e-14)
        st = L.orc_advance_rk4(C.byref(self.p), C.byref(self.box),
                               O._dp(self.s), O._dp(self.inv), self.t, dt,
                               C.byref(diag), C.byref(err))
        el = time.perf_counter() - t0
        if st:
            raise RuntimeError(f"oracle RK4 step failed ({st})")
        self.t += dt
        return self.cells / el, el


# ------------------------------------------- widened rows (one GPU each)


def _time(fn, reps=5, warmup=2):
    """Average ms of fn() over reps calls, CUDA events on the current
    stream, after warm-up."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def run_widened(hbm_peak):
    """The library paths beyond the benchmarked step, each timed on its own
    (inputs larger than L2 except where stated): the operator on CCZ4-
    stored geometry, the multi-box level exchange, the split SSPRK2 of a
    multi-box level, the KITP disk-driver source terms, the diagnostics
    reduction and the halo pack of a slab face."""
    import torch
    import grdzhadzha_b200 as G
    from grdzhadzha_b200 import workloads as W
    from grdzhadzha_b200 import halo as H
    out = {}
    # operator on CCZ4-stored geometry, KS torus a = 0.9, 128^3 (660 MB)
    n = 128
    op, lv = W.kerr_schild_torus(n)
    inv = [1.0 / op.dx] * 3
    lv36 = op.ccz4_state(lv)
    cop = G.LevelDataFiniteVolumeOperator(G.IdealGasEOS(op.eos.adiabatic_index))
    rhs = lv36.new_rhs()
    ms = _time(lambda: cop.compute_rhs(rhs, lv36, inverse_dx_U=inv))
    frhs = lv.new_rhs()
    ms_f = _time(lambda: op.compute_rhs(frhs, lv))
    cells = lv.num_cells
    # algorithmic bytes: the 36-component state read once, 5 written
    alg = cells * (36 + 5) * 8
    out["ccz4_rhs_128"] = {
        "value": cells / (ms / 1e3), "unit": "cell-RHS/s", "ms": ms,
        "fixed_background_rhs_ms": ms_f,
        "hbm_frac": alg / (ms / 1e3) / 1e9 / hbm_peak,
        "note": "FP64, one thread per cell, each face evaluated by both of its cells (a face-tiled version measured slower)"}
    out["fixed_background_rhs_128"] = {
        "value": cells / (ms_f / 1e3), "unit": "cell-RHS/s", "ms": ms_f,
        "note": "one FP64 compute_rhs of the fixed-background operator "
                "(ghost fill, per-cell pass, face pass) on the same grid"}
    del lv36, rhs, cop
    # multi-box level: 256^3 cut into 8 z-slabs, exchange + split SSPRK2
    n = 256
    op, lv = W.kerr_schild_torus(n)
    slabs = H.slab_boxes((0, 0, 0), (n - 1, n - 1, n - 1), 8)
    boxes = []
    for lo, hi in slabs:
        b = G.LevelBox(lo=lo, hi=hi, ghost=2, domain_lo=(0, 0, 0),
                       domain_hi=(n - 1,) * 3)
        g = 2
        b.state.copy_(lv.state[:, lo[2]:hi[2] + 2 * g + 1])
        boxes.append(b)
    stages = [G.LevelBox(lo=b.lo, hi=b.hi, ghost=2, domain_lo=b.domain_lo,
                         domain_hi=b.domain_hi) for b in boxes]
    moved = sum(H.region_cells(lo_, hi_)
                for r in range(len(slabs))
                for _, lo_, hi_ in H.halo_plan(slabs, r, (0, 0, 0),
                                               (n - 1,) * 3)[1])
    ms = _time(lambda: G.level_exchange(boxes), reps=10)
    byts = moved * 11 * 8 * 2
    out["level_exchange_256_8slabs"] = {
        "value": byts / (ms / 1e3) / 1e9, "unit": "GB/s", "ms": ms,
        "bytes": byts, "hbm_frac": byts / (ms / 1e3) / 1e9 / hbm_peak,
        "note": "14 halo regions of 2 x 256^2 cells, read + written"}
    dt = 0.5 * op.compute_stable_dt(lv, cfl=CFL)
    ms_split = _time(lambda: op.advance_level_ssprk2(boxes, stages, dt),
                     reps=3, warmup=1)
    ms_fused = _time(lambda: op.advance_ssprk2(lv, dt=dt), reps=3, warmup=1)
    out["ssprk2_256_8slabs"] = {
        "value": lv.num_cells / (ms_split / 1e3), "unit": "cell-updates/s",
        "ms": ms_split, "single_box_fused_ms": ms_fused}
    # halo pack of one slab face (2 planes of 260^2 cells, 11 components)
    face = (0, 0, slabs[1][0][2]), (n - 1, n - 1, slabs[1][0][2] + 1)
    buf = torch.empty(11 * H.region_cells(*face), dtype=torch.float64,
                      device="cuda")
    reg = H.DeviceRegions()
    ms = _time(lambda: reg.pack(boxes[1], face[0], face[1], buf), reps=20)
    byts = buf.numel() * 8 * 2
    out["halo_pack_face_256"] = {
        "value": byts / (ms / 1e3) / 1e9, "unit": "GB/s", "ms": ms,
        "bytes": byts}
    # diagnostics reduction over the 256^3 torus
    ms = _time(lambda: op.disk_diagnostics(lv), reps=5)
    byts = lv.num_cells * 7 * 8
    out["disk_diagnostics_256"] = {
        "value": byts / (ms / 1e3) / 1e9, "unit": "GB/s", "ms": ms,
        "hbm_frac": byts / (ms / 1e3) / 1e9 / hbm_peak,
        "note": "7 state components read per cell; includes the host sum"}
    del boxes, stages, lv, op
    torch.cuda.empty_cache()
    # the binary-disk configuration (circumbinary Keplerian disk on the
    # time-dependent PN metric), 320^3 mixed, 3 RK4 steps
    op, lv = W.binary_disk(320, precision="mixed")
    st = {"t": 0.0, "mi": 0.0}

    def disk_steps():
        st["t"], st["mi"], _ = op.advance_rk4_cfl_steps(
            lv, CFL, 3, time=st["t"], max_inverse_dt=st["mi"])
    ms = _time(disk_steps, reps=2, warmup=1) / 3.0
    out["binary_disk_320_mixed"] = {
        "value": lv.num_cells / (ms / 1e3), "unit": "cell-updates/s",
        "ms_per_step": ms, "note": "RK4, CFL 0.25, volume-time source on"}
    del op, lv
    torch.cuda.empty_cache()
    # KITP source terms on a binary-PN disk, 128^3
    n = 128
    op, lv = W.binary_pn_disk(n)
    rhs = lv.new_rhs()
    for name, fn in (("kitp_viscous_128",
                      lambda: op.kitp_viscous_rhs(rhs, lv, time=0.0)),
                     ("kitp_sink_rhs_128",
                      lambda: op.kitp_sink_rhs(rhs, lv, time=0.0)),
                     ("kitp_sink_decay_128",
                      lambda: op.kitp_sink_decay(lv, 0.0, 1e-6))):
        ms = _time(fn, reps=5)
        out[name] = {"value": lv.num_cells / (ms / 1e3),
                     "unit": "cells/s", "ms": ms}
    # the disk driver's step (operator RHS + viscous stress, sink decay)
    dt = 0.5 * op.compute_stable_dt(lv, cfl=CFL)
    st = {"t": 0.0}

    def kitp_step():
        op.kitp_advance_ssprk2(lv, st["t"], dt, cfg)
        st["t"] += dt
    from grdzhadzha_b200.operator import kitp_config
    cfg = kitp_config()
    ms = _time(kitp_step, reps=3, warmup=1)
    out["kitp_ssprk2_step_128"] = {
        "value": lv.num_cells / (ms / 1e3), "unit": "cell-updates/s",
        "ms": ms, "note": "SSPRK2 step, FP64, viscosity and sinks on"}
    torch.cuda.empty_cache()
    return out


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# -------------------------------------------------------------------- main


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_CELLS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", choices=["fp64", "mixed"],
                    default="fp64")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the mixed 256^3 and batched-ensemble legs")
    ap.add_argument("--ensemble-count", type=int, default=96)
    ap.add_argument("--ensemble-steps", type=int, default=100)
    ap.add_argument("--adjoint-n", type=int, default=128)
    ap.add_argument("--adjoint-steps", type=int, default=400)
    ap.add_argument("--adjoint-every", type=int, default=25)
    ap.add_argument("--adjoint-fd-steps", type=int, default=4)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the adjoint leg and print its JSON")
    ap.add_argument("--widened-only", action="store_true",
                    help="run only the legs beyond the step and print their "
                         "JSON")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        threads = host_threads()
        cb = CpuBaseline(threads)
        for _ in range(args.warmup):
            cb.sample()
        secs = [cb.sample()[1] for _ in range(args.steps)]
        total = sum(secs)
        value = cb.cells * args.steps / total
        line = {
            "impl": "reference", "metric": METRIC, "value": value,
            "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": workload_config(N_CELLS),
            "cpu_baseline": {"value": value, "unit": "cell-updates/s",
                             "cores": threads, "kind": cb.kind,
                             "build": cb.build,
                             "sample": cb.desc,
                             "cells_per_step": cb.cells},
            "e2e": {"value": value, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return

    if args.adjoint_only:
        import torch
        torch.cuda.set_device(local_rank)
        print(json.dumps({"adjoint": run_adjoint(
            args.adjoint_n, args.adjoint_steps, args.adjoint_every,
            args.adjoint_fd_steps, None)}), flush=True)
        return

    if args.widened_only:
        import torch
        torch.cuda.set_device(local_rank)
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        print(json.dumps({"widened": run_widened(
            peaks.get("hbm_gbs", 6650.0))}), flush=True)
        return

    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                 device_id=torch.device(f"cuda:{local_rank}"))
    res = run_ours(args, rank, world, local_rank)
    variants = None
    if rank == 0 and world == 1 and not args.no_variants:
        import copy
        import torch
        hbm_peak = res["roofline"]["peak"]
        res.pop("state")
        res.pop("op")
        torch.cuda.empty_cache()
        variants = {}
        if args.precision == "fp64":
            margs = copy.copy(args)
            margs.precision = "mixed"
            mres = run_ours(margs, rank, world, local_rank)
            variants["mixed"] = {
                "value": mres["value"], "unit": "cell-updates/s",
                "ms_per_step": mres["ms"] / args.steps,
                "speedup_vs_fp64": mres["value"] / res["value"],
                "e2e": mres["e2e"]["value"], "clocks": mres["clocks"],
                "gpu_launches": mres["launches"],
                "step_frac_of_hbm_roofline":
                    mres["roofline"]["step_frac_of_hbm_roofline"],
                "kernel_ms": mres["kernel_ms"]}
            del mres
            torch.cuda.empty_cache()
        ens = run_ensemble(args.ensemble_count, args.ensemble_steps,
                           args.warmup, hbm_peak)
        ens["mixed"]["speedup_vs_fp64_plain"] = (
            ens["mixed"]["value"] / res["value"])
        variants["batched_ensemble"] = ens
        try:
            variants["widened"] = run_widened(hbm_peak)
        except Exception as e:  # a failing extra leg keeps the bench line
            variants["widened"] = {"error": repr(e)}
        torch.cuda.empty_cache()
        if not args.no_adjoint:
            variants["adjoint"] = run_adjoint(
                args.adjoint_n, args.adjoint_steps, args.adjoint_every,
                args.adjoint_fd_steps, hbm_peak)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        cb = CpuBaseline(threads)
        cb.sample()
        rate = max(cb.sample()[0] for _ in range(2))
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": threads,
               "kind": cb.kind, "build": cb.build,
               "sample": cb.desc, "cells_per_step": cb.cells}
    if rank == 0:
        line = {
            "metric": METRIC, "value": res["value"],
            "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": res["ms"] / args.steps,
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded torus initial data generated on the "
                    "device)",
            "config": dict(workload_config(args.n, args.precision),
                           parallelism=f"replicas x{world}"),
            "e2e": res["e2e"], "roofline": res["roofline"],
            "cpu_baseline": cpu, "clocks": res["clocks"],
            "gpu_launches": res["launches"], "kernel_ms": res["kernel_ms"],
        }
        if variants is not None:
            # the headline variants as top-level keys, ahead of the long
            # `variants` object
            mx = variants.get("mixed")
            if mx:
                line["mixed_value"] = mx["value"]
                line["mixed_speedup_vs_fp64"] = mx["speedup_vs_fp64"]
            ens = variants.get("batched_ensemble", {})
            if "fp64" in ens:
                line["batched_fp64_value"] = ens["fp64"]["value"]
            if "mixed" in ens:
                line["batched_mixed_value"] = ens["mixed"]["value"]
                line["batched_mixed_speedup_vs_fp64_plain"] = (
                    ens["mixed"]["speedup_vs_fp64_plain"])
            adj = variants.get("adjoint")
            if adj:
                line["adjoint_backward_over_forward"] = (
                    adj["backward_over_forward"])
                rows = adj.get("fd_check", {}).get("rows", {})
                if rows:
                    line["adjoint_fd_max_rel_err"] = max(
                        r["rel_err"][0] for r in rows.values())
                if "tlm_check" in adj:
                    line["adjoint_tlm_rel_err_400_steps"] = next(
                        c["rel_err"] for c in adj["tlm_check"]
                        if c["direction"] == "random")
                    for R in (2.5, 5.0):
                        line[f"adjoint_tlm_max_rel_err_of_norm_25_steps_r{R}"] \
                            = max(c["rel_err_of_norm"]
                                  for c in adj["tlm_check"]
                                  if c.get("accretion_radius") == R)
            line["variants"] = variants
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
