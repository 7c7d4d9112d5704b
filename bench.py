#!/usr/bin/env python
"""Benchmark: Sedov3D 256^3 hydro steps on B200, FP32-bulk vs plain FP64.

Workload ("sedov3d_256"): uniform 256^3 grid (levelmin = levelmax = 8, unit
box, zero-gradient outflow boundaries), gamma = 1.4, ambient rho = 1, v = 0,
p = 1e-5, total energy 1 deposited as uniform pressure within 2 cells of the
centre; MUSCL-Hancock, moncen slopes, HLLC, Courant 0.8.  Synthetic input built
here (no dataset).  A step is one full hydro step through the C ABI in the
reference's call order: rh_cmpdt (CFL dt + conserved totals, synchronous like
gpu_cmpdt_2), rh_set_unew, rh_godunov, rh_set_uold.

value        cell-updates/s of the FP32-bulk step (state resident in HBM)
fp64         the same for the plain FP64 step
e2e          FP32-bulk step with the reference's FP64 uold in pinned host
             memory, copied in and out every step: rh_coarse_step_host (the
             copies overlapped with the pencils); beside it the three
             separate calls rh_set_grid_device, rh_coarse_step,
             rh_transfer_grid_host
roofline     dominant kernel (godunov_pencil_kernel), algorithmic bytes per
             cell-update (48 B FP32-bulk, 80 B FP64) / CUDA-event kernel time
cpu_baseline the CPU restatement of the reference path (oracle/, OpenMP over
             oct blocks) timed on this host on one 256^3 step
batch        the 1024-problem Riemann/blast ensemble (sides 16-128, 50 steps)
             in one persistent launch per step, FP32-bulk and FP64, tile
             autotuned on the ensemble
serve        a Poisson stream of 2D/3D solve requests served with continuous
             batching; solve_latency_s holds its p50/p99 time-to-solution
accuracy     density/momentum/energy relative L1 of one FP32-bulk step against
             the FP64 oracle step from the same state

--impl reference runs the reference arm: the reference's CPU algorithm on the
host cores (the CPU restatement; the Fortran reference cannot be compiled in
this image), same workload and metric.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LEVEL = 8
B_ALG = {"fp64": 80.0, "fp32_bulk": 48.0}
WORKLOAD = "sedov3d_256"


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(prec):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "godunov_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    e = d.get(prec)
    return None if e is None else e.get("bytes_per_launch_256")


def profile_pipes(prec):
    """Pipe and issue fractions of the dominant kernel from the committed ncu
    summary (an ncu capture, not measured by this run)."""
    p = os.path.join(ROOT, "profiles", "godunov_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    e = d.get(prec)
    return None if e is None else e.get("pipes")


class ClockSampler:
    """SM clock and throttle reasons sampled (read-only NVML queries, every
    ~5 ms) while the timed region runs; falls back to nvidia-smi polling."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, device):
        self.device = device
        self.sm = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self.t = None

    def __enter__(self):
        try:
            import pynvml as N

            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
            masks = {k: getattr(N, v) for k, v in self.REASONS.items()}

            def run():
                while not self._stop.is_set():
                    self.sm.append(float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)))
                    r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                    for k, m in masks.items():
                        if r & m:
                            self.reasons.add(k)
                    time.sleep(0.005)

            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
        except Exception:
            self.t = None
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.t is not None:
            self.t.join(timeout=2)

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(self.sm)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.sm)}


def make_problem():
    from ramses2_b200._abi import HydroParams
    from ramses2_b200.mesh import sedov3d, uniform_mesh

    m = uniform_mesh(LEVEL, nsubgrid=1, bc="outflow")
    sedov3d(m, gamma=1.4, rho0=1.0, p0=1e-5, energy=1.0, radius_cells=2.0)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc")
    return m, P


def bench_config(world, ncell):
    """The workload description both arms print (same keys, same values)."""
    return {"workload": WORKLOAD, "grid": "256^3 uniform (levelmin=levelmax=8)", "problem": "Sedov3D",
            "riemann": "hllc", "slope": "moncen", "courant": 0.8, "boundary": "outflow",
            "cells": ncell, "parallelism": "replicas" if world > 1 else "single-gpu",
            "l2": "state (>=805 MB) larger than L2 (126 MB); no flush needed"}


def rel_l1(a, b):
    num = np.abs(a - b).sum(axis=(0, 2))
    den = np.abs(b).sum(axis=(0, 2))
    return (num / np.where(den > 0, den, 1.0)).tolist()


def time_steps(gpu, lib, steps, warmup):
    """Per-step device time (CUDA events on the library stream) of one
    rh_coarse_step call (courant_fine with its synchronous dt read-back,
    set_unew, godunov_fine, set_uold)."""
    from ramses2_b200._lib import check
    import ctypes as C

    for _ in range(warmup):
        gpu.coarse_step()
    gpu.sync()
    per = []
    ms = C.c_float()
    for _ in range(steps):
        check(lib.rh_timer_start(), "rh_timer_start")
        gpu.coarse_step()
        check(lib.rh_timer_stop(C.byref(ms)), "rh_timer_stop")
        per.append(ms.value)
    gpu.sync()
    return float(np.sum(per)) / steps, per


def kernel_time(gpu, steps, dt):
    gpu.bench_godunov(LEVEL, 2, dt)
    return gpu.bench_godunov(LEVEL, max(3, steps), dt)


def bench_batch(args, rank, world, dist):
    """The batched ensemble: riemann_blast_ensemble(args.batch_problems) split
    over the ranks (whole problems per GPU, no exchange), tile autotuned on the
    ensemble itself, then ``args.batch_steps`` steps of every problem timed
    with CUDA events (graph replays).  Returns per-precision results with the
    max-over-ranks time and the whole-job cell-updates/s."""
    from ramses2_b200.batch import Batch, ensemble_octs, riemann_blast_ensemble

    from ramses2_b200.ranks import max_over_ranks, shard

    ens_all = riemann_blast_ensemble(args.batch_problems, steps=args.batch_steps)
    ens = shard(ens_all, rank, world)
    noct = ensemble_octs(ens)
    out = {"workload": "%d independent 3D Riemann/blast problems, sides in {16..128}, %d steps each, HLLC, "
                       "moncen, split over %d GPU(s)" % (len(ens_all), args.batch_steps, world),
           "cells": ensemble_octs(ens_all) * 8}
    for prec in ("fp32_bulk", "fp64"):
        b = Batch(prec, slope_type=2, riemann="hllc", pool_octs=noct + 64, device=int(os.environ.get("LOCAL_RANK", 0)))
        for p, ic in ens:
            p.max_steps = 1 << 30
            b.add(p, ic)
        best, _ = b.tune()
        for pid in list(b.problems):
            b.remove(pid)
        pids = []
        for p, ic in ens:
            p.max_steps = args.batch_steps
            pids.append(b.add(p, ic))
        sample = batch_sample(ens)
        init = {i: b.fetch_dense(pids[i]) for i in sample}
        if dist is not None:
            dist.barrier()
        with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
            ms = b.bench(args.batch_steps)
        done, nstep, _ = b.poll()
        ok = bool(done[:len(ens)].all() and (nstep[:len(ens)] == args.batch_steps).all())
        out.setdefault("_oracle_sample", {})[prec] = [
            {"problem": ens[i][0], "init": init[i], "final": b.fetch_dense(pids[i]), "nstep": int(nstep[pids[i]]),
             "t": float(b.status(pids[i])["t"]), "label": "ensemble[%d] side %d" % (i, ens[i][0].n[0])}
            for i in sample]
        b.close()
        ms = max_over_ranks([ms], dist)[0]
        out[prec] = {"value": out["cells"] / (ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": ms,
                     "tile": best, "all_problems_finished": ok, "clocks": clk.summary()}
    out["fp32_bulk_over_fp64"] = out["fp64"]["ms_per_step"] / out["fp32_bulk"]["ms_per_step"]
    return out


def batch_sample(ens, per_side=((16, 2), (32, 2), (48, 1))):
    """Indices of the ensemble problems whose results are checked against
    the oracle: the first few of the smallest sides (the oracle must solve
    each one for all its steps on the host)."""
    out = []
    for side, k in per_side:
        out += [i for i, (p, _) in enumerate(ens) if p.n[0] == side][:k]
    return out


def serve_sample(reqs, k2=2, k3=2):
    """Request ids checked against the oracle: the k2 2D and k3 3D requests of
    least work (cells x target steps)."""
    work = lambda r: r.solved_cells * r.target_steps  # noqa: E731
    two = sorted((r for r in reqs if int(r.prob.ndim) == 2), key=work)[:k2]
    three = sorted((r for r in reqs if int(r.prob.ndim) == 3), key=work)[:k3]
    return [r.rid for r in two + three]


def bench_serve(args, rank, world, dist):
    """A serving session per GPU: make_requests(args.serve_requests) arriving
    as a Poisson stream at args.serve_rate per second (own seed per rank),
    continuous batching over a 16 GiB pool.  Reports time-to-solution
    percentiles (rank 0's stream) and whole-job cell-updates/s, then the same
    requests all due at once ("burst": the server's capacity)."""
    from ramses2_b200.ranks import max_over_ranks, sum_over_ranks
    from ramses2_b200.serve import HydroServer, make_requests

    out = {"workload": "%d requests per GPU at %.1f/s: 2D 64^2-1024^2 Sedov/interfaces and 3D 32^3-192^3 "
                       "Sedov (E in [0.1,10]), 20-400 steps each, HLLC, moncen" % (args.serve_requests,
                                                                                  args.serve_rate)}
    for prec in ("fp32_bulk", "fp64"):
        srv = HydroServer(prec, pool_bytes=16 << 30, chunk=4, keep_results=False)
        srv.run(make_requests(4, rate_hz=1e6, seed=1, steps=(4, 8)), realtime=False)  # warm-up
        reqs = make_requests(args.serve_requests, rate_hz=args.serve_rate, seed=20261203 + rank)
        keep = serve_sample(reqs)
        srv.keep_results = set(keep)
        if dist is not None:
            dist.barrier()
        st = srv.run(reqs, realtime=True)
        srv.keep_results = False
        samples = []
        for r in reqs:
            if r.rid in keep and r.result is not None:
                pid = srv.batch.add(r.prob, r.ic)  # the request's initial state, as the device builds it
                init = srv.batch.fetch_dense(pid)
                srv.batch.remove(pid)
                from ramses2_b200.batch import octs_to_dense

                samples.append({"problem": r.prob, "init": init, "final": octs_to_dense(r.result, tuple(r.prob.n)),
                                "nstep": r.nsteps, "t": r.t,
                                "label": "request %d %s %s" % (r.rid, r.kind, "x".join(str(v) for v in r.prob.n))})
        out.setdefault("_oracle_sample", {})[prec] = samples
        # capacity: the same requests all due at once (closed loop)
        burst = make_requests(args.serve_requests, rate_hz=args.serve_rate, seed=20261203 + rank)
        if dist is not None:
            dist.barrier()
        sb = srv.run(burst, realtime=False)
        if dist is not None:
            sb["cell_updates"] = sum_over_ranks([sb["cell_updates"]], dist)[0]
            sb["makespan_s"] = max_over_ranks([sb["makespan_s"]], dist)[0]
            sb["cell_updates_per_s"] = sb["cell_updates"] / sb["makespan_s"]
        st["burst"] = {k: sb[k] for k in ("makespan_s", "cell_updates_per_s", "latency_p50_s", "latency_p99_s")}
        # latency against offered load: the sweep's request set (its problems
        # do not depend on the rate) served as a burst gives this GPU's
        # capacity in requests/s; Poisson streams of it then arrive at
        # fractions of that capacity
        if args.serve_sweep_requests > 0:
            probe = make_requests(args.serve_sweep_requests, rate_hz=1.0, seed=777 + rank)
            pb = srv.run(probe, realtime=False)
            mean_work = pb["cell_updates"] / max(1, pb["served"])
            cap_rps = pb["served"] / pb["makespan_s"]
            sweep = []
            for frac in (0.25, 0.5, 0.8, 0.95):
                reqs = make_requests(args.serve_sweep_requests, rate_hz=frac * cap_rps, seed=777 + rank)
                if dist is not None:
                    dist.barrier()
                sp = srv.run(reqs, realtime=True)
                sweep.append({"offered_load_of_burst": frac, "rate_hz": frac * cap_rps,
                              "latency_p50_s": sp["latency_p50_s"], "latency_p99_s": sp["latency_p99_s"],
                              "cell_updates_per_s": sp["cell_updates_per_s"], "makespan_s": sp["makespan_s"],
                              "requests": sp["requests"]})
            st["load_sweep"] = {"capacity_requests_per_s": cap_rps, "mean_cell_updates_per_request": mean_work,
                                "burst_cell_updates_per_s": pb["cell_updates_per_s"], "points": sweep}
        srv.close()
        if dist is not None:
            st["cell_updates"] = sum_over_ranks([st["cell_updates"]], dist)[0]
            st["makespan_s"] = max_over_ranks([st["makespan_s"]], dist)[0]
            st["cell_updates_per_s"] = st["cell_updates"] / st["makespan_s"]
        out[prec] = st
    return out


def _timed(L, fn):
    """Device time of fn() (CUDA events on the library stream), ms."""
    import ctypes as C

    from ramses2_b200._lib import check

    ms = C.c_float()
    check(L.rh_timer_start(), "rh_timer_start")
    fn()
    check(L.rh_timer_stop(C.byref(ms)), "rh_timer_stop")
    return ms.value


def bench_snapshot(L, m, prec, peak, reps=5):
    """Restart / snapshot file images (include/ramses_hydro_io.h) of the
    resident 256^3 state: device time of rh_file_image_device (CUDA events on
    the library's stream) and wall time of rh_file_image into pinned host
    memory.  Algorithmic bytes: state read once + image written once."""
    import ctypes as C

    from ramses2_b200._lib import check

    noct = int(m.noct[LEVEL])
    state_b = {"fp64": 320, "fp32_bulk": 192}[prec]
    out = {}
    for kind, name, rec in ((2, "hydro_backup", 320), (3, "hydro_output", 160)):
        ptr, n = C.c_void_p(), C.c_longlong()
        check(L.rh_file_image_device(kind, 1.4, C.byref(ptr), C.byref(n)), "rh_file_image_device")  # warm-up
        ms = []
        for _ in range(reps):
            check(L.rh_timer_start(), "rh_timer_start")
            check(L.rh_file_image_device(kind, 1.4, C.byref(ptr), C.byref(n)), "rh_file_image_device")
            t = C.c_float()
            check(L.rh_timer_stop(C.byref(t)), "rh_timer_stop")
            ms.append(t.value)
        dev_ms = float(np.median(ms))
        gbs = noct * (state_b + rec) / (dev_ms * 1e-3) / 1e9
        try:
            import torch

            host = torch.empty(int(n.value), dtype=torch.uint8, pin_memory=True)
            hptr = host.data_ptr()
        except Exception:
            host = np.empty(int(n.value), np.uint8)
            hptr = host.ctypes.data
        got = C.c_longlong()
        check(L.rh_file_image(kind, 1.4, C.c_void_p(hptr), n.value, C.byref(got)), "rh_file_image")
        t0 = time.perf_counter()
        for _ in range(reps):
            check(L.rh_file_image(kind, 1.4, C.c_void_p(hptr), n.value, C.byref(got)), "rh_file_image")
        host_ms = (time.perf_counter() - t0) / reps * 1e3
        out[name] = {"bytes": int(n.value), "device_ms": dev_ms, "device_GBps": gbs, "frac_of_hbm": gbs / peak,
                     "to_pinned_host_ms": host_ms, "to_host_GBps": n.value / (host_ms * 1e-3) / 1e9}
    return out


def leaf_rel_l1(m, a, b):
    """Relative L1 (rho, mx, my, mz, E) over the leaf cells of every level."""
    num = np.zeros(5)
    den = np.zeros(5)
    for lev in range(m.levelmin, m.levelmax + 1):
        if not m.noct[lev]:
            continue
        sl = m.level_slice(lev)
        leaf = m.leaf_mask(lev)[:, None, :]
        num += (np.abs(a[sl] - b[sl]) * leaf).sum(axis=(0, 2))
        den += (np.abs(b[sl]) * leaf).sum(axis=(0, 2))
    return dict(zip(["rho", "mx", "my", "mz", "E"], (num / np.where(den > 0, den, 1.0)).tolist()))


def bench_amr(args, rank, world, dist, device):
    """AMR Sedov on levels 7-10 refined by hydro_refine's 0.1
    density/pressure gradient criterion on a developed Sedov-like blast
    (2-6 M leaf cells), HLLC, moncen, Courant 0.8, args.amr_steps coarse
    steps with nsubcycle=1 (courant_fine of every level, then every level's
    Godunov step, one rh_coarse_step call), FP64 and FP32-bulk, each timed
    step by step.  Along the FP64 run the state before every
    args.amr_check_every-th step is kept (the oracle takes one coarse step
    from each later, on the host); the FP32-bulk run is repeated along the
    FP64 dt sequence and compared with those states (cumulative error)."""
    from ramses2_b200._abi import HydroParams
    from ramses2_b200._lib import lib
    from ramses2_b200.hydro import GodunovGPU, amr_coarse_step
    from ramses2_b200.mesh import sedov_amr_mesh
    from ramses2_b200.ranks import max_over_ranks

    m, g = sedov_amr_mesh(7, 10, radius=0.08)
    P = HydroParams.make(gamma=g, courant_factor=0.8, slope_type=2, riemann="hllc", interpol_var=0,
                         interpol_type=1)
    L = lib()
    u0 = m.uold.copy()
    leaf = m.ncells_leaf()
    allcells = int(m.noct_total) * 8
    out = {"workload": "AMR Sedov, levels 7-10, hydro_refine err_grad_d = err_grad_p = 0.1 on a developed blast",
           "leaf_cells": leaf, "cells_all_levels": allcells,
           "octs_per_level": {str(l): int(m.noct[l]) for l in range(7, 11)}, "steps": args.amr_steps,
           "check_every": args.amr_check_every}
    checks = set(range(0, args.amr_steps, max(1, args.amr_check_every)))
    keep_states = rank == 0 and not args.no_cpu
    # coarse-fine table build (rh_set_mesh wall time, FP64 state upload
    # included): best of three after one untimed warm-up build
    build_s = {"host": [], "device": []}
    for builder in ("device",) + ("host", "device") * 3:
        t0 = time.perf_counter()
        gpu = GodunovGPU(m, P, precision="fp64", device=device, table_builder=builder)
        build_s[builder].append(time.perf_counter() - t0)
        gpu.close()
    out["set_mesh_s"] = {k: min(v[-3:]) for k, v in build_s.items()}
    fp64_traj = None
    for prec in ("fp64", "fp32_bulk"):
        m.uold[:] = u0
        gpu = GodunovGPU(m, P, precision=prec, device=device)
        for _ in range(2):
            gpu.coarse_step()
        # the same coarse step driven call by call from Python (a round trip per leaf call)
        gpu.push_uold(u0)
        per_calls = [_timed(L, lambda: amr_coarse_step(gpu, m)) for _ in range(3)]
        gpu.push_uold(u0)
        per, dts, states = [], [], {}
        for s in range(args.amr_steps):
            if prec == "fp64" and s in checks:
                states[s] = gpu.fetch_uold()  # untimed: the state before step s+1
            res = {}
            per.append(_timed(L, lambda: res.__setitem__("dt", gpu.coarse_step())))
            dts.append(res["dt"])
        if prec == "fp64":
            fp64_traj = (dts, states)
        else:
            # cumulative accuracy along the FP64 trajectory: same dt sequence, untimed
            gpu.push_uold(u0)
            errs = []
            for s, dt in enumerate(fp64_traj[0]):
                if s in checks and s > 0:
                    e = leaf_rel_l1(m, gpu.fetch_uold(), fp64_traj[1][s])
                    e["after_steps"] = s
                    errs.append(e)
                gpu.coarse_step(dt)
            out["fp32_bulk_vs_fp64_trajectory_rel_l1"] = errs
        gpu.close()
        ms = max_over_ranks([float(np.mean(per))], dist)[0]
        out[prec] = {"value": world * leaf / (ms * 1e-3), "unit": "leaf cell-updates/s", "ms_per_coarse_step": ms,
                     "all_level_cell_updates_per_s": world * allcells / (ms * 1e-3),
                     "ms_each_step": [round(v, 3) for v in per],
                     "ms_per_coarse_step_python_leaf_calls": float(np.mean(per_calls))}
    out["fp32_bulk_over_fp64"] = out["fp64"]["ms_per_coarse_step"] / out["fp32_bulk"]["ms_per_coarse_step"]
    # the coarse step's corrections to father cells are summed in a fixed
    # order: two runs of 10 coarse steps from the same state, compared bit for bit
    out["repeat_bitwise"] = {}
    for prec in ("fp64", "fp32_bulk"):
        finals = []
        for _ in range(2):
            m.uold[:] = u0
            gpu = GodunovGPU(m, P, precision=prec, device=device)
            for _ in range(10):
                gpu.coarse_step()
            finals.append(gpu.fetch_uold())
            gpu.close()
        out["repeat_bitwise"][prec] = bool(np.array_equal(finals[0], finals[1]))
    m.uold[:] = u0
    out["_mesh"] = (m, P, u0, fp64_traj if keep_states else None)
    return out


def amr_oracle_checks(m, P, traj, oracle, nthreads, device):
    """Per-step accuracy along the FP64 AMR run: from each kept state S_k (the
    state before step k+1) the oracle takes one coarse step with the dt the
    GPU took there, and so do the FP64 and FP32-bulk GPU paths (a fresh
    context each, pushed S_k); leaf-cell relative L1 of each against the
    oracle, and the oracle's own courant_fine dt against the GPU's."""
    from ramses2_b200.hydro import GodunovGPU, amr_coarse_step

    if traj is None:
        return []
    dts, states = traj
    lev = [l for l in range(m.levelmin, m.levelmax + 1) if m.noct[l]]
    out = []
    for k in sorted(states):
        s_k = states[k]
        m.uold[:] = s_k
        o = oracle.OracleHydro(m, P, nthreads=nthreads)
        dt_or = min(min(m.dx(l) / P.smallc, o.courant_fine(l)[4]) for l in lev)
        amr_coarse_step(o, m, dts[k])
        ref = m.uold.copy()
        c = {"step": k + 1, "dt_gpu": dts[k], "dt_oracle_rel_diff": abs(dt_or / dts[k] - 1.0)}
        for prec in ("fp64", "fp32_bulk"):
            m.uold[:] = s_k
            gpu = GodunovGPU(m, P, precision=prec, device=device)
            gpu.coarse_step(dts[k])
            c[prec] = leaf_rel_l1(m, gpu.fetch_uold(), ref)
            gpu.close()
        out.append(c)
    m.uold[:] = states[min(states)]
    return out


def sample_vs_oracle(s, oracle, nthreads):
    """One batch problem or served request solved by the oracle from the
    state the device started it from, to the same stopping rule: relative L1
    per conserved variable of the device's final state, and both step counts."""
    from ramses2_b200._abi import HydroParams

    p = s["problem"]
    P = HydroParams.make(gamma=p.gamma, smallr=p.smallr, smallc=p.smallc, courant_factor=p.courant_factor,
                         slope_type=2, riemann="hllc")
    ref, t, ns = oracle.solve_box(s["init"], p.dx, P, bc=[int(v) for v in p.bound_type], ndim=int(p.ndim),
                                  t_end=p.t_end, max_steps=p.max_steps, nthreads=nthreads)
    num = np.abs(s["final"] - ref).sum(axis=(1, 2, 3))
    den = np.abs(ref).sum(axis=(1, 2, 3))
    l1 = num / np.where(den > 0, den, 1.0)
    return {"problem": s["label"], "rel_l1": dict(zip(["rho", "mx", "my", "mz", "E"], l1.tolist())),
            "steps": s["nstep"], "oracle_steps": ns, "t_rel_diff": abs(s["t"] / t - 1.0) if t else None}


PUBLISHED_512 = {"fp64": 4456e6, "fp32_bulk": 10093e6}  # reference B200, hydro double/single NSUBGRID=4


def bench_sedov512(args, rank, world, dist, device, tuned):
    """The reference's own published configuration: periodic Sedov3D 512^3,
    HLLC, moncen, whole hydro step (CFL, set_unew, Godunov, set_uold), with
    the tile tuned on 256^3 checked against a few others on this level
    (kernel-only, fastest kept: the pencil count per column, hence the last
    wave, differs at 512^3).  Reported next to the reference's published
    B200 figures for that setup (hydro double / single, NSUBGRID=4; the
    reference's "single" is all-FP32 storage, FP32-bulk keeps E in FP64)."""
    from ramses2_b200._abi import HydroParams
    from ramses2_b200._lib import lib
    from ramses2_b200.hydro import GodunovGPU
    from ramses2_b200.mesh import sedov3d, uniform_mesh
    from ramses2_b200.ranks import max_over_ranks

    m = uniform_mesh(9, nsubgrid=1, bc="periodic")
    sedov3d(m, gamma=1.4, rho0=1.0, p0=1e-5, energy=1.0, radius_cells=2.0)
    P = HydroParams.make(gamma=1.4, courant_factor=0.8, slope_type=2, riemann="hllc")
    L = lib()
    ncell = int(m.noct[9]) * 8
    out = {"workload": "Sedov3D 512^3 periodic, whole hydro step", "cells": ncell, "steps": args.sedov512_steps}
    others = {"fp32_bulk": [(7, 7, 2, 40), (7, 7, 2, 32), (15, 7, 1, 24), (15, 7, 1, 32)],
              "fp64": [(8, 8, 1, 32), (8, 8, 1, 40), (8, 4, 2, 32)]}
    for prec in ("fp64", "fp32_bulk"):
        gpu = GodunovGPU(m, P, precision=prec, device=device)
        t = tuned[prec]
        dt0 = gpu.coarse_step()
        best = None
        for c in [(t["txo"], t["tyo"], t["minb"], t["lz"])] + others[prec]:
            try:
                gpu.set_tile(c[0], c[1], c[3], c[2])
            except Exception:
                continue  # a shape not compiled for this precision
            gpu.bench_godunov(9, 1, dt0)
            kms = min(gpu.bench_godunov(9, 2, dt0) for _ in range(2))
            if best is None or kms < best[0]:
                best = (kms, c)
        c = best[1]
        gpu.set_tile(c[0], c[1], c[3], c[2])
        for _ in range(3):
            gpu.coarse_step()
        ms = _timed(L, lambda: [gpu.coarse_step() for _ in range(args.sedov512_steps)]) / args.sedov512_steps
        gpu.close()
        ms = max_over_ranks([ms], dist)[0]
        v = world * ncell / (ms * 1e-3)
        out[prec] = {"value": v, "unit": "cell-updates/s", "ms_per_step": ms,
                     "tile": {"txo": c[0], "tyo": c[1], "minb": c[2], "lz": c[3]},
                     "reference_published_b200": PUBLISHED_512[prec],
                     "over_reference_published": v / world / PUBLISHED_512[prec]}
    return out


def bench_turbulence(args, rank, world, dist, device):
    """Decaying supersonic turbulence on 256^3 (gamma 1.001, rms
    Mach 5, lognormal density, minmod, HLLC, periodic), tiles autotuned on
    this state, args.turb_steps FP32-bulk and FP64 steps; FP32-bulk relative
    L1 against FP64 after them."""
    from ramses2_b200._abi import HydroParams
    from ramses2_b200._lib import lib
    from ramses2_b200.hydro import GodunovGPU
    from ramses2_b200.mesh import turbulence3d, uniform_mesh
    from ramses2_b200.ranks import max_over_ranks

    m = uniform_mesh(LEVEL, nsubgrid=1, bc="periodic")
    turbulence3d(m, gamma=1.001, mach=5.0)
    P = HydroParams.make(gamma=1.001, courant_factor=0.8, slope_type=1, riemann="hllc")
    L = lib()
    u0 = m.uold.copy()
    ncell = int(m.noct[LEVEL]) * 8
    out = {"workload": "decaying turbulence 256^3, gamma 1.001, rms Mach 5, minmod, HLLC",
           "cells": ncell, "steps": args.turb_steps}
    final = {}
    from ramses2_b200 import autotune

    for prec in ("fp64", "fp32_bulk"):
        m.uold[:] = u0
        gpu = GodunovGPU(m, P, precision=prec, device=device)
        dt0 = gpu.coarse_step()
        best, _ = autotune.tune(gpu, LEVEL, dt0)  # tiles tuned on this workload itself
        out.setdefault("tile", {})[prec] = best
        gpu.push_uold(u0)
        ms = _timed(L, lambda: [gpu.coarse_step() for _ in range(args.turb_steps)]) / args.turb_steps
        final[prec] = gpu.fetch_uold()
        gpu.close()
        ms = max_over_ranks([ms], dist)[0]
        out[prec] = {"value": world * ncell / (ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": ms}
    out["fp32_bulk_over_fp64"] = out["fp64"]["ms_per_step"] / out["fp32_bulk"]["ms_per_step"]
    names = ["rho", "mx", "my", "mz", "E"]
    out["fp32_bulk_vs_fp64_rel_l1_after_steps"] = dict(zip(names, rel_l1(final["fp32_bulk"], final["fp64"])))
    out["_state"] = (m, P, final["fp64"])
    return out


def run_ours(args):
    import ctypes as C

    from ramses2_b200 import autotune
    from ramses2_b200._lib import check, lib
    from ramses2_b200.hydro import GodunovGPU

    rank, world, local = env_rank()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_

        torch.cuda.set_device(local)
        dist_.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = dist_
    device = local
    m, P = make_problem()
    ncell = int(m.noct[LEVEL]) * 8
    u0 = m.uold.copy()
    L = lib()
    results = {}
    kernel_ms = {}
    snapshot = {}
    tuned = {}
    for prec in ("fp64", "fp32_bulk"):
        m.uold[:] = u0
        gpu = GodunovGPU(m, P, precision=prec, device=device)
        dt0, _ = gpu.step_uniform()
        best, _ = autotune.tune(gpu, LEVEL, dt0)
        tuned[prec] = best
        m.uold[:] = u0
        gpu.push_uold()
        if dist is not None:
            dist.barrier()
        with ClockSampler(device) as clk:
            ms, per = time_steps(gpu, L, args.steps, args.warmup)
        results[prec] = {"ms_per_step": ms, "clocks": clk.summary(), "per_step": per}
        # dominant kernel, device time per launch
        m.uold[:] = u0
        gpu.push_uold()
        dt, _ = gpu.step_uniform()
        kernel_ms[prec] = kernel_time(gpu, args.steps, dt)
        snapshot[prec] = bench_snapshot(L, m, prec, measured_peaks()[0])
        # end to end through the ABI with host buffers (pinned)
        try:
            import torch

            host = torch.empty(m.uold.size, dtype=torch.float64, pin_memory=True).numpy().reshape(m.uold.shape)
        except Exception:
            host = np.empty_like(m.uold)
        if prec == "fp64":
            # rh_coarse_step_host of the FP64 mode (no record conversion), for comparison
            host[:] = u0
            _, nxt = gpu.coarse_step_host(host)
            for _ in range(args.warmup - 1):
                _, nxt = gpu.coarse_step_host(host, dt=nxt)
            e2e64 = C.c_float()
            check(L.rh_timer_start(), "rh_timer_start")
            for _ in range(args.steps):
                _, nxt = gpu.coarse_step_host(host, dt=nxt)
            check(L.rh_timer_stop(C.byref(e2e64)), "rh_timer_stop")
            results["e2e_fp64_ms"] = e2e64.value / args.steps
        if prec == "fp32_bulk":
            host[:] = u0
            from ramses2_b200._abi import dptr

            # the three separate calls (upload, step, read back), one after the other
            gpu.sync()
            check(L.rh_timer_start(), "rh_timer_start")
            for _ in range(args.steps):
                check(L.rh_set_grid_device(dptr(host), m.ngridmax, 5, 8), "rh_set_grid_device")
                gpu.coarse_step()
                check(L.rh_transfer_grid_host(dptr(host), m.ngridmax, 5, 8), "rh_transfer_grid_host")
            e2e_ms = C.c_float()
            check(L.rh_timer_stop(C.byref(e2e_ms)), "rh_timer_stop")
            results["e2e_serial_ms"] = e2e_ms.value / args.steps
            # rh_coarse_step_host: the copies overlapped with the pencils; each
            # call takes the dt_next its predecessor returned
            host[:] = u0
            _, nxt = gpu.coarse_step_host(host)
            for _ in range(args.warmup - 1):
                _, nxt = gpu.coarse_step_host(host, dt=nxt)
            check(L.rh_timer_start(), "rh_timer_start")
            t0 = time.perf_counter()
            for _ in range(args.steps):
                _, nxt = gpu.coarse_step_host(host, dt=nxt)
            wall = time.perf_counter() - t0
            check(L.rh_timer_stop(C.byref(e2e_ms)), "rh_timer_stop")
            results["e2e_ms"] = e2e_ms.value / args.steps
            results["e2e_wall_ms"] = wall * 1e3 / args.steps
            results["e2e_bytes"] = int(m.uold.nbytes)
        gpu.close()
    s512 = bench_sedov512(args, rank, world, dist, device, tuned) if args.sedov512_steps > 0 else None
    amr = bench_amr(args, rank, world, dist, device) if args.amr_steps > 0 else None
    turb = bench_turbulence(args, rank, world, dist, device) if args.turb_steps > 0 else None
    batch = bench_batch(args, rank, world, dist) if args.batch_problems > 0 else None
    serve = bench_serve(args, rank, world, dist) if args.serve_requests > 0 else None
    # max over ranks
    if dist is not None:
        from ramses2_b200.ranks import max_over_ranks

        (results["fp32_bulk"]["ms_per_step"], results["fp64"]["ms_per_step"], results["e2e_ms"],
         results["e2e_serial_ms"], results["e2e_fp64_ms"]) = max_over_ranks(
            [results["fp32_bulk"]["ms_per_step"], results["fp64"]["ms_per_step"], results["e2e_ms"],
             results["e2e_serial_ms"], results["e2e_fp64_ms"]], dist)
    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return
    # Accuracy on a developed blast (FP32-bulk vs FP64) and the CPU baseline:
    # both GPU paths run ACC_STEPS steps from the initial state (cumulative
    # error), then one step from the FP64 state is taken by the CPU oracle, the
    # FP32-bulk path and the FP64 path (per-step error).
    cpu = None
    acc = None
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        nthreads = os.cpu_count() or 1
        states = {}
        for prec in ("fp64", "fp32_bulk"):
            m.uold[:] = u0
            gpu = GodunovGPU(m, P, precision=prec, device=device)
            for _ in range(args.acc_steps):
                gpu.step_uniform()
            states[prec] = gpu.fetch_uold()
            gpu.close()
        s_dev = states["fp64"]
        m.uold[:] = s_dev
        o = oracle.OracleHydro(m, P, nthreads=nthreads)
        t0 = time.perf_counter()
        o.step_uniform()
        cpu_s = time.perf_counter() - t0
        ref = m.uold.copy()
        one = {}
        for prec in ("fp64", "fp32_bulk"):
            m.uold[:] = s_dev
            gpu = GodunovGPU(m, P, precision=prec, device=device)
            gpu.step_uniform()
            one[prec] = gpu.fetch_uold()
            gpu.close()
        names = ["rho", "mx", "my", "mz", "E"]
        cpu = {"value": ncell / cpu_s, "unit": "cell-updates/s", "cores": nthreads, "kind": "port",
               "sample": "one full 256^3 Sedov step (courant_fine + godunov_fine, OpenMP over oct blocks "
                         "on %d threads) of the CPU restatement of the reference path, %.2f s" % (nthreads, cpu_s)}
        # Sedov 64^3 (outflow, 100-step size) on one thread and on all of them, a few steps each
        from ramses2_b200.mesh import sedov3d, uniform_mesh

        c0 = {}
        for nth in (1, nthreads):
            m0 = uniform_mesh(6, nsubgrid=1, bc="outflow")
            sedov3d(m0, gamma=1.4, rho0=1.0, p0=1e-5, energy=1.0, radius_cells=2.0)
            o0 = oracle.OracleHydro(m0, P, nthreads=nth)
            o0.step_uniform()
            t0 = time.perf_counter()
            for _ in range(3):
                o0.step_uniform()
            c0["threads_%d" % nth] = 3 * int(m0.noct[6]) * 8 / (time.perf_counter() - t0)
        cpu["sedov64_cell_updates_per_s"] = c0
        acc = {"state": "Sedov3D 256^3 after %d FP64 steps" % args.acc_steps,
               "per_step_fp32_bulk_vs_fp64_oracle_rel_l1": dict(zip(names, rel_l1(one["fp32_bulk"], ref))),
               "per_step_fp64_vs_fp64_oracle_rel_l1": dict(zip(names, rel_l1(one["fp64"], ref))),
               "cumulative_fp32_bulk_vs_fp64_rel_l1": dict(zip(names, rel_l1(states["fp32_bulk"], s_dev))),
               "cumulative_steps": args.acc_steps}
        acc["density_l1_le_1e-5"] = bool(acc["per_step_fp32_bulk_vs_fp64_oracle_rel_l1"]["rho"] <= 1e-5 and
                                         acc["cumulative_fp32_bulk_vs_fp64_rel_l1"]["rho"] <= 1e-5)
        # one step of each precision against the oracle on the AMR and turbulence states
        from ramses2_b200.hydro import amr_coarse_step

        if amr is not None:
            ma, Pa, ua, traj = amr.pop("_mesh")
            amr["per_step_vs_oracle"] = amr_oracle_checks(ma, Pa, traj, oracle, nthreads, device)
            amr["fp64_per_step_le_1e-12"] = bool(all(
                max(c["fp64"][k] for k in names) <= 1e-12 for c in amr["per_step_vs_oracle"]))
            amr["fp32_bulk_density_le_1e-5"] = bool(
                all(c["fp32_bulk"]["rho"] <= 1e-5 for c in amr["per_step_vs_oracle"]) and
                all(e["rho"] <= 1e-5 for e in amr["fp32_bulk_vs_fp64_trajectory_rel_l1"]))
        for leg in (batch, serve):
            if leg is not None and "_oracle_sample" in leg:
                leg["results_vs_oracle"] = {p: [sample_vs_oracle(s, oracle, nthreads) for s in v]
                                            for p, v in leg.pop("_oracle_sample").items()}
        if turb is not None:
            mt, Pt, st = turb.pop("_state")
            mt.uold[:] = st
            ot = oracle.OracleHydro(mt, Pt, nthreads=nthreads)
            dtt, _ = ot.step_uniform()
            reft = mt.uold.copy()
            turb["one_step_vs_oracle_rel_l1"] = {}
            for prec in ("fp64", "fp32_bulk"):
                mt.uold[:] = st
                gpu = GodunovGPU(mt, Pt, precision=prec, device=device)
                gpu.step_uniform(dtt)
                turb["one_step_vs_oracle_rel_l1"][prec] = dict(zip(names, rel_l1(gpu.fetch_uold(), reft)))
                gpu.close()
    if amr is not None:
        amr.pop("_mesh", None)
    if turb is not None:
        turb.pop("_state", None)
    for leg in (batch, serve):
        if leg is not None:
            leg.pop("_oracle_sample", None)
    peak, peak_kind = measured_peaks()
    prec = "fp32_bulk"
    ms = results[prec]["ms_per_step"]
    value = world * ncell / (ms * 1e-3)
    kms = kernel_ms[prec]
    achieved = ncell * B_ALG[prec] / (kms * 1e-3) / 1e9
    launches = args.steps * 2  # pencil kernel + partial reduction per step (rh_cmpdt hits the fused CFL)
    line = {
        "metric": "cell-updates/s Sedov3D 256^3 FP32-bulk vs FP64 at L1<=1e-5; p50/p99 solve latency",
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32+fp64(E,p,dt,sums)",
        "data": "synthetic",
        "config": bench_config(world, ncell),
        "fp64": {"value": world * ncell / (results["fp64"]["ms_per_step"] * 1e-3),
                 "ms_per_step": results["fp64"]["ms_per_step"],
                 "kernel_ms": kernel_ms["fp64"],
                 "roofline_frac": ncell * B_ALG["fp64"] / (kernel_ms["fp64"] * 1e-3) / 1e9 / peak,
                 "pipes_ncu": profile_pipes("fp64"),
                 "clocks": results["fp64"]["clocks"]},
        "fp32_bulk_over_fp64": results["fp64"]["ms_per_step"] / ms,
        "step_latency_ms": {"p50": float(np.percentile(results[prec]["per_step"], 50)),
                            "p99": float(np.percentile(results[prec]["per_step"], 99))},
        "tile": {k: v for k, v in tuned.items()},
        "e2e": {"value": world * ncell / (results["e2e_ms"] * 1e-3), "unit": "cell-updates/s",
                "h2d_bytes_per_step": results["e2e_bytes"], "d2h_bytes_per_step": results["e2e_bytes"],
                "call": "rh_coarse_step_host (FP64 uold in pinned host memory, in and out every step)",
                "ms_per_step": results["e2e_ms"], "wall_ms_per_step": results["e2e_wall_ms"],
                "serial_calls_cell_updates_per_s": world * ncell / (results["e2e_serial_ms"] * 1e-3),
                "serial_calls_ms_per_step": results["e2e_serial_ms"],
                "fp64": {"value": world * ncell / (results["e2e_fp64_ms"] * 1e-3),
                         "ms_per_step": results["e2e_fp64_ms"],
                         "call": "rh_coarse_step_host in FP64 mode (the host's FP64 uold copied as it is)"}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": profile_traffic(prec), "peak_kind": peak_kind,
                     "kernel": "godunov_pencil2_kernel (FP32-bulk)", "kernel_ms": kms,
                     "bytes_per_cell_update": B_ALG[prec], "pipes_ncu": profile_pipes(prec)},
        "cpu_baseline": cpu,
        "accuracy": acc,
        "solve_latency_s": None if serve is None else {
            p: {"p50": serve[p]["latency_p50_s"], "p99": serve[p]["latency_p99_s"]} for p in ("fp32_bulk", "fp64")},
        "sedov512_periodic": s512,
        "amr": amr,
        "turbulence": turb,
        "batch": batch,
        "serve": serve,
        "snapshot": snapshot,
        "gpu_launches": launches,
        "clocks": results[prec]["clocks"],
    }
    print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    rank, world, local = env_rank()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    m, P = make_problem()
    ncell = int(m.noct[LEVEL]) * 8
    nthreads = os.cpu_count() or 1
    o = oracle.OracleHydro(m, P, nthreads=nthreads)
    for _ in range(args.warmup):
        o.step_uniform()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step_uniform()
    el = (time.perf_counter() - t0) / args.steps
    value = ncell / el
    line = {
        "impl": "reference",
        "metric": "cell-updates/s Sedov3D 256^3 FP32-bulk vs FP64 at L1<=1e-5; p50/p99 solve latency",
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": el * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(world, ncell),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": nthreads, "kind": "port",
                         "sample": "full 256^3 Sedov steps of the CPU restatement of the reference path "
                                   "(Fortran reference not compilable in this image)"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline / accuracy leg")
    ap.add_argument("--acc-steps", type=int, default=100, help="steps before the accuracy comparison")
    ap.add_argument("--sedov512-steps", type=int, default=5, help="periodic Sedov 512^3 steps (0: skip)")
    ap.add_argument("--amr-steps", type=int, default=200, help="AMR Sedov coarse steps (0: skip)")
    ap.add_argument("--amr-check-every", type=int, default=10,
                    help="oracle check of the AMR run before every n-th coarse step")
    ap.add_argument("--turb-steps", type=int, default=100, help="turbulence 256^3 steps (0: skip)")
    ap.add_argument("--batch-problems", type=int, default=1024, help="batched ensemble size (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=50)
    ap.add_argument("--serve-requests", type=int, default=60, help="serving session length (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=20.0, help="request arrivals per second")
    ap.add_argument("--serve-sweep-requests", type=int, default=100,
                    help="requests per point of the latency-vs-offered-load sweep (0: skip)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
