"""Serving loop: hydro solve requests admitted by HBM footprint into one
device-resident batch (include/ramses_hydro_batch.h), with continuous batching.

A request is one uniform-grid problem solved to its t_end by the reference's
single-level step (hydro/umuscl.f90 unsplit + courant_fine dt).  Requests
arrive over time; the loop admits every waiting request whose state fits the
device pool (first fit, in arrival order), advances all admitted problems
together (one persistent kernel launch per step, replayed from a CUDA graph),
and retires a problem when it reaches t_end: its state is read back and its
pool space is freed for the queue.  A request whose footprint exceeds the
whole pool is rejected.  Latency is arrival -> result on the host (for a
burst run, where every request is due at once, start of the run -> result).
"""
import math
import os
import time
from dataclasses import dataclass, field

import numpy as np

from .batch import Batch, ic_blast, ic_split, problem, random_state

# device bytes per oct: uold + unew (FP64: 320-byte records; FP32-bulk: 192-byte records)
BYTES_PER_OCT = {"fp64": 2 * 320, "fp32_bulk": 2 * 192}


@dataclass
class Request:
    rid: int
    arrival: float             # seconds after the start of the run
    prob: object               # rh_batch_problem
    ic: object                 # rh_batch_ic
    kind: str = ""
    target_steps: int = 0
    submitted: float = math.nan  # entered the server's queue (its arrival; 0 for a burst)
    admitted: float = math.nan
    finished: float = math.nan
    nsteps: int = 0
    t: float = 0.0
    result: np.ndarray = field(default=None, repr=False)
    snapshot: str = None
    rejected: bool = False
    failed: int = 0            # state check bits when the solve was stopped (1 NaN/Inf, 2 rho<=0, 4 eint<=0)

    @property
    def cells(self):
        """Cells held on the device (a 2D problem: its two-cell-deep z slab)."""
        n = self.prob.n
        return int(n[0]) * int(n[1]) * int(n[2])

    @property
    def solved_cells(self):
        """Cells of the problem as posed: nx*ny for a 2D request, whose
        device slab holds each cell twice (identical z planes)."""
        n = self.prob.n
        return int(n[0]) * int(n[1]) * (int(n[2]) if int(self.prob.ndim) == 3 else 1)

    @property
    def latency(self):
        return self.finished - self.submitted


def initial_dt(states, gamma, dx, ndim, courant):
    """courant_fine dt of a state made of the given primitive states (no
    gravity): min over states of 2C dx / (ctot (1 + sqrt(1 + 2C 1e-4))),
    ctot = sum over ndim directions of |u_d| + c (godunov_utils.f90:228-333)."""
    k0 = 2.0 * courant * dx / (1.0 + math.sqrt(1.0 + 2.0 * courant * 1e-4))
    dt = math.inf
    for q in states:
        c = math.sqrt(gamma * q[4] / q[0])
        ctot = sum(abs(q[1 + d]) + c for d in range(ndim))
        dt = min(dt, k0 / ctot)
    return dt


def _sedov_p_in(n, ndim, dx, gamma, energy, radius_cells=2.0):
    """Pressure that puts ``energy`` (per unit depth in 2D) into the cells
    within radius_cells of the box centre, counted as the device IC counts them."""
    c = np.arange(n) + 0.5
    r2 = (c[:, None] - n / 2) ** 2 + (c[None, :] - n / 2) ** 2
    if ndim == 3:
        r2 = r2[..., None] + (c[None, None, :] - n / 2) ** 2
    nin = int((r2 * dx * dx <= (radius_cells * dx) ** 2 * (1 + 1e-12)).sum())
    return (gamma - 1.0) * energy / (nin * dx ** ndim), radius_cells * dx


def make_requests(n_requests, rate_hz, seed=20261203, frac_2d=0.5, steps=(20, 400), sides_2d=(64, 1024),
                  sides_3d=(32, 192), courant=0.8):
    """A Poisson stream of solve requests: 2D (one z oct layer) Sedov blasts
    and random-state interfaces with sides in sides_2d, 3D Sedov blasts with
    E uniform in [0.1, 10] and sides in sides_3d; t_end is the target number
    of steps (uniform in ``steps``) times the initial CFL dt, and max_steps
    caps a solve at the top of the range."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n_requests):
        t += rng.exponential(1.0 / rate_hz)
        g = float(rng.uniform(1.1, 1.67))
        nsteps = int(rng.integers(steps[0], steps[1] + 1))
        if rng.uniform() < frac_2d:
            s = int(round(math.exp(rng.uniform(math.log(sides_2d[0]), math.log(sides_2d[1]))) / 16)) * 16
            dx = 1.0 / s
            if rng.uniform() < 0.5:
                kind = "sedov2d"
                amb = [1.0, 0.0, 0.0, 0.0, 1e-5]
                p_in, rad = _sedov_p_in(s, 2, dx, g, float(rng.uniform(0.1, 10.0)))
                ic = ic_blast(amb, p_in, rad, (0.5, 0.5, dx))
                dt0 = initial_dt([amb[:4] + [p_in]], g, dx, 2, courant)
            else:
                kind = "interface2d"
                a, b = random_state(rng, g), random_state(rng, g)
                a[3] = b[3] = 0.0
                ic = ic_split(int(rng.integers(0, 2)), a, b)
                dt0 = initial_dt([a, b], g, dx, 2, courant)
            p = problem((s, s, 2), dx=dx, ndim=2, bc=["outflow"] * 4 + ["periodic"] * 2, gamma=g,
                        courant_factor=courant)
        else:
            s = int(rng.integers(sides_3d[0] // 16, sides_3d[1] // 16 + 1)) * 16
            dx = 1.0 / s
            kind = "sedov3d"
            amb = [1.0, 0.0, 0.0, 0.0, 1e-5]
            p_in, rad = _sedov_p_in(s, 3, dx, g, float(rng.uniform(0.1, 10.0)))
            ic = ic_blast(amb, p_in, rad, (0.5, 0.5, 0.5))
            dt0 = initial_dt([amb[:4] + [p_in]], g, dx, 3, courant)
            p = problem((s, s, s), dx=dx, ndim=3, bc="outflow", gamma=g, courant_factor=courant)
        p.t_end = nsteps * dt0
        p.max_steps = steps[1]
        out.append(Request(rid, t, p, ic, kind=kind, target_steps=nsteps))
    return out


class HydroServer:
    """Continuous-batching server over one device pool of ``pool_bytes``."""

    def __init__(self, precision="fp32_bulk", pool_bytes=8 << 30, slope_type=2, riemann="hllc", tile=None,
                 chunk=4, keep_results=True, snapshot_dir=None, state_check=False):
        """keep_results: True keeps every request's final state (Request.result),
        False none, or a set of request ids whose states are kept.
        state_check: check every stepped state on the device after each step
        (rh_batch_set_state_check); a request whose state goes bad (NaN/Inf,
        rho <= 0, internal energy <= 0) is stopped and reported failed
        (Request.failed holds the bits) instead of returning garbage.
        snapshot_dir: when set, every finished request leaves an output
        directory ``<snapshot_dir>/req<rid>/output_00001`` in the reference's
        layout (amr and hydro files written from the device image, info.txt,
        hydro_header.txt) before its pool range is freed."""
        self.snapshot_dir = snapshot_dir
        self.precision = precision
        self.pool_octs = max(1, int(pool_bytes) // BYTES_PER_OCT[precision])
        self.batch = Batch(precision, slope_type=slope_type, riemann=riemann, pool_octs=self.pool_octs, tile=tile)
        self.chunk = int(chunk)
        self.keep_results = keep_results
        if state_check:
            self.batch.set_state_check(True)

    def close(self):
        self.batch.close()

    def run(self, requests, realtime=True, log=None):
        """Serve ``requests`` (sorted by arrival).  With realtime=False arrivals
        are taken as already due (a closed-loop burst).  Returns summary stats."""
        b = self.batch
        pending = sorted(requests, key=lambda r: r.arrival)
        queue, active = [], {}
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        i = 0
        steps_total = 0
        updates = 0
        while i < len(pending) or queue or active:
            tnow = now()
            while i < len(pending) and (not realtime or pending[i].arrival <= tnow):
                pending[i].submitted = pending[i].arrival if realtime else 0.0
                queue.append(pending[i])
                i += 1
            # admission: first fit in arrival order
            waiting = []
            for r in queue:
                if b.footprint(r.prob) > self.pool_octs * BYTES_PER_OCT[self.precision]:
                    r.rejected = True
                    continue
                pid = b.add(r.prob, r.ic)
                if pid is None:
                    waiting.append(r)
                    continue
                r.admitted = now()
                active[pid] = r
            queue = waiting
            if not active:
                if i < len(pending) and realtime:
                    time.sleep(max(0.0, min(pending[i].arrival - now(), 0.05)))
                continue
            b.step(self.chunk)
            done, nstep, tt = b.poll()
            steps_total += self.chunk
            for pid in list(active):
                if done[pid]:
                    r = active.pop(pid)
                    r.nsteps = int(nstep[pid])
                    r.t = float(tt[pid])
                    if done[pid] == 2:
                        r.failed = b.check_mask(pid)
                    keep = self.keep_results
                    if keep is True or (keep and not isinstance(keep, bool) and r.rid in keep):
                        r.result = b.fetch(pid)
                    if self.snapshot_dir:
                        r.snapshot = b.write_output(pid, os.path.join(self.snapshot_dir, "req%05d" % r.rid), 1)
                    b.remove(pid)
                    r.finished = now()
                    if not r.failed:
                        updates += r.solved_cells * r.nsteps
                    if log:
                        log("req %d %s %s done: %d steps, latency %.3f s" % (r.rid, r.kind, tuple(r.prob.n),
                                                                             r.nsteps, r.latency))
        makespan = now()
        served = [r for r in requests if not r.rejected and not r.failed]
        lat = np.array([r.latency for r in served])
        return {
            "requests": len(requests),
            "served": len(served),
            "rejected": sum(r.rejected for r in requests),
            "failed": sum(bool(r.failed) for r in requests),
            "makespan_s": makespan,
            "cell_updates": int(updates),
            "cell_updates_per_s": updates / makespan if makespan > 0 else 0.0,
            "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else math.nan,
            "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else math.nan,
            "steps_min": int(min(r.nsteps for r in served)) if served else 0,
            "steps_max": int(max(r.nsteps for r in served)) if served else 0,
        }
