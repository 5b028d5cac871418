#!/usr/bin/env python
"""Benchmark of the lcbinint B200 magnification path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload fs_batch|ps_batch|light_curve|adjoint|orbital]

Default workload (fs_batch): the uneven finite-source batch -- 4,096 light-curve
points from 64 random binary-lens models (s log-U[0.3,3], q log-U[1e-5,1], rho
log-U[1e-4,1e-2], u0 U[-0.2,0.2], alpha U[0,2pi], linear limb darkening
U[0,0.8]), 64 epochs per model spread over the caustic-crossing window,
Cartesian or polar grid per point (p = 0.5) and nbin log-U{20..200}, every
point integrated by inverse ray (lcbinint.binary_inverse_ray semantics), all
points in one launch sequence, FP64.  One step = the whole batch.

One JSON line on rank 0: value = magnifications/s with inputs resident on the
GPU; e2e = the same through the host-pointer C ABI (host->device copies and
result readback inside the timed region); roofline of the dominant kernel
against the device-measured FP64 FMA peak; cpu_baseline = the reference
compiled from source (oracle/_ref), one process per host core, on a bounded
sample of the same points.  Under torchrun the ranks' batches form one job
split over the GPUs by estimated cost (independent points: weak scaling), and
the only collective is the all-gather of the results.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "finite-source mags/s & rays/s on 1 B200 at 1e-4 rel err; fwd+grad/fwd ratio"
F_RAY = 32.0      # algorithmic flop per lens-map evaluation of one cell
# DRAM traffic measured with ncu (small single-kernel captures): the early
# Cartesian scan of the batch's largest point read 4.22 MB and wrote nothing
# for its 6.35e6 counted cells; the point-source kernel moved 32.17 MB per
# 1e6 positions.  The scans generate their lattice on the fly, so their
# traffic is a few bytes per thousand flop: HBM is not their bound.
RAY_DRAM_BYTES_PER_CELL = 4.222464e6 / 6.349603e6
PS_DRAM_BYTES = 32.158976e6 + 7.68e3
F_PS = 3500.0     # algorithmic FP64 flop per point-source solve

# --------------------------------------------------------------------------- workloads


def _critical_caustic_points(s, q_core, n_phase=256):
    """Caustic points (centre-of-mass frame) from the critical-curve quartic, numpy only."""
    qi = abs(q_core)
    q = qi if qi < 1.0 else 1.0 / qi
    a = -s if qi < 1.0 else s
    m1 = 1.0 / (1.0 + q)
    m2 = q * m1
    pts = []
    for phi in np.linspace(0.0, 2 * np.pi, n_phase, endpoint=False):
        e = np.exp(1j * phi)
        coef = [-e, 2 * e * a, m1 + m2 - e * a * a, -2 * m2 * a, m2 * a * a]
        for z in np.roots(coef):
            zc = np.conj(z)
            y = z - m1 / (zc - a) - m2 / zc - a * m1
            pts.append((y.real, y.imag))
    return np.array(pts)


def fs_batch_workload(seed=1, n_models=64, per_model=64):
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(n_models):
        s = float(np.exp(rng.uniform(np.log(0.3), np.log(3.0))))
        q = float(np.exp(rng.uniform(np.log(1e-5), 0.0)))
        rho = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))))
        u0 = float(rng.uniform(-0.2, 0.2))
        alpha = float(rng.uniform(0.0, 2 * np.pi))
        gam = float(rng.uniform(0.0, 0.8))
        pts = _critical_caustic_points(s, 1.0 / q)
        ca, sa = math.cos(alpha), math.sin(alpha)
        # entry/exit of the trajectory through the caustic bounding box (+- 3 rho)
        lo, hi = pts.min(axis=0) - 3 * rho, pts.max(axis=0) + 3 * rho
        tau_lo, tau_hi = -np.inf, np.inf
        for d, p0, a0, b0 in ((ca, -u0 * sa, lo[0], hi[0]), (sa, u0 * ca, lo[1], hi[1])):
            if abs(d) < 1e-12:
                if not (a0 <= p0 <= b0):
                    tau_lo, tau_hi = np.inf, -np.inf
                continue
            t1, t2 = sorted(((a0 - p0) / d, (b0 - p0) / d))
            tau_lo, tau_hi = max(tau_lo, t1), min(tau_hi, t2)
        if not tau_lo < tau_hi:  # misses the box: span the box's projection on the trajectory
            proj = pts @ np.array([ca, sa])
            tau_lo, tau_hi = proj.min() - 3 * rho, proj.max() + 3 * rho
        for tau in np.linspace(tau_lo, tau_hi, per_model):
            x = tau * ca - u0 * sa
            y = tau * sa + u0 * ca
            polar = rng.random() < 0.5
            nbin = int(round(math.exp(rng.uniform(math.log(20), math.log(200)))))
            rows.append((s, 1.0 / q, x, y, rho, gam, 2 if polar else 1, nbin))
    return np.array(rows)


def fs_settings_for(rows):
    from lcbinint_b200.api import LimbDarkening, Options
    keys = {}
    settings = []
    idx = np.empty(len(rows), dtype=np.int32)
    for i, r in enumerate(rows):
        k = (float(r[5]), int(r[6]), int(r[7]))
        if k not in keys:
            keys[k] = len(settings)
            o = Options(inverse_ray_grid="polar" if k[1] == 2 else "cartesian", nbin=k[2])
            st = o.fs_settings(LimbDarkening.linear(k[0]))
            # lcbinint.binary_inverse_ray thresholds (python/lcbinint_pybind.cpp:3831-3833)
            st.kinji_threshold = 1e18
            st.hex_threshold = 0.0
            st.adaptive_hex_threshold = 0.0
            settings.append(st)
        idx[i] = keys[k]
    return settings, idx


def fs_batch_arrays(rows):
    """The C-ABI inputs of a forced inverse-ray batch: the settings list (one
    entry per distinct (Gamma, grid, nbin)), the distinct lens models and the
    FS_POINT_DTYPE records that index them."""
    from lcbinint_b200.api import FS_POINT_DTYPE, PS_EXACT, PS_ON_DEVICE
    settings, sidx = fs_settings_for(rows)
    mkeys = {}
    mlist = []
    midx = np.empty(len(rows), dtype=np.int32)
    for i, r in enumerate(rows):
        k = (r[0], r[1])
        if k not in mkeys:
            mkeys[k] = len(mlist)
            mlist.append((r[0], r[1], 1400, 0))
        midx[i] = mkeys[k]
    models = np.array(mlist, dtype=np.dtype([("s", "f8"), ("q", "f8"), ("bins", "i4"), ("r", "i4")]))
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["settings"] = sidx
    pts["model"] = midx
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    return settings, models, pts


def reference_inverse_ray(rows, n_procs):
    """The reference's binary_inverse_ray on every row, one process per core
    (its solver keeps static state, so never threads); returns the
    magnifications and methods in row order and the pool's wall time."""
    import multiprocessing as mp
    n_procs = max(1, min(n_procs, len(rows)))
    chunks = [(rows[k::n_procs],) for k in range(n_procs)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(n_procs) as pool:
        pool.map(_ref_worker, [(rows[:1],)] * n_procs)  # imports and library loads
        t0 = time.perf_counter()
        res = pool.map(_ref_worker, chunks)
        wall = time.perf_counter() - t0
    A = np.empty(len(rows))
    M = np.empty(len(rows), dtype=np.int32)
    for k, (_, out, meth) in enumerate(res):
        A[k::n_procs] = out
        M[k::n_procs] = meth
    return A, M, wall


def parity_summary(A, method, status, R, RM):
    """Agreement of the device's results with the reference's on the same
    points: Cartesian magnifications bit for bit, polar ones (same cells, an
    exact sum instead of a running one) to 1e-12 relative, methods equal."""
    cart = method == 2
    pol = method == 3
    same_bits = A.view(np.int64) == R.view(np.int64)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(same_bits, 0.0, np.abs(A / R - 1.0))
    rel = np.where(np.isfinite(rel), rel, np.inf)
    return {
        "vs": "the reference compiled from its sources (oracle/_ref), binary_inverse_ray on the same points",
        "points": int(A.size), "bit_exact": int(same_bits.sum()),
        "cartesian": {"points": int(cart.sum()), "bit_exact": int(same_bits[cart].sum())},
        "polar": {"points": int(pol.sum()), "bit_exact": int(same_bits[pol].sum()),
                  "max_rel": float(rel[pol].max()) if pol.any() else 0.0},
        "max_rel": float(rel.max()) if rel.size else 0.0,
        "methods_equal": int((method == RM).sum()), "status_ok": int((status == 0).sum()),
        "pass": bool(same_bits[cart].all() and (rel[pol] <= 1e-12).all() and (method == RM).all()
                     and (status == 0).all()),
    }


# --------------------------------------------------------------------------- helpers

class ClockSampler:
    """nvidia-smi SM clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(buf):
    buf.add_(1.0)  # writes 256 MB (> 126 MB L2) between timed steps


# --------------------------------------------------------------------------- CPU reference


def _ref_worker(args):
    """One process (the reference solver keeps static state): forced inverse ray on a chunk."""
    rows, = args
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import Reference, default_settings
    ref = Reference()
    t = time.perf_counter()
    out = []
    meth = []
    for r in rows:
        st = default_settings(source_bins=int(r[7]), finite_mode=int(r[6]), limb_darkening_c=float(r[5]))
        A, m = ref.inverse_ray(st, r[0], r[1], r[2], r[3], r[4])
        out.append(A[0])
        meth.append(int(m[0]))
    return time.perf_counter() - t, out, meth


def cpu_reference_rate(rows, n_procs, target_seconds=20.0, seed=7):
    """Points/s of the reference on a bounded random sample, one process per core.

    The sample is grown until the pool's wall time reaches about target_seconds."""
    import multiprocessing as mp
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(rows))
    ctx = mp.get_context("spawn")
    with ctx.Pool(n_procs) as pool:
        # warm the workers up (imports, library loads), then calibrate on four
        # points per process
        pool.map(_ref_worker, [([rows[i]],) for i in order[:n_procs]])
        take = order[n_procs:5 * n_procs]
        t0 = time.perf_counter()
        pool.map(_ref_worker, [([rows[i] for i in take[k::n_procs]],) for k in range(n_procs)])
        cal = time.perf_counter() - t0
        per_point = max(cal / 4.0, 1e-4)  # per point, per process, in parallel
        m = int(max(1, min(len(rows) // n_procs, target_seconds / per_point)))
        sample = order[: m * n_procs]
        chunks = [([rows[i] for i in sample[k::n_procs]],) for k in range(n_procs)]
        t0 = time.perf_counter()
        res = pool.map(_ref_worker, chunks)
        wall = time.perf_counter() - t0
    n = sum(len(c[0]) for c in chunks)
    return n / wall, n, wall


# --------------------------------------------------------------------------- configs 1 and 2


def ps_batch_workload(n=1_000_000, seed=0):
    """Point-source batch (1e6 points): y uniform in [-1.5, 1.5]^2, s log-U[0.3, 3],
    q log-U[1e-5, 1] in the core convention, per point."""
    rng = np.random.default_rng(seed)
    s = np.exp(rng.uniform(np.log(0.3), np.log(3.0), n))
    q = np.exp(rng.uniform(np.log(1e-5), 0.0, n))
    y1 = rng.uniform(-1.5, 1.5, n)
    y2 = rng.uniform(-1.5, 1.5, n)
    return s, q, y1, y2


LC_PARAMS = dict(t0=0.0, tE=1.0, u0=-0.01, alpha=0.5, s=0.95, q=1e-2, rho=5e-3)


def adjoint_workload(seed=2, n_models=256, n_epochs=500):
    """Adjoint workload (256 models x 500 epochs): models drawn as in fs_batch, epochs uniform over t0 +- 2 tE.
    Returns params (M, 8) = (t0, tE, u0, alpha, s, q, rho, Gamma) and times (M, K)."""
    rng = np.random.default_rng(seed)
    P = np.empty((n_models, 8))
    P[:, 0] = 0.0
    P[:, 1] = 20.0
    P[:, 2] = rng.uniform(-0.2, 0.2, n_models)
    P[:, 3] = rng.uniform(0.0, 2.0 * np.pi, n_models)
    P[:, 4] = np.exp(rng.uniform(np.log(0.3), np.log(3.0), n_models))
    P[:, 5] = np.exp(rng.uniform(np.log(1e-5), 0.0, n_models))
    P[:, 6] = np.exp(rng.uniform(np.log(1e-4), np.log(1e-2), n_models))
    P[:, 7] = rng.uniform(0.0, 0.8, n_models)
    T = P[:, :1] + P[:, 1:2] * rng.uniform(-2.0, 2.0, (n_models, n_epochs))
    return P, np.sort(T, axis=1)


def _ref_lc_worker(args):
    P, T = args
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import Reference, default_settings
    ref = Reference()
    t = time.perf_counter()
    for p, times in zip(P, T):
        st = default_settings(source_bins=50, finite_mode=4, limb_darkening_c=float(p[7]))
        ref.light_curve_static(st, times, t0=p[0], tE=p[1], u0=p[2], alpha=p[3], s=p[4], q=p[5], rho=p[6])
    return time.perf_counter() - t


def cpu_adjoint_rate(P, T, n_procs, n_models):
    """The reference's forward on a sample of models, one process per core; a
    central finite-difference gradient in 8 parameters costs 17 forwards."""
    import multiprocessing as mp
    idx = np.random.default_rng(11).permutation(len(P))[:n_models]
    chunks = [(P[idx[k::n_procs]], T[idx[k::n_procs]]) for k in range(n_procs)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(n_procs) as pool:
        t0 = time.perf_counter()
        pool.map(_ref_lc_worker, chunks)
        wall = time.perf_counter() - t0
    n = len(idx) * T.shape[1]
    return n / wall / 17.0, n, wall


def orbital_workload(seed=3, n_models=1024, n_epochs=2000, parallax=False):
    """Orbital workload, its lens-orbital-motion half: models drawn as in fs_batch
    (t0 U[-20, 20] d, tE U[10, 40] d), half of them on circular and half on
    Keplerian orbits with ds/dt / s and dalpha/dt U[-1, 1] per year and the
    line-of-sight term g3 U[0, 0.5] per year (Keplerian: lom_szs U[-0.5, 0.5],
    lom_ar U[1, 2]); 2000 epochs spanning 200 days; with parallax, piEN and
    piEE U[-0.5, 0.5].  Returns the parameter dictionaries, their
    orbital-motion modes, their limb-darkening coefficients and the epochs."""
    rng = np.random.default_rng(seed)
    dicts, modes, gams = [], [], []
    for m in range(n_models):
        p = dict(t0=float(rng.uniform(-20.0, 20.0)), tE=float(rng.uniform(10.0, 40.0)),
                 u0=float(rng.uniform(-0.2, 0.2)), alpha=float(rng.uniform(0.0, 2.0 * np.pi)),
                 s=float(np.exp(rng.uniform(np.log(0.3), np.log(3.0)))), q=float(np.exp(rng.uniform(np.log(1e-5), 0.0))),
                 rho=float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2)))),
                 g1=float(rng.uniform(-1.0, 1.0)) / 365.25, g2=float(rng.uniform(-1.0, 1.0)) / 365.25,
                 g3=float(rng.uniform(0.0, 0.5)) / 365.25)
        mode = 1 if m % 2 == 0 else 2
        if mode == 2:
            p.update(lom_szs=float(rng.uniform(-0.5, 0.5)), lom_ar=float(rng.uniform(1.0, 2.0)))
        dicts.append(p)
        modes.append(mode)
        gams.append(float(rng.uniform(0.0, 0.8)))
    if parallax:
        # Drawn from a stream of their own, so that the rest of the workload is
        # the same with and without parallax.
        prng = np.random.default_rng(seed + 1000)
        for p in dicts:
            p.update(piEN=float(prng.uniform(-0.5, 0.5)), piEE=float(prng.uniform(-0.5, 0.5)))
    return dicts, modes, gams, np.linspace(-100.0, 100.0, n_epochs)


# Sky position of the orbital workload's events (the Galactic bulge) for parallax.
ORBITAL_EVENT = dict(ra=268.5, dec=-29.0)


def orbital_ephemeris():
    """A synthetic Earth ephemeris for the parallax half of the orbital workload (the
    reference's table is not in its repository), named through
    LCBININT_EARTH_EPHEMERIS so that this process, the reference and the CPU
    workers read the same one."""
    import tempfile
    from lcbinint_b200.ephemeris import write_synthetic_ephemeris
    path = os.path.join(tempfile.mkdtemp(prefix="lcbi_eph_"), "earth.txt")
    write_synthetic_ephemeris(path)
    os.environ["LCBININT_EARTH_EPHEMERIS"] = path
    return path


def _ref_orbital_worker(args):
    """One process: the reference's LightCurve (dictionary route) on a list of
    (parameters, mode, Gamma, epochs) tasks."""
    tasks, = args
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import import_reference_module
    ref = import_reference_module()
    modes = [ref.STATIC, ref.CIRCULAR, ref.KEPLER]
    t = time.perf_counter()
    n = 0
    for p, mode, gam, times in tasks:
        par = "piEN" in p
        lc = ref.LightCurve(limb_darkening=ref.LimbDarkening.linear(gam), orbital_motion_mode=modes[mode],
                            parallax=par, event=ref.EventCoordinates(**ORBITAL_EVENT))
        lc(times, p)
        n += len(times)
    return time.perf_counter() - t, n


def cpu_orbital_rate(dicts, modes, gams, times, n_procs, target_seconds):
    """Magnifications/s of the reference on a bounded sample: runs of 25
    consecutive epochs from random models, one process per core, sized to
    about target_seconds (1.5-2 ms per epoch on one core: every epoch
    re-samples the caustic of its own separation)."""
    import multiprocessing as mp
    rng = np.random.default_rng(13)
    run = 25
    per_epoch = 2.0e-3
    n_runs = int(max(n_procs, target_seconds * n_procs / (per_epoch * run)))
    tasks = []
    for _ in range(n_runs):
        m = int(rng.integers(len(dicts)))
        e = int(rng.integers(len(times) - run))
        tasks.append((dicts[m], modes[m], gams[m], times[e:e + run]))
    ctx = mp.get_context("spawn")
    with ctx.Pool(n_procs) as pool:
        t0 = time.perf_counter()
        res = pool.map(_ref_orbital_worker, [(tasks[k::n_procs],) for k in range(n_procs)])
        wall = time.perf_counter() - t0
    n = sum(r[1] for r in res)
    return n / wall, n, wall


def _ref_ps_worker(args):
    s, q, y1, y2, reps = args
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import Reference
    ref = Reference()
    t = time.perf_counter()
    for _ in range(reps):
        ref.binary_mag0(s, q, y1, y2)
    return time.perf_counter() - t


def cpu_ps_rate(s, q, y1, y2, n_procs, target_seconds):
    """Point-source magnifications/s of the reference, one process per core,
    each repeating its share of the batch until about target_seconds."""
    import multiprocessing as mp
    share = [(s[k::n_procs], q[k::n_procs], y1[k::n_procs], y2[k::n_procs]) for k in range(n_procs)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(n_procs) as pool:
        cal = max(pool.map(_ref_ps_worker, [(a, b, c, d, 1) for a, b, c, d in share]))
        reps = int(max(1, min(50, target_seconds / max(cal, 1e-3))))
        t0 = time.perf_counter()
        pool.map(_ref_ps_worker, [(a, b, c, d, reps) for a, b, c, d in share])
        wall = time.perf_counter() - t0
    n = reps * s.size
    return n / wall, n, wall


def cpu_light_curve_rate(target_seconds):
    """The reference's own light-curve path (one curve, one core) on the README light curve."""
    from oracle.oracle import Reference, default_settings
    ref = Reference()
    times = np.linspace(-0.5, 0.5, 200)
    st = default_settings(source_bins=50, finite_mode=1, limb_darkening_c=0.5)
    n, t0 = 0, time.perf_counter()
    while True:
        ref.light_curve_static(st, times, **LC_PARAMS)
        n += times.size
        if time.perf_counter() - t0 > target_seconds:
            break
    wall = time.perf_counter() - t0
    return n / wall, n, wall


def run_other_workload(args, world, rank, local_rank, ncores):
    """Configs 2 (ps_batch) and 1 (light_curve): same JSON line as fs_batch."""
    common = {"metric": METRIC, "unit": "magnifications/s", "steps": args.steps, "warmup": args.warmup,
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
              "data": "synthetic"}
    if args.workload == "ps_batch":
        config = {"workload": "ps_batch: 1e6 point-source magnifications, y U[-1.5,1.5]^2, s log-U[0.3,3], "
                              "q log-U[1e-5,1]", "points": 1_000_000, "l2": "flushed between steps (256 MB write)",
                  "parallelism": f"replicas x{world}"}
    else:
        config = {"workload": "light_curve: README curve, 200 epochs, t0=0 tE=1 u0=-0.01 alpha=0.5 s=0.95 "
                              "q=1e-2 rho=5e-3, linear LD 0.5, Cartesian nbin 50, VBM coordinates",
                  "points": 200, "l2": "inputs and workspaces under 1 MB; not flushed (one curve)",
                  "parallelism": f"replicas x{world}"}
    if args.workload == "adjoint":
        run_adjoint(args, world, rank, local_rank, ncores, common)
        return
    if args.workload == "orbital":
        run_orbital(args, world, rank, local_rank, ncores, common)
        return
    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload == "ps_batch":
            s, q, y1, y2 = ps_batch_workload()
            rate, n, wall = cpu_ps_rate(s, q, y1, y2, ncores, max(2.0, args.cpu_seconds / 2))
            cores, sample = ncores, f"{n} solves ({n // s.size} passes over the batch), {wall:.1f} s on {ncores} processes"
        else:
            rate, n, wall = cpu_light_curve_rate(max(2.0, args.cpu_seconds / 4))
            cores, sample = 1, f"{n // 200} evaluations of the 200-epoch curve, {wall:.1f} s, one process"
        out = dict(common, impl="reference", value=rate, n_gpus=args.gpus, ms_per_step=1e3 * wall * 200 / n
                   if args.workload == "light_curve" else 1e3 * wall * 1e6 / n, config=config,
                   cpu_baseline={"value": rate, "unit": "magnifications/s", "cores": cores, "kind": "reference",
                                 "sample": sample},
                   e2e={"value": rate, "unit": "magnifications/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(out))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib
    ctx = lb.context(local_rank)
    L = ctx._L
    stream = torch.cuda.current_stream(dev)
    L.lcbi_gpu_set_stream(ctx.handle, stream.cuda_stream)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    if args.workload == "ps_batch":
        host = [np.ascontiguousarray(a) for a in ps_batch_workload(seed=rank)]
        n = host[0].size
        d_in = [torch.from_numpy(a).to(dev) for a in host]
        d_A = torch.empty(n, dtype=torch.float64, device=dev)
        d_n = torch.empty(n, dtype=torch.int32, device=dev)
        pinned = [torch.from_numpy(a).pin_memory() for a in host]
        h_A = torch.empty(n, dtype=torch.float64).pin_memory()
        h_n = torch.empty(n, dtype=torch.int32).pin_memory()

        def step_device():
            rc = L.lcbi_gpu_binary_mag0(ctx.handle, n, *[t.data_ptr() for t in d_in], d_A.data_ptr(),
                                        d_n.data_ptr(), None, 1)
            ctx.check(rc, "lcbi_gpu_binary_mag0")

        def step_e2e():
            rc = L.lcbi_gpu_binary_mag0(ctx.handle, n, *[t.data_ptr() for t in pinned], h_A.data_ptr(),
                                        h_n.data_ptr(), None, 0)
            ctx.check(rc, "lcbi_gpu_binary_mag0")
        h2d, d2h = sum(a.nbytes for a in host), n * 12
        flush_between = True
    else:
        P = np.array([[LC_PARAMS[k] for k in ("t0", "tE", "u0", "alpha", "s", "q", "rho")]], dtype=np.float64)
        times = np.linspace(-0.5, 0.5, 200)
        n = times.size
        opt = lb.Options(inverse_ray_grid="cartesian", nbin=50)
        st = opt.fs_settings(lb.LimbDarkening.linear(0.5))
        first = np.zeros(1, dtype=np.int64)
        cnt = np.array([n], dtype=np.int32)
        A = np.empty(n)

        def step_device():
            rc = L.lcbi_gpu_light_curves(ctx.handle, __import__("ctypes").byref(st), 1, _lib.ptr(P),
                                         _lib.ptr(first), _lib.ptr(cnt), _lib.ptr(times), n, _lib.ptr(A), None,
                                         None)
            ctx.check(rc, "lcbi_gpu_light_curves")
        step_e2e = step_device
        h2d, d2h = times.nbytes + P.nbytes, A.nbytes
        flush_between = False
    for _ in range(args.warmup):
        if flush_between:
            flush_l2(flush)
        step_device()
    torch.cuda.synchronize(dev)
    launches0 = ctx.launches
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local_rank) as clocks:
        for k in range(args.steps):
            if flush_between:
                flush_l2(flush)
            ev0[k].record(stream)
            step_device()
            ev1[k].record(stream)
        torch.cuda.synchronize(dev)
    my_ms = float(sum(a.elapsed_time(b) for a, b in zip(ev0, ev1)))
    launches = ctx.launches - launches0
    if world > 1:
        torch.distributed.barrier()
    stage_ms = None
    if args.workload == "light_curve":
        # Where one curve's time goes: the stages of one more call, CUDA-event timed.
        L.lcbi_gpu_set_timing(ctx.handle, 1)
        step_device()
        sm = np.zeros(8)
        sn = np.zeros(8, dtype=np.int64)
        L.lcbi_gpu_stage_times(ctx.handle, _lib.ptr(sm), _lib.ptr(sn), 8)
        L.lcbi_gpu_set_timing(ctx.handle, 0)
        names = ["caustics+ld", "decide", "seeds", "cartesian", "polar", "point_source"]
        stage_ms = {names[i]: float(sm[i]) for i in range(6)}
    e2e_s = 0.0
    for _ in range(args.steps):
        if flush_between:
            flush_l2(flush)
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        step_e2e()
        e2e_s += time.perf_counter() - t1
    (max_ms, max_e2e), (n_all,) = reduce_over_ranks([my_ms, e2e_s], [n], world, dev)
    ms_per_step = max_ms / args.steps
    peak = ctypes_double()
    L.lcbi_gpu_measure_fp64_peak(ctx.handle, peak.ref())
    out = dict(common, value=n_all / (ms_per_step * 1e-3), n_gpus=world, ms_per_step=ms_per_step, config=config,
               e2e={"value": n_all * args.steps / max_e2e, "unit": "magnifications/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
               gpu_launches=int(launches), clocks=clocks.summary())
    if stage_ms is not None:
        out["stage_ms_one_call"] = stage_ms
    if args.workload == "ps_batch":
        achieved = n * F_PS / (ms_per_step * 1e-3) / 1e12
        out["roofline"] = {"bound": "fp64", "kernel": "ps_batch_kernel", "achieved": achieved, "peak": peak.value,
                           "unit": "TFLOP/s", "frac": achieved / peak.value if peak.value else None,
                           "peak_no_fma": peak.value / 2.0,
                           "frac_of_no_fma_peak": 2.0 * achieved / peak.value if peak.value else None,
                           "traffic": PS_DRAM_BYTES * n / 1e6,
                           "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 1e6-point "
                                             "launch, scaled by points",
                           "flop_per_solve": F_PS,
                           "peak_source": "device-measured FP64 FMA loop (lcbi_gpu_measure_fp64_peak); the no-FMA "
                                          "figure is half of it (the kernel is built without contraction)"}
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        if args.workload == "ps_batch":
            rate, nn, wall = cpu_ps_rate(*host, ncores, args.cpu_seconds / 2)
            out["cpu_baseline"] = {"value": rate, "unit": "magnifications/s", "cores": ncores, "kind": "reference",
                                   "sample": f"{nn} solves, {wall:.1f} s on {ncores} processes"}
        else:
            rate, nn, wall = cpu_light_curve_rate(args.cpu_seconds / 4)
            out["cpu_baseline"] = {"value": rate, "unit": "magnifications/s", "cores": 1, "kind": "reference",
                                   "sample": f"{nn // 200} curves, {wall:.1f} s, one process"}
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def adjoint_forward_error(P, T, A, method, device, n_sample=96, seed=17):
    """Relative error of the adjoint workload's forward magnifications against
    a converged finite-source value on a random sample of its finite-source
    epochs (hexadecapole and inverse ray): the same source forced to Cartesian
    inverse ray at nbin 400, whose own convergence is shown by nbin 800."""
    import lcbinint_b200 as lb
    M, K = T.shape
    fs = np.nonzero(method.ravel() >= 1)[0]
    if fs.size == 0:
        return None
    idx = np.random.default_rng(seed).choice(fs, min(n_sample, fs.size), replace=False)
    m, e = np.divmod(idx, K)
    t0, tE, u0, al, s_, q_, rho, gam = (P[m, j] for j in range(8))
    tau = (T[m, e] - t0) * (1.0 / tE)
    y1 = tau * np.cos(al) - u0 * np.sin(al)
    y2 = tau * np.sin(al) + u0 * np.cos(al)
    conv = {}
    for nb in (400, 800):
        vals = np.empty(idx.size)
        for g in np.unique(gam[:]):
            sel = gam == g
            vals[sel] = lb.binary_inverse_ray_batch(s_[sel], 1.0 / q_[sel], y1[sel], y2[sel], np.abs(rho[sel]),
                                                    lb.LimbDarkening.linear(float(g)),
                                                    lb.Options(inverse_ray_grid="cartesian", nbin=nb), device=device)
        conv[nb] = vals
    err = np.abs(A.ravel()[idx] / conv[800] - 1.0)
    ref = np.abs(conv[400] / conv[800] - 1.0)
    return {"vs": "forced Cartesian inverse ray at nbin 800 on the same epochs", "points": int(idx.size),
            "median_rel": float(np.median(err)), "p90_rel": float(np.quantile(err, 0.9)),
            "max_rel": float(err.max()), "frac_within_1e-4": float(np.mean(err <= 1e-4)),
            "reference_convergence": {"nbin 400 vs 800 median_rel": float(np.median(ref)),
                                      "max_rel": float(ref.max())}}


def run_adjoint(args, world, rank, local_rank, ncores, common):
    """Adjoint workload: magnifications and their gradients in (t0, tE, u0, alpha, s,
    q, rho, Gamma) for 256 models x 500 epochs through the library's adjoint
    (lcbi_gpu_light_curves_grad), against the forward alone, against a plain
    GPU forward of one point per call with central finite differences (17
    forwards per point), and against the reference's CPU forward with the same
    finite differences."""
    P, T = adjoint_workload(seed=2 + rank)
    M, K = T.shape
    n = M * K
    config = {"workload": "adjoint: 256 models x 500 epochs (fs_batch model distribution, t0 +- 2 tE), auto "
                          "decision tree, nbin 50, dA/d(t0, tE, u0, alpha, s, q, rho, Gamma)",
              "points": n, "l2": "not flushed (inputs and results under 11 MB; workspaces reused)",
              "parallelism": f"replicas x{world}"}
    if args.impl == "reference":
        if rank != 0:
            return
        rate, nn, wall = cpu_adjoint_rate(P, T, ncores, max(ncores, 32))
        out = dict(common, impl="reference", value=rate, n_gpus=args.gpus, ms_per_step=1e3 * n / rate,
                   config=config,
                   cpu_baseline={"value": rate, "unit": "magnifications/s", "cores": ncores, "kind": "reference",
                                 "sample": f"forward on {nn} epochs of {nn // K} models, {wall:.1f} s; "
                                           "x17 for central differences in 8 parameters"},
                   e2e={"value": rate, "unit": "magnifications/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(out))
        return
    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib
    from lcbinint_b200.autograd import light_curves_with_grad
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, PS_EXACT, PS_ON_DEVICE, LcbiStructs
    ctx = lb.context(local_rank)
    L = ctx._L
    for _ in range(args.warmup):
        light_curves_with_grad(P, T, device=local_rank)
        light_curves_with_grad(P, T, device=local_rank, with_grad=False)
    launches0 = ctx.launches
    with ClockSampler(local_rank) as clocks:
        tg = tf = 0.0
        for _ in range(args.steps):
            t1 = time.perf_counter()
            A, dA, method, status = light_curves_with_grad(P, T, device=local_rank)
            tg += time.perf_counter() - t1
            t1 = time.perf_counter()
            light_curves_with_grad(P, T, device=local_rank, with_grad=False)
            tf += time.perf_counter() - t1
    launches = (ctx.launches - launches0) // 2
    # Plain GPU baseline: one point per call (positions as the light curves
    # form them), 17 calls per point for central differences.
    rng = np.random.default_rng(3)
    sample = rng.integers(0, n, 64)
    opt = lb.Options()
    st_cache = {}
    pts = np.zeros(1, dtype=FS_POINT_DTYPE)
    res = np.zeros(1, dtype=FS_RESULT_DTYPE)
    t_plain = 0.0
    for k in sample:
        m, e = divmod(int(k), K)
        t0, tE, u0, al, s_, q_, rho, gam = P[m]
        tau = (T[m, e] - t0) * (1.0 / tE)
        g = float(gam)
        if g not in st_cache:
            st_cache[g] = opt.fs_settings(lb.LimbDarkening.linear(g))
        st = st_cache[g]
        pts[0] = (s_, 1.0 / q_, tau * math.cos(al) - u0 * math.sin(al), tau * math.sin(al) + u0 * math.cos(al),
                  abs(rho), 0.0, 0, 0, PS_EXACT | PS_ON_DEVICE, 0)
        t1 = time.perf_counter()
        rc = L.lcbi_gpu_binary_mag(ctx.handle, __import__("ctypes").byref(st), 1, None, 0, 1, pts.ctypes.data,
                                   res.ctypes.data, 0)
        t_plain += time.perf_counter() - t1
        ctx.check(rc, "lcbi_gpu_binary_mag")
    plain_rate = len(sample) / t_plain / 17.0
    (max_g, max_f), (n_all,) = reduce_over_ranks([tg, tf], [n], world, dev)
    value = n_all * args.steps / max_g
    out = dict(common, value=value, n_gpus=world, ms_per_step=1e3 * max_g / args.steps, config=config,
               fwd_grad_over_fwd=max_g / max_f,
               forward_only={"value": n_all * args.steps / max_f, "unit": "magnifications/s"},
               plain_gpu_fd={"value": plain_rate, "unit": "magnifications/s",
                             "how": "one point per lcbi_gpu_binary_mag call, 17 calls per gradient, 64 points"},
               speedup_vs_plain_gpu_fd=value / plain_rate,
               methods={str(k): int((method == k).sum()) for k in range(4)},
               status_ok=int((status == 0).sum()), grad_finite=int(np.isfinite(dA).all(axis=2).sum()),
               e2e={"value": value, "unit": "magnifications/s", "h2d_bytes_per_step": int(P.nbytes + T.nbytes),
                    "d2h_bytes_per_step": int(n * 8 * 9)},
               gpu_launches=int(launches), clocks=clocks.summary())
    out["forward_error"] = adjoint_forward_error(P, T, A, method, local_rank)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        rate, nn, wall = cpu_adjoint_rate(P, T, ncores, max(ncores, 32))
        out["cpu_baseline"] = {"value": rate, "unit": "magnifications/s", "cores": ncores, "kind": "reference",
                               "sample": f"forward on {nn} epochs of {nn // K} models, {wall:.1f} s on {ncores} "
                                         "processes; x17 for central differences in 8 parameters"}
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def run_orbital(args, world, rank, local_rank, ncores, common):
    """Orbital workload: 1024 models x 2000 epochs with circular or Keplerian lens
    orbital motion and annual parallax through the batched C ABI
    (lcbi_gpu_magnification_arrays, LensModel's route), host arrays in and
    out.  The Earth ephemeris is synthetic (the reference's table is not in
    its repository); --no-parallax measures the orbital-motion half alone."""
    parallax = not args.no_parallax
    if parallax:
        orbital_ephemeris()
    dicts, modes, gams, times = orbital_workload(seed=3 + rank, parallax=parallax)
    if args.models > 0:
        dicts, modes, gams = dicts[:args.models], modes[:args.models], gams[:args.models]
    M, K = len(dicts), times.size
    n = M * K
    config = {"workload": f"orbital: {M} models x 2000 epochs over 200 days, half circular / half Keplerian lens "
                          "orbital motion (g1, g2 U[-1,1]/yr, g3 U[0,0.5]/yr), fs_batch model distribution, "
                          "linear LD U[0,0.8], auto decision tree, nbin 50; " +
                          ("annual parallax piEN, piEE U[-0.5,0.5] (synthetic Earth ephemeris, event at the "
                           "Galactic bulge)" if parallax else "no parallax"),
              "points": n, "l2": "not flushed (per-epoch caustic samples, 2.9 GB per chunk, exceed L2)",
              "parallelism": f"replicas x{world}"}
    if args.impl == "reference":
        if rank != 0:
            return
        rate, nn, wall = cpu_orbital_rate(dicts, modes, gams, times, ncores, max(4.0, args.cpu_seconds / 2))
        out = dict(common, impl="reference", value=rate, n_gpus=args.gpus, ms_per_step=1e3 * n / rate,
                   config=config,
                   cpu_baseline={"value": rate, "unit": "magnifications/s", "cores": ncores, "kind": "reference",
                                 "sample": f"{nn} epochs in runs of 25 from random models, {wall:.1f} s on "
                                           f"{ncores} processes"},
                   e2e={"value": rate, "unit": "magnifications/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(out))
        return
    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib, api
    ctx = lb.context(local_rank)
    L = ctx._L
    ev = lb.EventCoordinates(**ORBITAL_EVENT)
    cps = np.concatenate([api.binary_c_params([p], lb.LimbDarkening.linear(g), ev, orbital_motion_mode=m,
                                              parallax=parallax)
                          for p, m, g in zip(dicts, modes, gams)])
    co = lb.Options().c_options()
    first = (np.arange(M, dtype=np.int64) * K)
    count = np.full(M, K, dtype=np.int32)
    all_times = np.ascontiguousarray(np.tile(times, M))
    res = np.zeros(n, dtype=_lib.RESULT_DTYPE)
    status = np.zeros(M, dtype=np.int32)

    def step():
        rc = L.lcbi_gpu_magnification_arrays(ctx.handle, M, _lib.ptr(cps), _lib.ptr(co), _lib.ptr(first),
                                             _lib.ptr(count), _lib.ptr(all_times), n, 0, _lib.ptr(res),
                                             _lib.ptr(status))
        ctx.check(rc, "lcbi_gpu_magnification_arrays")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    launches0 = ctx.launches
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local_rank) as clocks:
        wall = 0.0
        for _ in range(args.steps):
            torch.cuda.synchronize(dev)
            t1 = time.perf_counter()
            step()
            wall += time.perf_counter() - t1
    launches = (ctx.launches - launches0) // max(1, args.steps)
    # Device stage times of one further step (per-stage CUDA events, which
    # run the stages one after another).
    L.lcbi_gpu_set_timing(ctx.handle, 1)
    step()
    stage_ms = np.zeros(8)
    stage_n = np.zeros(8, dtype=np.int64)
    L.lcbi_gpu_stage_times(ctx.handle, _lib.ptr(stage_ms), _lib.ptr(stage_n), 8)
    L.lcbi_gpu_set_timing(ctx.handle, 0)
    (max_wall,), (n_all,) = reduce_over_ranks([wall], [n], world, dev)
    value = n_all * args.steps / max_wall
    names = ["caustics+ld", "decide", "seeds", "cartesian", "polar", "point_source"]
    out = dict(common, value=value, n_gpus=world, ms_per_step=1e3 * max_wall / args.steps, config=config,
               status_ok_sets=int((status == 0).sum()),
               finite_source_evaluated=int(np.isfinite(res["finite_source_magnification"]).sum()),
               stage_ms_one_call={names[i]: float(stage_ms[i]) for i in range(6)},
               timing="wall clock around the host-pointer call (host orbit geometry on the host cores, "
                      "H2D, kernels, D2H); the device stages of one further call are CUDA-event timed",
               e2e={"value": value, "unit": "magnifications/s", "h2d_bytes_per_step": int(cps.nbytes + all_times.nbytes),
                    "d2h_bytes_per_step": int(res.nbytes + status.nbytes)},
               gpu_launches=int(launches), clocks=clocks.summary())
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        rate, nn, w = cpu_orbital_rate(dicts, modes, gams, times, ncores, args.cpu_seconds)
        out["cpu_baseline"] = {"value": rate, "unit": "magnifications/s", "cores": ncores, "kind": "reference",
                               "sample": f"{nn} epochs in runs of 25 from random models, {w:.1f} s on {ncores} "
                                         "processes"}
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


# --------------------------------------------------------------------------- main


def reduce_over_ranks(maxes, sums, world, device):
    """Across the ranks: the max of each entry of `maxes` (timings: the job is
    as slow as its slowest rank) and the sum of each entry of `sums` (points
    and cells processed), so that a replica job's throughput is the work of
    all ranks over the slowest rank's time."""
    maxes = [float(v) for v in maxes]
    sums = [float(v) for v in sums]
    if world == 1:
        return maxes, sums
    import torch
    import torch.distributed as dist
    t = torch.tensor(maxes, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor(sums, dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return t.cpu().tolist(), c.cpu().tolist()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fs_batch", choices=["fs_batch", "ps_batch", "light_curve", "adjoint",
                                                                   "orbital"])
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--points", type=int, default=0,
                    help="use only N points of the batch, chosen at random, with a small workspace (one "
                         "first-pass warp per SM, eight second-pass blocks): small cases for profiler captures")
    ap.add_argument("--point", type=int, default=-1,
                    help="fs_batch: only point N of the batch, on a second-pass block (cell budget 1), with a "
                         "small workspace (one first-pass warp per SM, eight second-pass blocks, hence eight "
                         "early-pass blocks for its seed-half units): the one-kernel "
                         "case for profiler captures of the block scan (point 1285: the batch's largest "
                         "Cartesian point)")
    ap.add_argument("--rays", default="f64", choices=["f64", "f32"],
                    help="fs_batch: lens map of the inverse-ray cells in FP64 (bit-exact) or FP32 about "
                         "image-centred anchors (sums FP64); f32 also reports its error against f64")
    ap.add_argument("--autotune", action="store_true",
                    help="fs_batch: launch shapes picked by lcbi_gpu_autotune on the batch before the warm-up")
    ap.add_argument("--no-parallax", action="store_true",
                    help="orbital workload: lens orbital motion only (no annual parallax)")
    ap.add_argument("--models", type=int, default=0,
                    help="orbital workload: use only the first N models (small cases for profiler captures)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    if args.workload != "fs_batch":
        run_other_workload(args, world, rank, local_rank, ncores)
        return
    # One batch of 4,096 points per GPU; with several GPUs the batches form one
    # job of 4,096 N points that is split over the ranks (weak scaling).
    rows = np.concatenate([fs_batch_workload(seed=1 + r) for r in range(world)]) if world > 1 \
        else fs_batch_workload(seed=1)
    if args.points > 0:
        rows = rows[np.random.default_rng(5).permutation(len(rows))[: args.points]]
    if args.point >= 0:
        rows = rows[[args.point]]
    config = {"workload": "fs_batch: 4096 forced inverse-ray points, 64 models x 64 epochs, "
                          "Cartesian/polar mixed, nbin 20-200, linear LD",
              "points": int(len(rows)), "models": 64,
              "precision": "fp64" if args.rays == "f64" else
                           "fp32 ray map about image-centred anchors, fp64 sums, fp64 seeds and decisions",
              "l2": "flushed between steps (256 MB write)",
              "parallelism": "one GPU" if world == 1 else
                             f"{world} GPUs: one batch of {len(rows)} points split by LPT on estimated cells "
                             "(lcbinint_b200.shard), results all-gathered over NCCL inside the step"}

    if args.impl == "reference":
        if rank != 0:
            return
        per_step = []
        for _ in range(args.warmup + args.steps):
            rate, n, wall = cpu_reference_rate(rows, ncores, target_seconds=max(2.0, args.cpu_seconds / 4))[:3]
            per_step.append((rate, n, wall))
        timed = per_step[args.warmup:]
        tot_n = sum(x[1] for x in timed)
        tot_t = sum(x[2] for x in timed)
        value = tot_n / tot_t
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": "magnifications/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config,
            "cpu_baseline": {"value": value, "unit": "magnifications/s", "cores": ncores, "kind": "reference",
                             "sample": f"{tot_n} points of the batch over {args.steps} steps"},
            "e2e": {"value": value, "unit": "magnifications/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)

    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_RESULT_DTYPE, LcbiStructs

    ctx = lb.context(local_rank)
    L = ctx._L
    stream = torch.cuda.current_stream(dev)
    L.lcbi_gpu_set_stream(ctx.handle, stream.cuda_stream)
    if args.point >= 0:
        ctx.check(L.lcbi_gpu_set_cell_budget(ctx.handle, 1), "lcbi_gpu_set_cell_budget")
        ctx.check(L.lcbi_gpu_set_workspace(ctx.handle, 1, 8, 16384), "lcbi_gpu_set_workspace")
    elif args.points > 0:
        # A small case for profiler captures: about 2 GB of device workspace.
        ctx.check(L.lcbi_gpu_set_workspace(ctx.handle, 1, 8, 131072), "lcbi_gpu_set_workspace")

    settings, models, pts_all = fs_batch_arrays(rows)
    st_arr = (LcbiStructs.FsSettings * len(settings))(*settings)
    parts = None
    if world > 1:
        # Every rank computes the same partition from the same points.
        from lcbinint_b200.shard import gather_results, lpt_partition, point_costs
        a_ps = lb.binary_mag0_batch(pts_all["s"], pts_all["q"], pts_all["y1"], pts_all["y2"], device=local_rank)
        parts = lpt_partition(point_costs(pts_all, settings, a_ps=a_ps), world)
        pts = np.ascontiguousarray(pts_all[parts[rank]])
        config["points_per_rank"] = [int(len(p)) for p in parts]
    else:
        pts = pts_all
    n = len(pts)
    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).to(dev)
    d_res = torch.zeros(n * FS_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    if world > 1:
        # The result gather: every rank's records, padded to the largest share.
        g_in = torch.zeros(max(len(p) for p in parts) * FS_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        g_out = [torch.empty_like(g_in) for _ in range(world)]

    def step_device():
        rc = L.lcbi_gpu_binary_mag(ctx.handle, st_arr, len(settings), models.ctypes.data, len(models), n,
                                   d_pts.data_ptr(), d_res.data_ptr(), _lib.DEVICE_POINTERS | 2)
        ctx.check(rc, "lcbi_gpu_binary_mag")
        if world > 1:
            g_in[: d_res.numel()].copy_(d_res)
            torch.distributed.all_gather(g_out, g_in)

    res_host = np.zeros(n, dtype=FS_RESULT_DTYPE)

    def step_e2e():
        rc = L.lcbi_gpu_binary_mag(ctx.handle, st_arr, len(settings), None, 0, n, pts.ctypes.data,
                                   res_host.ctypes.data, 0)
        ctx.check(rc, "lcbi_gpu_binary_mag")
        if world > 1:
            gather_results(res_host, parts, len(pts_all), device=dev)

    fp32_error = None
    if args.rays == "f32":
        # The FP64 magnifications of the same points, for the FP32 arm's error.
        step_device()
        res64 = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=FS_RESULT_DTYPE)["magnification"].copy()
        L.lcbi_gpu_set_ray_precision(ctx.handle, 32)
    if args.autotune:
        # Launch shapes picked on this batch by the library's autotuner.
        shape = np.zeros(3, dtype=np.int32)
        best = ctypes_double()
        rc = L.lcbi_gpu_autotune(ctx.handle, st_arr, len(settings), models.ctypes.data, len(models), n,
                                 d_pts.data_ptr(), d_res.data_ptr(), _lib.DEVICE_POINTERS | 2, _lib.ptr(shape),
                                 best.ref())
        ctx.check(rc, "lcbi_gpu_autotune")
        config["launch_shape"] = {"tile_flood_blocks_per_sm": int(shape[0]), "warps_per_sm": int(shape[1]),
                                  "second_pass_blocks": int(shape[2]), "picked_by": "lcbi_gpu_autotune",
                                  "best_ms": best.value}
    for _ in range(args.warmup):
        flush_l2(flush)
        step_device()
    torch.cuda.synchronize(dev)
    launches0 = ctx.launches
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local_rank) as clocks:
        for k in range(args.steps):
            flush_l2(flush)
            ev0[k].record(stream)
            step_device()
            ev1[k].record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    step_ms = [a.elapsed_time(b) for a, b in zip(ev0, ev1)]
    my_ms = float(np.sum(step_ms))
    launches = ctx.launches - launches0
    # Where a step's time goes: further steps with per-stage CUDA events.  With
    # stage timing on the library runs the stages one after another (the timed
    # steps above run the second Cartesian pass beside the polar passes), so
    # these stage times add up to more than a timed step.
    stage_steps = min(args.steps, 3)
    # Where each stream of an overlapped step ends (stream marks: timing
    # events recorded where the early, side and polar streams' work ends,
    # the overlap unchanged), over further steps.
    L.lcbi_gpu_set_stream_marks(ctx.handle, 1)
    marks = []
    for _ in range(stage_steps):
        flush_l2(flush)
        step_device()
        m = np.zeros(3)
        L.lcbi_gpu_stream_marks(ctx.handle, _lib.ptr(m), 3)
        marks.append(m)
    L.lcbi_gpu_set_stream_marks(ctx.handle, 0)
    marks = np.median(np.array(marks), axis=0)
    stream_end_ms = {"early": float(marks[0]), "side": float(marks[1]), "polar": float(marks[2]),
                     "from": "the start of the seeding stage, median of further overlapped steps"}
    L.lcbi_gpu_set_timing(ctx.handle, 1)
    for _ in range(stage_steps):
        flush_l2(flush)
        step_device()
    torch.cuda.synchronize(dev)
    stage_ms = np.zeros(8)
    stage_n = np.zeros(8, dtype=np.int64)
    L.lcbi_gpu_stage_times(ctx.handle, _lib.ptr(stage_ms), _lib.ptr(stage_n), 8)
    L.lcbi_gpu_set_timing(ctx.handle, 0)
    rays = np.zeros(n, dtype=np.uint64)
    L.lcbi_gpu_last_ray_counts(ctx.handle, n, _lib.ptr(rays))
    res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=FS_RESULT_DTYPE)
    if args.rays == "f32":
        a32 = res["magnification"]
        ok = np.isfinite(a32) & np.isfinite(res64) & (res64 != 0)
        rel = np.abs(a32[ok] / res64[ok] - 1.0)
        fp32_error = {"vs": "the same points with the FP64 map (bit-exact with the reference)",
                      "points": int(ok.sum()), "max_rel": float(rel.max()), "p99_rel": float(np.quantile(rel, 0.99)),
                      "median_rel": float(np.median(rel)), "identical": int((rel == 0).sum())}

    # end to end: host arrays through the public C ABI (planning, H2D copies,
    # kernels, D2H of the results), wall-clocked per step
    for _ in range(2):
        step_e2e()
    if world > 1:
        torch.distributed.barrier()
    e2e_s = 0.0
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        step_e2e()
        e2e_s += time.perf_counter() - t1
    (max_ms, max_e2e_s), (n_all, rays_all) = reduce_over_ranks([my_ms, e2e_s], [n, float(rays.sum())], world, dev)
    ms_per_step = max_ms / args.steps
    value = n_all / (ms_per_step * 1e-3)

    peak = ctypes_double()
    L.lcbi_gpu_measure_fp64_peak(ctx.handle, peak.ref())
    names = ["caustics+ld", "decide", "seeds", "cartesian", "polar", "point_source"]
    shares = {names[i]: float(stage_ms[i]) for i in range(6)}
    cart = res["method"] == 2
    polar_m = res["method"] == 3
    # The step's dominant work is the inverse-ray integration (the Cartesian
    # and polar scans; the serialised stage times below show the split).  Its
    # achieved rate is over the device-timed step itself: every counted cell
    # of the step (all ranks) x F_RAY flop / ms_per_step, so it follows from
    # rays_per_s and the step time alone.  The scans are built without FMA
    # contraction (bit-exact FP64), so one FP64 instruction is one flop: the
    # attainable peak is half the FMA probe's.
    achieved = rays_all * F_RAY / (ms_per_step * 1e-3) / 1e12
    chip_peak = peak.value * world
    roofline = {"bound": "fp64", "kernel": "inverse-ray scans (cartesian_*_kernel, tile_flood_kernel, "
                                           "polar_*_kernel) over the whole step",
                "achieved": achieved, "peak": chip_peak, "unit": "TFLOP/s",
                "frac": achieved / chip_peak if chip_peak else None,
                "peak_no_fma": chip_peak / 2.0,
                "frac_of_no_fma_peak": 2.0 * achieved / chip_peak if chip_peak else None,
                "traffic": RAY_DRAM_BYTES_PER_CELL * rays_all,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the early-pass scan of "
                                  "point 1285 (6.35e6 cells), per cell, times the step's counted cells",
                "peak_source": "device-measured FP64 FMA loop (lcbi_gpu_measure_fp64_peak) x GPUs; the no-FMA "
                               "figure is half of it (one flop per FP64 instruction)",
                "achieved_over": "ms_per_step (device-timed steps): counted cells of the step x flop_per_ray",
                "stage_ms_serialised": {k: v / stage_steps for k, v in shares.items()},
                "stream_end_ms": stream_end_ms,
                "stage_timing": f"{stage_steps} further steps with the stages serialised by per-stage events "
                                "(they overlap on three streams in the timed steps, so they add up to more)",
                "flop_per_ray": F_RAY}
    out = {
        "metric": METRIC, "value": value, "unit": "magnifications/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
        "rays_per_s": rays_all / (ms_per_step * 1e-3),
        "methods": {"cartesian": int(cart.sum()), "polar": int(polar_m.sum())},
        "status_ok": int((res["status"] == 0).sum()),
        "roofline": roofline,
        "e2e": {"value": n_all * args.steps / max_e2e_s, "unit": "magnifications/s",
                "h2d_bytes_per_step": int(pts.nbytes), "d2h_bytes_per_step": int(res_host.nbytes)},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if fp32_error is not None:
        out["fp32_error"] = fp32_error
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        # The reference on every point of the batch: its rate is the CPU
        # baseline, and its magnifications are the parity check of this run.
        R, RM, wall = reference_inverse_ray(rows, ncores)
        out["cpu_baseline"] = {"value": len(rows) / wall, "unit": "magnifications/s", "cores": ncores,
                               "kind": "reference",
                               "sample": f"all {len(rows)} points of the batch, {wall:.1f} s wall on {ncores} "
                                         "processes"}
        if args.rays == "f64":
            out["parity"] = parity_summary(res["magnification"].copy(), res["method"].copy(),
                                           res["status"].copy(), R, RM)
            if out["parity"]["pass"]:
                config["precision"] = "fp64, bit-exact vs reference (see parity)"
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


class ctypes_double:
    def __init__(self):
        import ctypes
        self._v = ctypes.c_double(0.0)

    def ref(self):
        import ctypes
        return ctypes.byref(self._v)

    @property
    def value(self):
        return self._v.value


if __name__ == "__main__":
    main()
