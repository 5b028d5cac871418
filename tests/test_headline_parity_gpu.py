"""Parity on the headline finite-source batch at its own sizes.

The batch is the bench's default workload: 4,096 forced inverse-ray points
from 64 models (q to 1e-5, rho to 1e-4, nbin 20-200, Cartesian and polar
mixed, linear limb darkening).  The device integrates the whole batch in one
call, as the bench does; the reference (compiled from its own sources,
``oracle/_ref``) then integrates a stratified subset of the same points with
``binary_inverse_ray`` semantics (python/lcbinint_pybind.cpp:3826-3847):

* the batch's largest Cartesian point (index 1285, about 6.4e6 counted cells);
* the 32 Cartesian points with the most counted cells;
* the 32 polar points with the most azimuthal bins (the finest polar
  lattices: rho near 1e-4 at nbin near 200);
* 256 random others.

Bar: Cartesian magnifications bit for bit; polar ones within 1e-12 relative
of the reference (the same cells, summed exactly here and by a running sum
there), and bit for bit equal, with the same cell count, to the oracle's
integral of the same lattice with its cells summed the device's way (a
128-bit fixed-point sum): that pins every polar cell and every cell's term,
not only the total; methods equal and status 0 on every point.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POLAR_REL_TOL = 1e-12


def _device_batch(rows):
    import bench
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_RESULT_DTYPE, LcbiStructs
    settings, models, pts = bench.fs_batch_arrays(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    ctx = _lib.Context(0)
    try:
        L = ctx._L
        res = np.zeros(len(pts), dtype=FS_RESULT_DTYPE)
        rc = L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), models.ctypes.data, len(models), len(pts),
                                   pts.ctypes.data, res.ctypes.data, 2)
        ctx.check(rc, "lcbi_gpu_binary_mag")
        rays = np.zeros(len(pts), dtype=np.uint64)
        L.lcbi_gpu_last_ray_counts(ctx.handle, len(pts), _lib.ptr(rays))
    finally:
        ctx.close()
    return res, rays


def _polar_phi_bins(rows):
    """The reference's azimuthal bin count (finite_source_magnifier.cpp:1181-1197)
    with the source position standing in for the farthest seed."""
    r = np.hypot(rows[:, 2], rows[:, 3])
    rho = rows[:, 4]
    dr = rho / rows[:, 7]
    return 2.0 * np.pi * np.maximum(1.0, r + 4.0 * rho) / (dr * 4.0)


def _subset(rows, rays):
    cart = np.nonzero(rows[:, 6] == 1)[0]
    polar = np.nonzero(rows[:, 6] == 2)[0]
    big_cart = cart[np.argsort(rays[cart].astype(np.float64))[::-1][:32]]
    fine_polar = polar[np.argsort(_polar_phi_bins(rows[polar]))[::-1][:32]]
    rest = np.setdiff1d(np.arange(len(rows)), np.concatenate([big_cart, fine_polar, [1285]]))
    rnd = np.random.default_rng(2024).choice(rest, 256, replace=False)
    return np.unique(np.concatenate([[1285], big_cart, fine_polar, rnd]))


def test_headline_batch_subset_matches_reference(ref_lib):
    import bench
    rows = bench.fs_batch_workload(seed=1)
    assert len(rows) == 4096
    res, rays = _device_batch(rows)
    sel = _subset(rows, rays)
    # The batch's largest Cartesian point is in the subset.
    cart_all = rows[:, 6] == 1
    assert int(np.argmax(np.where(cart_all, rays.astype(np.float64), -1.0))) == 1285
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    R, RM, _ = bench.reference_inverse_ray(rows[sel], ncores)
    A = res["magnification"][sel].copy()
    M = res["method"][sel].copy()
    S = res["status"][sel].copy()
    cells = rays[sel]
    summary = bench.parity_summary(A, M, S, R, RM)
    assert (S == 0).all(), np.unique(S, return_counts=True)
    assert (M == RM).all(), f"{int((M != RM).sum())} methods differ"
    assert (M == rows[sel, 6].astype(np.int32) + 1).all()
    cart = M == 2
    bad = np.nonzero(cart & (A.view(np.int64) != R.view(np.int64)))[0]
    assert bad.size == 0, (f"{bad.size} Cartesian points differ, e.g. point {int(sel[bad[0]])}: "
                           f"{A[bad[0]]!r} vs {R[bad[0]]!r}; {summary}")
    pol = M == 3
    fixed, fcells = _oracle_polar_fixed(rows[sel[pol]])
    diff = np.nonzero((A[pol].view(np.int64) != fixed.view(np.int64)) | (cells[pol] != fcells))[0]
    detail = [(int(sel[pol][k]), int(cells[pol][k]), int(fcells[k]), float(A[pol][k] / fixed[k] - 1.0))
              for k in diff[:8]]
    assert diff.size == 0, f"{diff.size} polar points differ from the oracle's exact sum (point, cells, oracle cells, rel): {detail}"
    rel = np.abs(A[pol] / R[pol] - 1.0)
    assert rel.max() <= POLAR_REL_TOL, summary
    assert summary["pass"], summary


def _oracle_polar_fixed(rows):
    """The oracle's polar integrals of the rows with the device's exact sum,
    and their cell counts, one process per core."""
    import multiprocessing as mp
    n = max(1, min(len(rows), len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()))
    with mp.get_context("spawn").Pool(n) as pool:
        res = pool.map(_fixed_worker, [rows[k::n] for k in range(n)])
    fixed = np.empty(len(rows))
    cells = np.empty(len(rows), dtype=np.uint64)
    for k, (f, c) in enumerate(res):
        fixed[k::n] = f
        cells[k::n] = c
    return fixed, cells


def _fixed_worker(rows):
    from oracle.oracle import Oracle, default_settings
    orc = Oracle()
    f, c = [], []
    for r in rows:
        st = default_settings(source_bins=int(r[7]), finite_mode=int(r[6]), limb_darkening_c=float(r[5]))
        _, _, Af, cells = orc.inverse_ray_fixed(st, r[0], r[1], r[2], r[3], r[4])
        f.append(Af[0])
        c.append(int(cells[0]))
    return f, c
