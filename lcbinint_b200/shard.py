"""One finite-source batch split over several GPUs.

The points of a batch are independent (FiniteSourceMagnifier::binary_mag,
src/lcbinint/magnification/finite_source_magnifier.cpp:4633-4843, evaluates
each on its own), so a batch shards with no exchange on the data path: every
device integrates its share and the results are gathered in input order.

Per-point cost spans four orders of magnitude (1e3 to 1e7 lattice cells), so
an even split by count leaves one device holding the largest points while the
others idle.  The split here is longest-processing-time-first (LPT) on the
estimated cell count of each point, the estimate the library's early routing
uses on the device: pi nbin^2 max(|A_ps|, 1), with A_ps the point-source
magnification.  The estimate only decides where a point runs, never its
result.

Two ways to use it:

* ``binary_mag_multi_device(points, settings, devices)``: one process, one
  host thread and one library context per device, results gathered in input
  order on the host;
* ``rank_share`` and ``gather_results`` for one process per GPU under
  ``torch.distributed``: every rank computes the same deterministic partition
  from the same inputs (no communication), integrates its share, and one
  all-gather of the fixed-size result records puts the whole batch on every
  rank.
"""
from __future__ import annotations

import threading

import numpy as np

from . import _lib
from .api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs

_MODEL_DTYPE = np.dtype([("s", "f8"), ("q", "f8"), ("bins", "i4"), ("r", "i4")])


def lpt_partition(costs, n_parts: int) -> list[np.ndarray]:
    """Longest-processing-time-first split of items with the given costs into
    n_parts lists of indices: items in decreasing cost (ties by index), each to
    the part with the least load so far (ties to the lowest part).  Every part
    lists its indices in increasing order.  Deterministic: the same costs give
    the same split on every rank."""
    costs = np.asarray(costs, dtype=np.float64).ravel()
    if n_parts < 1:
        raise ValueError("n_parts must be at least 1")
    if not np.all(np.isfinite(costs)) or np.any(costs < 0):
        raise ValueError("costs must be finite and non-negative")
    order = np.lexsort((np.arange(costs.size), -costs))
    load = np.zeros(n_parts)
    owner = np.empty(costs.size, dtype=np.int64)
    for i in order:
        p = int(np.argmin(load))  # the first of the least-loaded parts
        owner[i] = p
        load[p] += costs[i]
    return [np.nonzero(owner == p)[0] for p in range(n_parts)]


def point_costs(points, settings_list, a_ps=None) -> np.ndarray:
    """Estimated lattice cells of each point: pi nbin^2 max(|A_ps|, 1), nbin the
    point's settings' source_bins.  a_ps (the point-source magnifications) is
    computed on device 0 when not given."""
    pts = np.ascontiguousarray(points, dtype=FS_POINT_DTYPE)
    if a_ps is None:
        from . import binary_mag0_batch
        a_ps = binary_mag0_batch(pts["s"], pts["q"], pts["y1"], pts["y2"]) if pts.size else np.zeros(0)
    bins = np.array([max(int(st.source_bins), 1) for st in settings_list], dtype=np.float64)
    nb = bins[pts["settings"]]
    return np.pi * nb * nb * np.maximum(np.abs(np.asarray(a_ps, dtype=np.float64)), 1.0)


def _run_share(device, points, settings_list, models, out, idx, errors):
    try:
        ctx = _lib.Context(device)
        try:
            sub = np.ascontiguousarray(points[idx])
            res = np.zeros(sub.size, dtype=FS_RESULT_DTYPE)
            if sub.size:
                st = (LcbiStructs.FsSettings * len(settings_list))(*settings_list)
                mptr, nm, flags = None, 0, 0
                if models is not None:
                    mptr, nm, flags = models.ctypes.data, len(models), 2
                rc = ctx._L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings_list), mptr, nm, sub.size,
                                                sub.ctypes.data, res.ctypes.data, flags)
                ctx.check(rc, f"lcbi_gpu_binary_mag on device {device}")
            out[idx] = res
        finally:
            ctx.close()
    except Exception as e:  # re-raised on the calling thread
        errors.append(e)


def binary_mag_multi_device(points, settings_list, devices, *, models=None, costs=None):
    """lcbinint_b200.binary_mag over several devices: the batch is split by
    LPT on the estimated cell counts (costs, else point_costs), every share
    runs on its device through its own context on its own host thread, and
    the results come back in input order.  Same results as one device."""
    pts = np.ascontiguousarray(points, dtype=FS_POINT_DTYPE)
    devices = list(devices)
    if not devices:
        raise ValueError("devices must name at least one device")
    md = None if models is None else np.ascontiguousarray(models, dtype=_MODEL_DTYPE)
    out = np.zeros(pts.size, dtype=FS_RESULT_DTYPE)
    if pts.size == 0:
        return out
    if costs is None:
        costs = point_costs(pts, settings_list)
    parts = lpt_partition(costs, len(devices))
    errors: list[Exception] = []
    threads = [threading.Thread(target=_run_share, args=(d, pts, settings_list, md, out, idx, errors))
               for d, idx in zip(devices, parts)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return out


def rank_share(costs, rank: int, world: int) -> np.ndarray:
    """This rank's indices of the LPT partition over `world` ranks."""
    return lpt_partition(costs, world)[rank]


def gather_results(local_results, parts, n: int, group=None, device=None) -> np.ndarray:
    """All-gather of the ranks' FS_RESULT_DTYPE records into one array in input
    order, on every rank.  parts[r] are rank r's input indices (lpt_partition);
    local_results are this rank's records in that order.  One collective: the
    records travel as bytes, padded to the largest share (NCCL needs device
    tensors: pass the rank's device; gloo works on the host)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    rec = FS_RESULT_DTYPE.itemsize
    width = max(max(len(p) for p in parts), 1) * rec
    local = np.ascontiguousarray(local_results, dtype=FS_RESULT_DTYPE)
    if local.size != len(parts[rank]):
        raise ValueError("local_results must hold this rank's share")
    buf = np.zeros(width, dtype=np.uint8)
    buf[: local.nbytes] = local.view(np.uint8)
    t = torch.from_numpy(buf)
    if device is not None:
        t = t.to(device)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    full = np.zeros(n, dtype=FS_RESULT_DTYPE)
    for r, o in enumerate(outs):
        k = len(parts[r])
        if k:
            full[parts[r]] = o.cpu().numpy()[: k * rec].view(FS_RESULT_DTYPE)
    return full


__all__ = ["lpt_partition", "point_costs", "binary_mag_multi_device", "rank_share", "gather_results"]
