"""GPU parity tests of the point-source path (C ABI lcbi_gpu_binary_mag0*).

Bar: bit-exact against the oracle restatement (itself bit-exact against the
reference compiled from source), which is stricter than the 1e-10 relative
tolerance the reference's own tests apply (tests/regression/test_vbm_consistency.py:232-255).
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # point-source tolerance stated for this path


def _cfg2_points(n, seed):
    rng = np.random.default_rng(seed)
    y = rng.uniform(-1.5, 1.5, (n, 2))
    s = np.exp(rng.uniform(np.log(0.3), np.log(3.0), n))
    q = np.exp(rng.uniform(np.log(1e-5), 0.0, n))
    return s, q, y[:, 0], y[:, 1]


def test_known_answers():
    import lcbinint_b200 as lb
    from tests.test_oracle_golden import BINARY_POINT_CASES
    for s, q, y1, y2, expected in BINARY_POINT_CASES:
        assert math.isclose(lb.binary_mag0(s, q, y1, y2), expected, rel_tol=REL_TOL, abs_tol=1e-11)


def test_bit_exact_vs_golden_fixture(golden):
    import lcbinint_b200 as lb
    g = golden("point_source.npz")
    A, nimg = lb.binary_mag0_batch(g["s"], g["q"], g["y1"], g["y2"], return_images=True)
    assert np.array_equal(A.view(np.int64), g["A"].view(np.int64))
    assert np.array_equal(nimg, g["nimg"])


@pytest.mark.parametrize("seed,invert", [(0, False), (1, True)])
def test_bit_exact_vs_oracle(oracle_lib, seed, invert):
    import lcbinint_b200 as lb
    s, q, y1, y2 = _cfg2_points(100_000, seed)
    if invert:
        q = 1.0 / q
    A, nimg = lb.binary_mag0_batch(s, q, y1, y2, return_images=True)
    Ao, no = oracle_lib.binary_mag0(s, q, y1, y2)
    same = A.view(np.int64) == Ao.view(np.int64)
    assert same.all(), f"{(~same).sum()} mismatches; worst rel {np.max(np.abs(A / Ao - 1))}"
    assert np.array_equal(nimg, no)


def test_derivative_indicator_bit_exact(oracle_lib):
    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib
    s, q, y1, y2 = (np.ascontiguousarray(v) for v in _cfg2_points(50_000, 2))
    ctx = lb.context()
    n = s.size
    A = np.empty(n); nimg = np.empty(n, dtype=np.int32); ind = np.empty(n)
    rc = ctx._L.lcbi_gpu_binary_mag0_derivatives(ctx.handle, n, _lib.ptr(s), _lib.ptr(q), _lib.ptr(y1),
                                                 _lib.ptr(y2), _lib.ptr(A), _lib.ptr(nimg), _lib.ptr(ind), 0)
    ctx.check(rc, "derivatives")
    Ao, no, io = oracle_lib.binary_mag0_derivatives(s, q, y1, y2)
    assert np.array_equal(A.view(np.int64), Ao.view(np.int64))
    assert np.array_equal(ind.view(np.int64), io.view(np.int64))


def test_edge_cases(oracle_lib):
    import lcbinint_b200 as lb
    # zero separation / non-positive q return 0 like the reference (point_source_magnifier.cpp:658-660)
    assert lb.binary_mag0(0.0, 0.5, 0.1, 0.1) == 0.0
    assert lb.binary_mag0(1.0, 0.0, 0.1, 0.1) == 0.0
    assert lb.binary_mag0(1.0, -1.0, 0.1, 0.1) == 0.0
    # equal masses, q exactly 1, far source
    a = lb.binary_mag0(1.0, 1.0, 3.0, -2.0)
    b = oracle_lib.binary_mag0([1.0], [1.0], [3.0], [-2.0])[0][0]
    assert a == b
    # source exactly on the lighter lens: reference never terminates; here NaN + status
    s, q = 1.5, 0.5
    x = -((-s) * (1.0 / (1.0 + q)))
    A = lb.binary_mag0_batch([s], [q], [x], [0.0])
    assert np.isnan(A[0])
    # empty batch
    assert lb.binary_mag0_batch(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0)).size == 0


def test_full_size_properties():
    """1e6 points (the point-source batch size): finite, image counts 3/5, and the
    reflection symmetry A(y1, y2) == A(y1, -y2) of the binary lens."""
    import lcbinint_b200 as lb
    s, q, y1, y2 = _cfg2_points(1_000_000, 7)
    A, n = lb.binary_mag0_batch(s, q, y1, y2, return_images=True)
    assert np.isfinite(A).all()
    assert np.isin(n, (3, 5)).all()
    assert (A >= 1.0 - 1e-12).all()
    B = lb.binary_mag0_batch(s, q, y1, -y2)
    assert np.max(np.abs(A / B - 1.0)) < 1e-9


@pytest.mark.parametrize("pinned", [False, True])
def test_host_batch_pipeline_matches_device_pointers(oracle_lib, pinned):
    """Host-memory batches of two or more 262,144-position chunks run chunk by
    chunk on three streams (copies beside kernels); magnifications, image
    counts and statuses must be the bytes of one device-pointer launch, and a
    sample must match the oracle.  700,001 positions: two full chunks and a
    ragged third, with degenerate positions (s = 0, q = 0, source on the
    lighter lens) spread through it."""
    import torch
    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib
    n = 700_001
    s, q, y1, y2 = (np.ascontiguousarray(v) for v in _cfg2_points(n, 7))
    s[::99_991] = 0.0
    q[5::123_457] = 0.0
    s[7], q[7], y2[7] = 1.5, 0.5, 0.0
    y1[7] = -((-s[7]) * (1.0 / (1.0 + q[7])))  # source exactly on the lighter lens: NaN, status 2
    ctx = lb.context()
    L = ctx._L
    host_in = [s, q, y1, y2]
    if pinned:
        host_in = [torch.from_numpy(a).pin_memory() for a in host_in]
        A = torch.empty(n, dtype=torch.float64).pin_memory()
        nimg = torch.empty(n, dtype=torch.int32).pin_memory()
        st = torch.empty(n, dtype=torch.int32).pin_memory()
        ptrs = [t.data_ptr() for t in host_in] + [A.data_ptr(), nimg.data_ptr(), st.data_ptr()]
    else:
        A = np.empty(n); nimg = np.empty(n, dtype=np.int32); st = np.empty(n, dtype=np.int32)
        ptrs = [_lib.ptr(a) for a in host_in] + [_lib.ptr(A), _lib.ptr(nimg), _lib.ptr(st)]
    ctx.check(L.lcbi_gpu_binary_mag0(ctx.handle, n, *ptrs, 0), "lcbi_gpu_binary_mag0 (host)")
    dev = [torch.from_numpy(a).cuda() for a in (s, q, y1, y2)]
    dA = torch.empty(n, dtype=torch.float64, device="cuda")
    dn = torch.empty(n, dtype=torch.int32, device="cuda")
    ds = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.check(L.lcbi_gpu_binary_mag0(ctx.handle, n, *[t.data_ptr() for t in dev], dA.data_ptr(), dn.data_ptr(),
                                     ds.data_ptr(), 1), "lcbi_gpu_binary_mag0 (device)")
    A, nimg, st = (np.asarray(v) for v in (A, nimg, st))
    assert A.view(np.int64).tobytes() == dA.cpu().numpy().view(np.int64).tobytes()
    assert np.array_equal(nimg, dn.cpu().numpy())
    assert np.array_equal(st, ds.cpu().numpy())
    assert st[7] == 2 and (st == 0).sum() == n - 1
    assert np.isnan(A[7]) and A[0] == 0.0 and A[5] == 0.0
    idx = np.random.default_rng(3).choice(n, 20_000, replace=False)
    idx = np.union1d(idx, [n - 1])
    idx = idx[(s[idx] != 0.0) & (q[idx] != 0.0) & (idx != 7)]
    Ao, no = oracle_lib.binary_mag0(s[idx], q[idx], y1[idx], y2[idx])
    assert np.array_equal(A[idx].view(np.int64), Ao.view(np.int64))
    assert np.array_equal(nimg[idx], no)
