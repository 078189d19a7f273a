"""Edge cases of the CUDA path against the oracle (the C restatement of the
reference, itself pinned to the compiled reference in test_oracle.py).

FP64 within 1e-12 relative (forces RMS, energy), mixed within 1e-5 of the FP64
oracle.  Cases: positions outside the box (negative and beyond L, several box
lengths away), a single charge, zero atoms, all charges in one cell, zero
charges, a large non-cubic grid, the smallest tiled grid, and stencils of
every supported width on the tiled path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5


def run(M, box, sigma, xyzq, precision):
    from gse_b200.gse import CpuGSEk
    ct = np.float64 if precision == "fp64" else np.float32
    x = np.ascontiguousarray(xyzq, dtype=ct).reshape(-1, 4)
    n = x.shape[0]
    g = CpuGSEk(M[0], M[1], M[2], sigma, 0.4, 3.0, 3.0, box[0], box[1], box[2],
                precision=precision)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    E = g.forward(n, x, fx, fy, fz)
    return E, np.stack([fx, fy, fz], 1)


def check(M, box, sigma, xyzq, tol64=FP64_TOL, tolm=MIXED_TOL):
    import oracle
    E0, F0 = oracle.gsek_forward(M, box, sigma, np.asarray(xyzq, np.float64))
    for precision, tol in (("fp64", tol64), ("mixed", tolm)):
        E, F = run(M, box, sigma, xyzq, precision)
        if np.abs(F0).sum() > 0:
            assert oracle.force_rms(F, F0) <= tol, (precision, oracle.force_rms(F, F0))
        else:
            assert np.abs(F).max() == 0.0
        if E0 != 0.0:
            assert abs(E - E0) <= tol * abs(E0), (precision, E, E0)
        else:
            assert abs(E) <= 1e-30


def waters(n, L, seed):
    from gse_b200 import workloads as W
    return W.triplets(n, L, seed).astype(np.float64)


def test_positions_outside_the_box():
    """The reference wraps grid indices, not positions: atoms anywhere in space
    spread and gather with their periodic images' grid points."""
    L, M = 18.0, 18
    x = waters(300, L, 11)
    rng = np.random.default_rng(3)
    shift = rng.integers(-3, 4, size=(300, 3)) * L
    x[:, :3] += shift
    x[:5, :3] -= 0.5 * L  # a few straddling the faces
    check((M, M, M), (L, L, L), 2.0, x)


def test_single_charge_and_empty_system():
    """The mesh force of an isolated charge on itself is a lattice residue that
    cancels to ~1e-3 of the force between two unit charges 1 A apart, so it is
    compared against that pair force: FP64 within 1e-12, mixed within 1e-5."""
    import oracle
    M, box = (16, 16, 16), (16.0, 16.0, 16.0)
    one = np.array([[3.3, 7.1, 12.9, 1.0]])
    pair = np.array([[3.3, 7.1, 12.9, 1.0], [4.3, 7.1, 12.9, -1.0]])
    _, Fp = oracle.gsek_forward(M, box, 2.0, pair)
    scale = float(np.abs(Fp).max())
    E0, F0 = oracle.gsek_forward(M, box, 2.0, one)
    for precision, tol in (("fp64", FP64_TOL), ("mixed", MIXED_TOL)):
        E, F = run(M, box, 2.0, one, precision)
        assert np.abs(F - F0).max() <= tol * scale, (precision, np.abs(F - F0).max() / scale)
        assert abs(E - E0) <= tol * abs(E0)
    E, F = run((16, 16, 16), (16.0, 16.0, 16.0), 2.0, np.zeros((0, 4)), "fp64")
    assert E == 0.0 and F.shape == (0, 3)
    E, F = run((16, 16, 16), (16.0, 16.0, 16.0), 2.0, np.zeros((0, 4)), "mixed")
    assert E == 0.0 and F.shape == (0, 3)


def test_all_charges_in_one_cell_and_zero_charges():
    rng = np.random.default_rng(5)
    x = np.zeros((200, 4))
    x[:, :3] = 8.0 + rng.uniform(-0.2, 0.2, (200, 3))
    x[:, 3] = rng.choice([-1.0, 1.0], 200)
    check((16, 16, 16), (16.0, 16.0, 16.0), 2.0, x, tolm=2e-5)
    x[:, 3] = 0.0
    check((16, 16, 16), (16.0, 16.0, 16.0), 2.0, x)


@pytest.mark.parametrize("M,box", [((10, 11, 12), (10.0, 11.0, 12.0)),
                                   ((96, 80, 112), (93.0, 77.0, 108.0))])
def test_small_and_large_noncubic_grids(M, box):
    rng = np.random.default_rng(8)
    n = 600 if M[0] < 20 else 30000
    x = waters(n, box[0], 9)
    x[:, :3] *= np.array(box) / box[0]
    x[:, :3] += rng.uniform(0, 1e-3, (n, 3))
    check(M, box, 2.0, x)


@pytest.mark.parametrize("h", [1.45, 1.2, 1.0, 0.86])
def test_every_tiled_stencil_width(h):
    """rcut1 = 5.367 for sigma 2: h sets n = ceil(rcut/h) to 4, 5, 6, 7 --
    stencil widths 9, 11, 13 and 15 on the tiled path."""
    M = 24
    L = M * h
    x = waters(900, L, 12)
    check((M, M, M), (L, L, L), 2.0, x)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonfinite_input_is_reported(precision):
    """A NaN or infinite position or charge makes the call that reads it return
    GSE_ERR_NONFINITE when its outputs are host memory, or the next
    gse_synchronize when they are device memory; later calls work again."""
    import torch
    from gse_b200._lib import GseError
    from gse_b200.gse import Context
    L, M = 24.0, 24
    x = waters(900, L, 12)
    ctx = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, L, L, L, precision=precision)
    ct = np.float64 if precision == "fp64" else np.float32
    n = x.shape[0]
    f = [np.zeros(n) for _ in range(3)]
    bad = x.copy()
    bad[17, 1] = np.nan
    with pytest.raises(GseError) as ei:
        ctx.forward(n, bad.astype(ct), *f)
    assert ei.value.status == 8
    E = ctx.forward(n, x.astype(ct), *f)  # works again
    assert np.isfinite(E)
    bad[17, 1] = 1.0
    bad[3, 3] = np.inf
    xd = torch.from_numpy(bad.astype(ct)).cuda()
    fd = torch.zeros(3, n, dtype=torch.float64, device="cuda")
    ed = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.forward(n, xd, fd[0], fd[1], fd[2], energy_out=ed)  # asynchronous: no status yet
    with pytest.raises(GseError) as ei:
        ctx.synchronize()
    assert ei.value.status == 8
    ctx.synchronize()  # reported once


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_misaligned_device_pointers_are_refused_on_the_host(precision):
    """Device pointers that a kernel would read or write in place must be
    aligned to the width it accesses them with: position records 16 (mixed)
    or 32 (FP64) bytes, forces 8 bytes, spectra 16 bytes.  A view a few bytes
    into an allocation is refused with GSE_ERR_INVALID_ARG before any work is
    queued, and the context stays usable."""
    import ctypes
    import torch
    from gse_b200 import _lib
    from gse_b200.gse import Context
    L = _lib.load()
    M, box, n = 16, 16.0, 30
    ctx = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, box, box, box, precision=precision)
    dt = torch.float32 if precision == "mixed" else torch.float64
    rec = 16 if precision == "mixed" else 32
    from gse_b200 import workloads as W
    x = torch.zeros(4 * n + 8, dtype=dt, device="cuda")
    x[:4 * n] = torch.from_numpy(W.triplets(n, box, 3).reshape(-1)).to(dt)
    f = torch.zeros(3, n + 1, dtype=torch.float64, device="cuda")
    e = ctypes.c_double()
    h = ctx.h

    def status(call):
        st = call()
        return st, L.gse_last_error().decode()

    off = x.element_size()  # one element in: 4 or 8 bytes
    st, msg = status(lambda: L.gse_forward(h, n, x.data_ptr() + off, ctypes.addressof(e),
                                           f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr()))
    assert st == 1 and f"{rec}-byte aligned" in msg, msg
    st, msg = status(lambda: L.gse_spread_charge(h, n, x.data_ptr() + off))
    assert st == 1 and "xyzq" in msg, msg
    st, msg = status(lambda: L.gse_forward(h, n, x.data_ptr(), ctypes.addressof(e),
                                           f[0].data_ptr() + 4, f[1].data_ptr(),
                                           f[2].data_ptr()))
    assert st == 1 and "8-byte aligned" in msg, msg
    k = torch.zeros(2 * (M // 2 + 1) * M * M + 4, dtype=dt, device="cuda")
    st, msg = status(lambda: L.gse_green_mul(h, 2.0, box, box, box, k.data_ptr() + 4))
    assert st == 1 and "16-byte aligned" in msg, msg
    # aligned pointers still work on the same context
    st = L.gse_forward(h, n, x.data_ptr(), ctypes.addressof(e), f[0].data_ptr(),
                       f[1].data_ptr(), f[2].data_ptr())
    assert st == 0, L.gse_last_error().decode()
    torch.cuda.synchronize()
    assert np.isfinite(e.value) and torch.isfinite(f).all()
    ctx.close()


def test_ewald_refuses_misaligned_device_records():
    import torch
    from gse_b200 import _lib
    import ctypes
    L = _lib.load()
    x = torch.zeros(4 * 10 + 4, dtype=torch.float64, device="cuda")
    e = ctypes.c_double()
    st = L.gse_ewald_recip(0, None, 2.0, 8, 10.0, 10.0, 10.0, 332.0716, 10, x.data_ptr() + 16,
                           ctypes.addressof(e), None, None, None)
    assert st == 1 and "32-byte aligned" in L.gse_last_error().decode()
    st = L.gse_ewald_direct(0, None, 2.0, 4.0, 10.0, 10.0, 10.0, 332.0716, 10,
                            x.data_ptr() + 8, 0, None, None, ctypes.addressof(e), None, None,
                            None)
    assert st == 1 and "32-byte aligned" in L.gse_last_error().decode()


def test_mixed_range_overflow_is_reported():
    """The mixed form accumulates each 16^3-cell brick in an int32 tile at a
    power-of-two scale; a charge so large that even the coarsest scale leaves
    no headroom (one charge above ~6.5e4 e at sigma1 1.26) makes the call
    return GSE_ERR_RANGE instead of a wrapped grid.  The FP64 form has no such
    limit, and the mixed context works again afterwards."""
    from gse_b200._lib import GseError
    from gse_b200.gse import Context
    L, M = 24.0, 24
    x = waters(900, L, 12)
    n = x.shape[0]
    f = [np.zeros(n) for _ in range(3)]
    big = x.copy()
    big[10, 3] = 1.0e5
    ctx = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, L, L, L, precision="mixed")
    with pytest.raises(GseError) as ei:
        ctx.forward(n, big.astype(np.float32), *f)
    assert ei.value.status == 9 and "fixed-point range" in str(ei.value)
    E = ctx.forward(n, x.astype(np.float32), *f)
    assert np.isfinite(E)
    c64 = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, L, L, L, precision="fp64")
    assert np.isfinite(c64.forward(n, big, *f))


def test_staged_copy_wait_that_runs_out_is_reported(monkeypatch):
    """The FFT's staged plane copies are awaited with a bounded wait.  With
    GSE_B200_TEST_FFT_STALL=1 at context creation the forward plane pass
    expects 16 bytes more than its first copy brings (every copy still
    completes), so its first wait runs out after about a millisecond: the
    CTAs set the stall flag and return, and the call reports
    GSE_ERR_TIMEOUT.  The GPU stays usable: a context made afterwards
    without the variable evaluates normally."""
    from gse_b200 import GseError
    from gse_b200 import workloads as W
    from gse_b200.gse import Context
    M, L = 64, 62.0
    x = W.triplets(600, L, 5).astype(np.float32)
    n = x.shape[0]
    monkeypatch.setenv("GSE_B200_TEST_FFT_STALL", "1")
    a = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, L, L, L, precision="mixed")
    assert a.paths() & 8
    f = [np.zeros(n) for _ in range(3)]
    with pytest.raises(GseError) as ei:
        a.forward(n, x, *f)
    assert ei.value.name == "GSE_ERR_TIMEOUT"
    a.close()
    monkeypatch.delenv("GSE_B200_TEST_FFT_STALL")
    b = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, L, L, L, precision="mixed")
    g = [np.zeros(n) for _ in range(3)]
    E = b.forward(n, x, *g)
    c = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, L, L, L, precision="mixed")
    h = [np.zeros(n) for _ in range(3)]
    assert c.forward(n, x, *h) == E
    assert all(np.array_equal(u, v) for u, v in zip(g, h))
    b.close()
    c.close()
