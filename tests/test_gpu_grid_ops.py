"""The grid operations of CpuGaussCharge beside the force path on the GPU:
spreadChargeOnGrid (CpuGaussCharge.cpp:390-519), calcElectricFieldOnGrid
(:62-98) and calcDipoleSum (:188-226), in both calculation types.

The convolution and the field repeat the reference's operations in its order
with every product and sum rounded as it rounds them, so they must equal the
reference bit for bit (golden fixtures from the reference itself, and the
oracle restatement on grids too large for fixtures).  The dipole terms are the
reference's; their sum is a fixed tree, within 1e-12 of the sum of |terms|.
"""
import numpy as np
import pytest

from conftest import load_grid_goldens

pytestmark = pytest.mark.gpu

GRID_CASES = sorted(load_grid_goldens().keys())
PREC = [("fp64", "d", np.float64), ("mixed", "f", np.float32)]


def gauss(M, precision):
    from gse_b200.gse import CpuGaussCharge
    return CpuGaussCharge(M[0], M[1], M[2], precision=precision)


def grid(M, data, dtype):
    """A CpuGrid of M holding `data` (zeros for None)."""
    from gse_b200.gse import CpuGrid
    g = CpuGrid(M[0], M[1], M[2], dtype=dtype)
    if data is not None:
        g.data[...] = np.asarray(data, dtype).reshape(g.data.shape)
    return g


def dipole_scale(M, box, rho):
    """Sum of |terms| of the dipole sum, the scale of its rounding."""
    h = np.array(box, np.float64) / np.array(M)
    z, y, x = np.meshgrid(np.arange(M[2]), np.arange(M[1]), np.arange(M[0]), indexing="ij")
    v = np.abs(rho.astype(np.float64)) * h.prod()
    return np.array([(v * x * h[0]).sum(), (v * y * h[1]).sum(), (v * z * h[2]).sum()])


@pytest.mark.parametrize("case", GRID_CASES)
@pytest.mark.parametrize("precision,sfx,dt", PREC)
def test_grid_ops_equal_reference(grid_goldens, case, precision, sfx, dt):
    g = grid_goldens[case]
    M, box = tuple(int(v) for v in g["M"]), tuple(float(v) for v in g["box"])
    gc = gauss(M, precision)
    rho = grid(M, g["rho_" + sfx], dt)
    out = grid(M, None, dt)
    gc.spreadChargeOnGrid(float(g["sigma"]), float(g["rcut"]), *box, rho, out)
    assert np.array_equal(out.data.reshape(M[::-1]), g["rhoS_" + sfx])
    E = [grid(M, None, dt) for _ in range(3)]
    gc.calcElectricFieldOnGrid(*box, rho, *E)
    for e, k in zip(E, ("Ex_", "Ey_", "Ez_")):
        assert np.array_equal(e.data.reshape(M[::-1]), g[k + sfx])
    dip = np.array(gc.calcDipoleSum(*box, rho))
    ref = g["dip_" + sfx]
    scale = dipole_scale(M, box, g["rho_" + sfx])
    assert (np.abs(dip - ref) <= 1e-12 * scale).all(), (dip, ref)


@pytest.mark.parametrize("precision,sfx,dt", PREC)
def test_large_noncubic_grid_equals_oracle(precision, sfx, dt):
    """A 96 x 80 x 112 grid (n = 4 along x, 4 along y, 4 along z at sigma2 of
    sigma 2) through device buffers, against the restatement."""
    import torch
    import oracle
    from gse_b200.gse import Context
    M, box = (96, 80, 112), (93.0, 77.0, 108.0)
    s1, s2, _ = oracle.gse_params(2.0)
    rc2 = 3.0 * np.sqrt(2.0) * s2
    rng = np.random.default_rng(12)
    rho = rng.standard_normal(M[::-1]).astype(dt)
    ctx = Context(*M, 2.0, 0.4, 3.0, 3.0, *box, precision=precision)
    tdt = torch.float64 if dt == np.float64 else torch.float32
    x = torch.from_numpy(rho).cuda()
    out = torch.empty_like(x)
    ctx.gauss_spread_on_grid(s2, rc2, *box, x, out)
    want = oracle.spread_on_grid(M, box, s2, rc2, rho, dt)
    assert np.array_equal(out.cpu().numpy(), want)
    # in place on one device grid
    ctx.gauss_spread_on_grid(s2, rc2, *box, x, x)
    assert np.array_equal(x.cpu().numpy(), want)
    E = torch.empty((3,) + M[::-1], dtype=tdt, device="cuda")
    phi = torch.from_numpy(rho).cuda()
    ctx.gauss_efield_on_grid(*box, phi, E[0], E[1], E[2])
    for e, w in zip(E.cpu().numpy(), oracle.efield(M, box, rho, dt)):
        assert np.array_equal(e, w)
    dip = torch.zeros(3, dtype=torch.float64, device="cuda")
    ctx.gauss_dipole_sum(*box, phi, dip)
    ctx.synchronize()
    ref = oracle.dipole_sum(M, box, rho, dt)
    assert (np.abs(dip.cpu().numpy() - ref) <= 1e-12 * dipole_scale(M, box, rho)).all()


@pytest.mark.parametrize("sigma", [0.2, 0.45, 0.7, 0.9, 1.15, 1.4, 1.6, 1.85, 2.3])
@pytest.mark.parametrize("precision,dt", [("fp64", np.float64), ("mixed", np.float32)])
def test_every_tap_count_equals_oracle(sigma, precision, dt):
    """h = 1 and rcut = 3 sqrt(2) sigma give 2n + 1 = 3, 5, ..., 17 and 21 taps:
    the kernels specialised per tap count and the general one (3, 17, 21),
    wider than the 20-point axis at 21."""
    import oracle
    M = (24, 20, 28)
    box = tuple(float(m) for m in M)
    rcut = 3.0 * np.sqrt(2.0) * sigma
    rng = np.random.default_rng(int(sigma * 100))
    rho = rng.standard_normal(M[::-1]).astype(dt)
    gc = gauss(M, precision)
    out = grid(M, None, dt)
    gc.spreadChargeOnGrid(sigma, rcut, *box, grid(M, rho, dt), out)
    assert np.array_equal(out.data, oracle.spread_on_grid(M, box, sigma, rcut, rho, dt))


@pytest.mark.parametrize("precision,dt,tol", [("fp64", np.float64, 1e-12), ("mixed", np.float32, 1e-5)])
def test_convolution_total_is_input_total_times_tap_sums(precision, dt, tol):
    """A size-independent property at the benchmark grid (144^3, the GSE-r
    second spreading of sigma 2 on h = 0.972): a periodic convolution
    multiplies the grid total by the product of the three tap sums."""
    import torch
    import oracle
    from gse_b200.gse import Context
    M, box = (144, 144, 144), (140.0, 140.0, 140.0)
    _, s2, _ = oracle.gse_params(2.0)
    rc2 = 3.0 * np.sqrt(2.0) * s2
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.uniform(0.0, 1.0, M[::-1]).astype(dt)).cuda()
    out = torch.empty_like(x)
    ctx = Context(*M, 2.0, 0.4, 3.0, 3.0, *box, precision=precision)
    ctx.gauss_spread_on_grid(s2, rc2, *box, x, out)
    h = np.array(box) / np.array(M)
    prod = (2.0 * np.pi * s2 * s2) ** -1.5 * h.prod()
    for hd in h:
        n = int(np.ceil(rc2 / hd))
        i = np.arange(-n, n + 1)
        prod *= np.exp(-(hd * hd) * i * i / (2.0 * s2 * s2)).sum()
    tot_in = x.double().sum().item()
    tot_out = out.double().sum().item()
    assert abs(tot_out - tot_in * prod) <= tol * abs(tot_in * prod)


def test_grid_ops_argument_errors():
    from gse_b200._lib import GseError
    from gse_b200.gse import Context
    gc = gauss((16, 16, 16), "fp64")
    a, b = grid((16, 16, 16), None, np.float64), grid((16, 16, 8), None, np.float64)
    with pytest.raises(GseError):
        gc.spreadChargeOnGrid(1.0, 4.0, 16.0, 16.0, 16.0, a, b)
    with pytest.raises(GseError):
        gc.calcElectricFieldOnGrid(16.0, 16.0, 16.0, a, a, a, b)
    with pytest.raises(GseError):
        gc.calcDipoleSum(16.0, 16.0, 16.0, b)
    with pytest.raises(GseError) as ei:  # 2n + 1 = 81 > the widest supported stencil
        gc.spreadChargeOnGrid(1.0, 40.0, 16.0, 16.0, 16.0, a, a)
    assert ei.value.status == 2
    ctx = Context(16, 16, 16, 2.0, 0.4, 3.0, 3.0, 16.0, 16.0, 16.0)
    with pytest.raises(GseError) as ei:
        ctx.gauss_efield_on_grid(-1.0, 16.0, 16.0, a.data, a.data, a.data, a.data)
    assert ei.value.status == 1
