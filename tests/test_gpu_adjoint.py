"""Reverse mode: gse_adjoint (through the C ABI) against central finite
differences of the FP64 forward (h = 1e-4), torch.autograd.gradcheck on a
tiny system, and the mixed form against the FP64 gradient.

The loss is L = gE E + sum_i G_i . F_i with gE = 1 and G ~ N(0, 1).  The
spherical cut of the force gather is not differentiable where a grid point
crosses the sphere; finite-difference probes whose +-h positions change the
atom's point set are skipped (the test checks that there are few)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_ctx(M, L, precision="fp64"):
    from gse_b200.gse import Context
    return Context(M, M, M, 2.0, 0.4, 3.0, 3.0, L, L, L, precision=precision)


def loss_and_grads(ctx, xyzq, G, gE=1.0):
    n = xyzq.shape[0]
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    E = ctx.forward(n, xyzq, fx, fy, fz)
    L = gE * E + float((G * np.stack([fx, fy, fz], 1)).sum())
    dq, dx, dy, dz = (np.zeros(n) for _ in range(4))
    ctx.adjoint(n, xyzq, gE, np.ascontiguousarray(G[:, 0]), np.ascontiguousarray(G[:, 1]),
                np.ascontiguousarray(G[:, 2]), dq, dx, dy, dz)
    return L, dq, np.stack([dx, dy, dz], 1)


def loss(ctx, xyzq, G, gE=1.0):
    n = xyzq.shape[0]
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    E = ctx.forward(n, xyzq, fx, fy, fz)
    return gE * E + float((G * np.stack([fx, fy, fz], 1)).sum())


def sphere_set(x, L, M, sigma1, rcut):
    """Grid offsets inside atom x's sphere (the gather's point set)."""
    h = L / M
    c = np.round(x / h).astype(int)
    n = int(math.ceil(rcut / h))
    t = np.arange(-n, n + 1)
    d = [x[k] - (c[k] + t) * h for k in range(3)]
    r2 = d[0][None, None, :] ** 2 + d[1][None, :, None] ** 2 + d[2][:, None, None] ** 2
    return r2 < rcut * rcut


@pytest.mark.parametrize("n_atoms,L,M", [(300, 16.0, 16), (48000, 78.4, 80)])
def test_adjoint_matches_finite_differences(n_atoms, L, M):
    from gse_b200 import workloads as W
    import oracle
    xyzq = W.triplets(n_atoms, L, 7).astype(np.float64)
    rng = np.random.default_rng(1)
    G = rng.standard_normal((n_atoms, 3))
    ctx = make_ctx(M, L)
    L0, dq, dxyz = loss_and_grads(ctx, xyzq, G)
    s1, _, rc = oracle.gse_params(2.0)
    h = 1e-4
    atoms = rng.choice(n_atoms, size=8, replace=False)
    errs, skipped = [], 0
    for i in atoms:
        # charge derivative
        xp, xm = xyzq.copy(), xyzq.copy()
        xp[i, 3] += h
        xm[i, 3] -= h
        fd = (loss(ctx, xp, G) - loss(ctx, xm, G)) / (2 * h)
        errs.append(abs(fd - dq[i]) / max(abs(dq[i]), 1.0))
        for d in range(3):
            xp, xm = xyzq.copy(), xyzq.copy()
            xp[i, d] += h
            xm[i, d] -= h
            if not np.array_equal(sphere_set(xp[i, :3], L, M, s1, rc),
                                  sphere_set(xm[i, :3], L, M, s1, rc)):
                skipped += 1
                continue
            fd = (loss(ctx, xp, G) - loss(ctx, xm, G)) / (2 * h)
            errs.append(abs(fd - dxyz[i, d]) / max(abs(dxyz[i, d]), 1.0))
    print(n_atoms, "max rel FD error", max(errs), "skipped", skipped)
    assert skipped <= 4
    assert max(errs) < 1e-4


def test_mixed_gradient_matches_fp64():
    from gse_b200 import workloads as W
    xyzq = W.triplets(48000, 78.4, 7)
    rng = np.random.default_rng(1)
    G = rng.standard_normal((48000, 3))
    _, dq64, dx64 = loss_and_grads(make_ctx(80, 78.4, "fp64"), xyzq.astype(np.float64), G)
    _, dqm, dxm = loss_and_grads(make_ctx(80, 78.4, "mixed"), xyzq.astype(np.float32), G)
    eq = np.sqrt(((dqm - dq64) ** 2).sum() / (dq64 ** 2).sum())
    ex = np.sqrt(((dxm - dx64) ** 2).sum() / (dx64 ** 2).sum())
    print("mixed vs fp64 gradient rel RMS: dq", eq, "dx", ex)
    assert eq < 1e-4 and ex < 1e-4


def test_energy_gradient_is_potential_and_cube_force():
    """gE = 1, no force gradients: dE/dq_i = c h^3 sum_cube g phi (the potential
    seen by atom i) -- E is quadratic in q, so sum_i q_i dE/dq_i = 2 E."""
    from gse_b200 import workloads as W
    xyzq = W.triplets(3000, 31.0, 3).astype(np.float64)
    ctx = make_ctx(32, 31.0)
    n = xyzq.shape[0]
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    E = ctx.forward(n, xyzq, fx, fy, fz)
    dq, dx, dy, dz = (np.zeros(n) for _ in range(4))
    ctx.adjoint(n, xyzq, 1.0, None, None, None, dq, dx, dy, dz)
    assert abs(float((xyzq[:, 3] * dq).sum()) - 2 * E) <= 1e-10 * abs(E)
    F = np.stack([fx, fy, fz], 1)
    Fc = -np.stack([dx, dy, dz], 1)
    # cube-spread force vs the sphere-cut force: the same up to the Gaussian tail
    assert np.sqrt(((Fc - F) ** 2).sum() / (F ** 2).sum()) < 2e-3


def test_torch_autograd_gradcheck():
    import torch
    from gse_b200.torch_binding import gse_energy_forces
    ctx = make_ctx(12, 11.0)
    rng = np.random.default_rng(4)
    xyz = torch.tensor(rng.uniform(0, 11.0, (4, 3)), dtype=torch.float64, device="cuda",
                       requires_grad=True)
    q = torch.tensor([0.8, -0.5, -0.4, 0.1], dtype=torch.float64, device="cuda",
                     requires_grad=True)

    def f(a, b):
        E, F = gse_energy_forces(a, b, ctx)
        return E, F

    assert torch.autograd.gradcheck(f, (xyz, q), eps=1e-6, atol=1e-5, rtol=1e-4)


def test_mixed_adjoint_is_deterministic_and_consistent():
    """The mixed reverse pass accumulates its source in 64-bit fixed point and
    sums per atom in a fixed order: two runs give the same bits.  With gE = 1
    and no force gradients, sum_i q_i dE/dq_i = 2 E holds to FP32 accuracy."""
    from gse_b200 import workloads as W
    xyzq = W.triplets(48000, 78.4, 7).astype(np.float32)
    rng = np.random.default_rng(2)
    G = rng.standard_normal((48000, 3))
    ctx = make_ctx(80, 78.4, "mixed")
    _, dq1, dx1 = loss_and_grads(ctx, xyzq, G)
    _, dq2, dx2 = loss_and_grads(ctx, xyzq, G)
    assert np.array_equal(dq1, dq2) and np.array_equal(dx1, dx2)
    n = xyzq.shape[0]
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    E = ctx.forward(n, xyzq, fx, fy, fz)
    dq, dx, dy, dz = (np.zeros(n) for _ in range(4))
    ctx.adjoint(n, xyzq, 1.0, None, None, None, dq, dx, dy, dz)
    assert abs(float((xyzq[:, 3].astype(np.float64) * dq).sum()) - 2 * E) <= 1e-5 * abs(E)
