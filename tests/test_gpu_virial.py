"""The reciprocal-space virial (gse_virial; the reference computes none, so
it is checked through the energy it differentiates):

- against the Ewald reciprocal virial of the same charges and total width
  sigma, W_ab = sum_k E_k (delta_ab - 2 k_a k_b (1/k^2 + sigma^2/2)), summed
  here in numpy over a converged k set (the GSE-k mesh energy matches the Ewald
  energy to ~1e-7 at these parameters, and so do its k-space terms);
- against central finite differences of the FP64 GSE energy under the diagonal
  strains x_a -> (1 + e) x_a, L_a -> (1 + e) L_a (orthorhombic boxes only, so no
  shear): W_aa = -dE/de.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CCELEC = 332.0716


def system():
    from gse_b200 import workloads as W
    L, M = 18.0, 20
    x = W.triplets(300, L, 7).astype(np.float64)
    return x, L, M


def ewald_virial(x, box, sigma):
    V = box[0] * box[1] * box[2]
    K = [int(np.ceil(np.sqrt(2.0 * 40.0) / sigma * b / (2 * np.pi))) for b in box]
    n = [np.arange(-k, k + 1) for k in K]
    kx, ky, kz = np.meshgrid(*(2 * np.pi * a / b for a, b in zip(n, box)), indexing="ij")
    k = np.stack([kx.ravel(), ky.ravel(), kz.ravel()], 1)
    k2 = (k * k).sum(1)
    k, k2 = k[k2 > 0], k2[k2 > 0]
    S = np.zeros(len(k), complex)
    for c0 in range(0, x.shape[0], 64):
        xs = x[c0:c0 + 64]
        S += (xs[:, 3][None, :] * np.exp(1j * (k @ xs[:, :3].T))).sum(1)
    Ek = 2 * np.pi / V * CCELEC * np.exp(-sigma * sigma * k2 / 2) / k2 * np.abs(S) ** 2
    c = 2 * (1 / k2 + sigma * sigma / 2)
    W = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            W[a, b] = (Ek * ((1.0 if a == b else 0.0) - c * k[:, a] * k[:, b])).sum()
    return Ek.sum(), np.array([W[0, 0], W[1, 1], W[2, 2], W[0, 1], W[0, 2], W[1, 2]])


def gse(x, box, M, precision):
    from gse_b200.gse import Context
    ctx = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, *box, precision=precision)
    xx = x.astype(np.float64 if precision == "fp64" else np.float32)
    n = x.shape[0]
    f = [np.zeros(n) for _ in range(3)]
    E = ctx.forward(n, xx, *f)
    return E, ctx.virial(), ctx


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_virial_matches_ewald(precision):
    x, L, M = system()
    E_ew, W_ew = ewald_virial(x, (L, L, L), 2.0)
    E, W, _ = gse(x, (L, L, L), M, precision)
    scale = np.abs(W_ew).max()
    print(precision, E, E_ew, W, W_ew, np.abs(W - W_ew).max() / scale)
    assert abs(E - E_ew) <= 1e-5 * abs(E_ew)
    assert np.abs(W - W_ew).max() <= 1e-4 * scale
    # the trace is -dE/d(ln V) of the energy: for the Gaussian-split form
    # sum_a W_aa = E - sigma^2 sum_k E_k k^2 - ..., nothing to check beyond Ewald


def test_virial_is_minus_strain_derivative_of_the_energy():
    x, L, M = system()
    _, W, _ = gse(x, (L, L, L), M, "fp64")
    eps = 1e-5
    fd = []
    for a in range(3):
        Es = []
        for sgn in (1, -1):
            s = np.ones(3)
            s[a] += sgn * eps
            xs = x.copy()
            xs[:, :3] *= s
            E, _, _ = gse(xs, tuple(L * s), M, "fp64")
            Es.append(E)
        fd.append(-(Es[0] - Es[1]) / (2 * eps))
    fd = np.array(fd)
    print(W[:3], fd, np.abs(W[:3] - fd).max() / np.abs(W[:3]).max())
    assert np.abs(W[:3] - fd).max() <= 1e-4 * np.abs(W[:3]).max()


def test_virial_is_deterministic_and_needs_a_spread():
    from gse_b200._lib import GseError
    from gse_b200.gse import Context
    x, L, M = system()
    _, W1, ctx = gse(x, (L, L, L), M, "mixed")
    assert np.array_equal(ctx.virial(), W1)
    fresh = Context(M, M, M, 2.0, 0.4, 3.0, 3.0, L, L, L, precision="mixed")
    with pytest.raises(GseError) as ei:
        fresh.virial()
    assert ei.value.status == 6
