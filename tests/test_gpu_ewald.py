"""The GPU FP64 Ewald reciprocal sum (gse_ewald_recip) against the CPU
restatement of CpuEwaldRecip, which the CPU tests pin to the reference's own
build and known answer."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,L,kcut", [(2, 20.0, 32), (64, 16.0, 12), (3000, 31.0, 18)])
def test_gpu_ewald_matches_oracle(n, L, kcut):
    import oracle
    from gse_b200 import workloads as W
    from gse_b200.gse import ewald_recip
    if n == 2:
        xyzq = W.reference_pair(1.0)
    elif n == 64:
        xyzq = W.random_charges(64, L, 3)
    else:
        xyzq = W.triplets(n, L, 9).astype(np.float64)
    e_ref, f_ref = oracle.ewald_recip(2.0, kcut, (L, L, L), xyzq)
    e, f = ewald_recip(2.0, kcut, (L, L, L), xyzq)
    assert abs(e - e_ref) <= 1e-11 * abs(e_ref)
    assert oracle.force_rms(f, f_ref) <= 1e-11


def test_gse_method_error_against_ewald():
    """FP64 GSE-k against converged Ewald at the 23,559-charge water box: the
    method error the reference's parameters give (reported, loosely bounded)."""
    import oracle
    from gse_b200 import workloads as W
    from gse_b200.gse import ewald_kcut, ewald_recip
    s = W.config_water_23k()
    x = s.xyzq.astype(np.float64)
    e_gse, f_gse = oracle.gsek_forward(s.grid, s.boxes, s.sigma, x)
    e_ew, f_ew = ewald_recip(s.sigma, ewald_kcut(s.sigma, s.boxes), s.boxes, x)
    frms = oracle.force_rms(f_gse, f_ew)
    erel = abs(e_gse - e_ew) / abs(e_ew)
    print("GSE-k (FP64) vs Ewald: force rms", frms, "energy rel", erel)
    assert frms < 1e-2 and erel < 1e-2


# ---- direct sum (gse_ewald_direct) -----------------------------------------

def shuffled_images(xyzq, box, seed):
    """Some atoms moved by whole box vectors: the minimum image must not care."""
    x = np.array(xyzq, dtype=np.float64)
    rng = np.random.default_rng(seed)
    k = rng.integers(-2, 3, size=(x.shape[0], 3))
    k[rng.uniform(size=x.shape[0]) < 0.5] = 0
    x[:, :3] += k * np.array(box)
    return x


DIRECT_CASES = [
    # name, n, box, rcut, exclusions, images: cells per axis from 1 to 4
    ("pair", 2, (20.0, 20.0, 20.0), 9.0, False, False),
    ("odd300_2cells", 300, (14.0, 13.0, 15.0), 6.0, True, False),
    ("water3000_3cells", 3000, (31.0, 31.0, 31.0), 9.0, True, True),
    ("water6000_ortho", 6000, (40.0, 31.0, 19.0), 9.0, True, False),
    ("random64_1cell", 64, (16.0, 16.0, 16.0), 12.0, False, True),
]


@pytest.mark.parametrize("case", DIRECT_CASES, ids=[c[0] for c in DIRECT_CASES])
def test_gpu_ewald_direct_matches_oracle(case):
    import oracle
    from gse_b200 import workloads as W
    from gse_b200.gse import ewald_direct
    from test_oracle import odd_exclusions
    name, n, box, rcut, excl, images = case
    if n == 2:
        xyzq = W.reference_pair(1.0) + np.array([10.0, 10.0, 10.0, 0.0])
    elif n == 64:
        xyzq = W.random_charges(64, box[0], 3)
    else:
        b = np.array(box) / box[0]
        xyzq = W.triplets(n, box[0], 9).astype(np.float64) * np.array(list(b) + [1.0])
    if images:
        xyzq = shuffled_images(xyzq, box, 4)
    ib = nb = None
    if excl:
        ib, nb = odd_exclusions(n) if n == 300 else W.triplet_exclusions(n)
    e_ref, f_ref = oracle.ewald_direct(2.0, rcut, box, xyzq, iblo14=ib, inb14=nb)
    e, f = ewald_direct(2.0, rcut, box, xyzq, ib, nb)
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref), (e, e_ref)
    assert oracle.force_rms(f, f_ref) <= 1e-12
    e2, f2 = ewald_direct(2.0, rcut, box, xyzq, ib, nb)
    assert e2 == e and np.array_equal(f2, f)  # independent of block scheduling


def test_gpu_ewald_direct_class_and_device_buffers():
    """The CpuEwaldDirect mirror (setupExclusions + calcForceEnergy), device
    arrays through the C ABI, and the empty, single-charge and no-force cases."""
    import ctypes
    import torch
    import oracle
    from gse_b200 import _lib, workloads as W
    from gse_b200.gse import CpuEwaldDirect, check, ewald_direct
    n, box = 1500, (25.0, 25.0, 25.0)
    xyzq = W.triplets(n, 25.0, 2).astype(np.float64)
    ib, nb = W.triplet_exclusions(n)
    d = CpuEwaldDirect(2.0, 8.0, *box)
    d.setupExclusions(n, ib, nb)
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    e = d.calcForceEnergy(n, xyzq, fx, fy, fz)
    e_ref, f_ref = oracle.ewald_direct(2.0, 8.0, box, xyzq, iblo14=ib, inb14=nb)
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref)
    assert oracle.force_rms(np.stack([fx, fy, fz], 1), f_ref) <= 1e-12
    # device buffers
    L = _lib.load()
    xd = torch.from_numpy(xyzq).cuda()
    fd = torch.zeros((3, n), dtype=torch.float64, device="cuda")
    ed = ctypes.c_double()
    check(L.gse_ewald_direct(0, None, 2.0, 8.0, *box, oracle.CCELEC, n, xd.data_ptr(), n,
                             ib.ctypes.data, nb.ctypes.data, ctypes.addressof(ed),
                             fd[0].data_ptr(), fd[1].data_ptr(), fd[2].data_ptr()))
    assert ed.value == e
    assert np.array_equal(fd.cpu().numpy().T, np.stack([fx, fy, fz], 1))
    e_nf, f_nf = ewald_direct(2.0, 8.0, box, xyzq, ib, nb, forces=False)
    assert e_nf == e and f_nf is None
    assert ewald_direct(2.0, 8.0, box, np.zeros((0, 4)))[0] == 0.0
    e1, f1 = ewald_direct(2.0, 8.0, box, [[1.0, 2.0, 3.0, -0.834]])
    assert abs(e1 - oracle.ewald_direct(2.0, 8.0, box, [[1.0, 2.0, 3.0, -0.834]])[0]) <= 1e-13
    assert np.array_equal(f1, np.zeros((1, 3)))


def test_gpu_ewald_direct_argument_errors():
    from gse_b200._lib import GseError
    from gse_b200.gse import ewald_direct
    x = np.zeros((4, 4))
    with pytest.raises(GseError) as ei:  # one iblo14 entry per atom
        ewald_direct(2.0, 8.0, (10.0, 10.0, 10.0), x, np.array([0, 0, 0]), np.array([0]))
    assert ei.value.status == 1
    with pytest.raises(GseError):  # decreasing cumulative ends
        ewald_direct(2.0, 8.0, (10.0, 10.0, 10.0), x, np.array([1, 0, 1, 1]), np.array([2]))
    for bad in ((0.0, 8.0), (2.0, 0.0), (2.0, float("nan"))):
        with pytest.raises(GseError):
            ewald_direct(bad[0], bad[1], (10.0, 10.0, 10.0), x)


def test_ewald_total_independent_of_splitting_width():
    """Physics check of direct + reciprocal together: with both sums
    converged (erfc(rcut / sqrt2 sigma) < 1e-13, exp(-sigma^2 k^2 / 2) below
    1e-14 at kcut) the total Coulomb energy and forces of a neutral periodic
    system do not depend on the width sigma that splits them."""
    import oracle
    from gse_b200 import workloads as W
    from gse_b200.gse import ewald_direct, ewald_kcut, ewald_recip
    L = 31.0
    x = W.triplets(3000, L, 11).astype(np.float64)
    tot = []
    for sigma in (1.5, 2.0):
        ed, fd = ewald_direct(sigma, 15.4, (L, L, L), x)
        er, fr = ewald_recip(sigma, ewald_kcut(sigma, (L, L, L), 1e-14), (L, L, L), x)
        tot.append((ed + er, fd - fr))  # direct: gradient; reciprocal: force
    (e1, f1), (e2, f2) = tot
    assert abs(e1 - e2) <= 1e-9 * abs(e1), (e1, e2)
    assert oracle.force_rms(f2, f1) <= 1e-8


def test_gpu_ewald_direct_full_size_properties():
    """At the 262,143-charge water box (L 140, rcut 9, water exclusions):
    the forces sum to zero (every pair term enters its two atoms with opposite
    signs), repeated calls agree bit for bit, and moving every atom by whole
    box vectors or translating the system changes the result only by
    rounding."""
    from gse_b200 import workloads as W
    from gse_b200.gse import ewald_direct
    s = W.config_water_262k()
    x = s.xyzq.astype(np.float64)
    box = s.boxes
    ib, nb = W.triplet_exclusions(x.shape[0])
    e, f = ewald_direct(2.0, 9.0, box, x, ib, nb)
    e2, f2 = ewald_direct(2.0, 9.0, box, x, ib, nb)
    assert e == e2 and np.array_equal(f, f2)
    assert np.abs(f.sum(axis=0)).max() <= 1e-10 * np.abs(f).sum()
    e3, f3 = ewald_direct(2.0, 9.0, box, shuffled_images(x, box, 5), ib, nb)
    xt = x.copy()
    xt[:, :3] += np.array([0.37, -5.1, 70.3])
    e4, f4 = ewald_direct(2.0, 9.0, box, xt, ib, nb)
    fs = np.sqrt((f * f).sum())
    for ee, ff in ((e3, f3), (e4, f4)):
        assert abs(ee - e) <= 1e-11 * abs(e)
        assert np.sqrt(((ff - f) ** 2).sum()) <= 1e-10 * fs
