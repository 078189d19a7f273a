"""The CPU oracle, pinned: the C restatement against the reference's own
classes (golden fixtures made by tests/golden/make_goldens.py, and the
reference build in oracle/_ref when present), the project FFT against
numpy.fft, and the Ewald restatement against the reference's known answer."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_goldens, load_grid_goldens

CASES = sorted(load_goldens().keys())
GRID_CASES = sorted(load_grid_goldens().keys())


@pytest.mark.parametrize("shape", [(20, 20, 20), (16, 18, 20), (7, 9, 11), (5, 6, 9), (13, 1, 4),
                                   (64, 32, 48)])
def test_fft_matches_numpy(oracle_lib, shape):
    rng = np.random.default_rng(7)
    x = rng.standard_normal(shape)
    k = oracle_lib.fft_r2c(x)
    kn = np.fft.rfftn(x)
    assert np.abs(k - kn).max() <= 1e-14 * np.abs(kn).max()
    y = oracle_lib.fft_c2r(kn, shape[2])
    yn = np.fft.irfftn(kn, s=shape, axes=(0, 1, 2)) * np.prod(shape)
    assert np.abs(y - yn).max() <= 1e-14 * np.abs(yn).max()


@pytest.mark.parametrize("case", CASES)
def test_restatement_forward_equals_reference(oracle_lib, goldens, case):
    g = goldens[case]
    E, F, rho, phi = oracle_lib.gsek_forward(tuple(g["M"]), tuple(g["box"]), float(g["sigma"]),
                                             g["xyzq"], want_grids=True)
    # same operations in the same order: bit-identical to the reference
    assert np.array_equal(rho, g["rhoS"])
    assert np.array_equal(phi, g["phi"])
    assert np.array_equal(F, g["F"])
    assert E == float(g["E"])


@pytest.mark.parametrize("case", CASES)
def test_restatement_float_stages_equal_reference(oracle_lib, goldens, case):
    g = goldens[case]
    M, box, sigma = tuple(g["M"]), tuple(g["box"]), float(g["sigma"])
    s1, s2, rc = oracle_lib.gse_params(sigma)
    xf = g["xyzq"].astype(np.float32)
    rho_f = oracle_lib.spread(M, box, s1, rc, xf, dtype=np.float32)
    assert np.array_equal(rho_f, g["rho_f"])
    F = np.stack(oracle_lib.gather(M, box, s1, rc, xf, g["phi"].astype(np.float32),
                                   dtype=np.float32), axis=1)
    assert np.array_equal(F, g["F_f"])
    rho_n = oracle_lib.spread(M, box, s1, rc, g["xyzq"], normalize=True)
    assert np.array_equal(rho_n, g["rho_norm"])


@pytest.mark.parametrize("case", GRID_CASES)
@pytest.mark.parametrize("sfx,dt", [("d", np.float64), ("f", np.float32)])
def test_restatement_grid_ops_equal_reference(oracle_lib, grid_goldens, case, sfx, dt):
    """spreadChargeOnGrid, calcElectricFieldOnGrid and calcDipoleSum restated:
    the same operations in the same order, bit-identical to the reference."""
    g = grid_goldens[case]
    M, box = tuple(int(v) for v in g["M"]), tuple(float(v) for v in g["box"])
    rho = g["rho_" + sfx]
    assert rho.dtype == dt
    out = oracle_lib.spread_on_grid(M, box, float(g["sigma"]), float(g["rcut"]), rho, dt)
    assert np.array_equal(out, g["rhoS_" + sfx])
    E = oracle_lib.efield(M, box, rho, dt)
    for e, k in zip(E, ("Ex_", "Ey_", "Ez_")):
        assert np.array_equal(e, g[k + sfx])
    assert np.array_equal(oracle_lib.dipole_sum(M, box, rho, dt), g["dip_" + sfx])


def test_restatement_green_equals_reference(oracle_lib):
    if not oracle_lib.have_reference():
        pytest.skip("reference build not present")
    rng = np.random.default_rng(3)
    for M in [(16, 18, 20), (17, 17, 17), (20, 20, 20)]:
        k = (rng.standard_normal((M[2], M[1], M[0] // 2 + 1)) +
             1j * rng.standard_normal((M[2], M[1], M[0] // 2 + 1)))
        a = oracle_lib.green_mul(M, (15.0, 16.0, 17.0), 0.9, k)
        b = oracle_lib.ref_green_mul(M, (15.0, 16.0, 17.0), 0.9, k)
        assert np.array_equal(a, b)


def test_water_23559_golden(oracle_lib):
    from gse_b200 import workloads as W
    z = np.load(os.path.join(GOLDEN, "water_23559.npz"))
    s = W.config_water_23k()
    import hashlib
    assert hashlib.sha256(s.xyzq.tobytes()).digest() == z["xyzq_sha"].tobytes()
    E, F = oracle_lib.gsek_forward(s.grid, s.boxes, s.sigma, s.xyzq.astype(np.float64))
    assert E == float(z["E"])
    assert np.array_equal(F, z["F"])


def test_ewald_recip_restatement_matches_reference(oracle_lib):
    if not oracle_lib.have_reference():
        pytest.skip("reference build not present")
    from gse_b200 import workloads as W
    ortho = W.triplets(60, 10.0, 7).astype(np.float64) * np.array([1.0, 1.3, 0.8, 1.0])
    for xyzq, box, kcut in [(W.reference_pair(1.0), (20.0,) * 3, 32),
                            (W.random_charges(40, 12.0, 2), (12.0,) * 3, 9),
                            (W.triplets(60, 10.0, 5).astype(np.float64), (10.0,) * 3, 11),
                            (ortho, (10.0, 13.0, 8.0), 10)]:
        e1, f1 = oracle_lib.ewald_recip(2.0, kcut, box, xyzq)
        e2, f2 = oracle_lib.ref_ewald_recip(2.0, kcut, box, xyzq)
        assert abs(e1 - e2) <= 1e-12 * abs(e2)
        assert oracle_lib.force_rms(f1, f2) <= 1e-12


def test_ewald_direct_restatement_matches_reference(oracle_lib):
    if not oracle_lib.have_reference():
        pytest.skip("reference build not present")
    from gse_b200 import workloads as W
    xyzq = W.triplets(300, 14.0, 6).astype(np.float64)
    e1, f1 = oracle_lib.ewald_direct(2.0, 6.0, (14.0, 14.0, 14.0), xyzq)
    e2, f2 = oracle_lib.ref_ewald_direct(2.0, 6.0, (14.0, 14.0, 14.0), xyzq)
    assert e1 == e2
    assert np.array_equal(f1, f2)


def odd_exclusions(n):
    """Water exclusions plus entries the reference reads but never matches or
    matches in one direction only: a negative (1-4) entry, a partner listed
    under the larger index, a duplicate, a zero and one beyond the last atom."""
    from gse_b200 import workloads as W
    ib, nb = W.triplet_exclusions(n)
    lists = [list(nb[(ib[a - 1] if a else 0):ib[a]]) for a in range(n)]
    lists[0] += [-5, 2, 0, n + 7]  # -5: pair (0, 4); 2 again; 0 and n + 7 match nothing
    lists[7] += [2]                # (7, 1) listed under 7 only: not excluded
    lists[9] += [-(n)]             # pair (9, n - 1)
    ib2 = np.cumsum([len(l) for l in lists]).astype(np.int32)
    nb2 = np.array([v for l in lists for v in l], dtype=np.int32)
    return ib2, nb2


def test_ewald_direct_exclusions_match_reference(oracle_lib):
    if not oracle_lib.have_reference():
        pytest.skip("reference build not present")
    from gse_b200 import workloads as W
    xyzq = W.triplets(300, 14.0, 6).astype(np.float64)
    ib, nb = odd_exclusions(300)
    box = (14.0, 13.0, 15.0)
    e0, _ = oracle_lib.ewald_direct(2.0, 6.0, box, xyzq)
    e1, f1 = oracle_lib.ewald_direct(2.0, 6.0, box, xyzq, iblo14=ib, inb14=nb)
    e2, f2 = oracle_lib.ref_ewald_direct(2.0, 6.0, box, xyzq, iblo14=ib, inb14=nb)
    assert e1 == e2
    assert np.array_equal(f1, f2)
    assert abs(e1 - e0) > 1.0  # the intramolecular pairs carry most of the direct energy


def test_ewald_known_answer():
    """cpu_gse.cpp:324-330: energy_ew = 1733.61 for data/xyzq_48k.txt,
    sigma 2.12132034355964, box 80, kcut 64 (tests/golden/make_ewald_kat.py)."""
    with open(os.path.join(GOLDEN, "ewald_kat_48k.json")) as f:
        kat = json.load(f)
    assert round(kat["oracle_energy"], 2) == kat["reference_energy"] == 1733.61


def test_force_rms_definition(oracle_lib):
    F = np.array([[1.0, 0, 0], [0, 2.0, 0]])
    G = F + np.array([[0.1, 0, 0], [0, 0, 0]])
    assert abs(oracle_lib.force_rms(G, F) - 0.1 / np.sqrt(5.0)) < 1e-15


def test_reference_test48k_golden(oracle_lib, ref48k):
    """The restatement reproduces the reference's own real-system case
    (test48K, cpu_gse.cpp:216-250) bit for bit: energy, the sampled forces and
    the force moments over all 48,191 atoms."""
    import hashlib
    x, z = ref48k
    assert hashlib.sha256(x.tobytes()).digest() == z["xyzq_sha"].tobytes()
    g = int(z["grid"])
    E, F = oracle_lib.gsek_forward((g, g, g), (float(z["box"]),) * 3, float(z["sigma"]), x)
    assert E == float(z["E"])
    assert np.array_equal(F[z["idx"]], z["F"])
    assert (F * F).sum() == float(z["F2sum"])


@pytest.mark.parametrize("kappa,lam", [(0.3, 2.5), (0.45, 3.5), (0.25, 4.0)])
def test_restatement_matches_reference_at_other_splittings(oracle_lib, kappa, lam):
    """The reference drivers always use kappa 0.4 and lambda 3 (cpu_gse.cpp:424-426);
    the classes take any kappa < 0.5 and lambda.  The restatement equals the
    compiled reference bit for bit away from those values too."""
    if not oracle_lib.have_reference():
        pytest.skip("reference build not present")
    from gse_b200 import workloads as W
    x = W.triplets(300, 15.0, 5).astype(np.float64) * np.array([1.0, 1.1, 1.2, 1.0])
    M, box = (16, 18, 20), (15.0, 16.5, 18.0)
    e1, f1 = oracle_lib.gsek_forward(M, box, 2.0, x, kappa=kappa, lambda_sigma1=lam)
    e2, f2 = oracle_lib.ref_gsek_forward(M, box, 2.0, x, kappa=kappa, lambda_sigma=lam,
                                         lambda_sigma1=lam)
    assert e1 == e2
    assert np.array_equal(f1, f2)


@pytest.mark.parametrize("name", ["water_48000_L78.4_M80", "water_262143_L140_M144"])
def test_restatement_equals_reference_on_benchmark_boxes(oracle_lib, name):
    """The restatement reproduces the compiled reference's CpuGSEk<double,double>
    bit for bit on the two large benchmark boxes (make_ref_configs.py): energy,
    4096 sampled forces and the force moments over every atom."""
    from conftest import load_ref_config
    system, z = load_ref_config(name)
    E, F = oracle_lib.gsek_forward(system.grid, system.boxes, system.sigma,
                                   system.xyzq.astype(np.float64))
    assert E == float(z["E"])
    assert np.array_equal(F[z["idx"]], z["F"])
    assert (F * F).sum() == float(z["F2sum"])
    assert np.array_equal(F.sum(axis=0), z["Fsum"])
