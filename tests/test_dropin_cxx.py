"""The C++ drop-in classes (gse_b200/cxx/gse_dropin.h) compiled into a caller
written against the reference's class API (gse_dropin_check.cpp).

CPU: the program builds, links against libgse_b200.so and reports a clean
error without a GPU.  GPU: CpuGSEk and the stage classes reproduce the
reference's energies and forces (FP64 within 1e-12, mixed within 1e-5)."""
import os
import subprocess

import numpy as np
import pytest


def program():
    from gse_b200 import build
    build.build_lib()
    return build.build_cxx_check()


def run(prog, precision, g, tmp_path, env=None):
    M = [int(v) for v in g["M"]]
    box = [float(v) for v in g["box"]]
    path = tmp_path / "xyzq.txt"
    np.savetxt(path, g["xyzq"], fmt="%.17g")
    out = subprocess.run([prog, precision, *map(str, M), *map(repr, box), repr(float(g["sigma"])),
                          str(path)], capture_output=True, text=True, timeout=300,
                         env=dict(os.environ, **(env or {})))
    return out


def parse(text):
    E = Es = None
    F, Fs = [], []
    for line in text.splitlines():
        tag, *vals = line.split()
        if tag == "PATHS":
            continue
        if tag == "E":
            E = float(vals[0])
        elif tag == "E_stages":
            Es = float(vals[0])
        elif tag == "F":
            F.append([float(v) for v in vals])
        elif tag == "F_stages":
            Fs.append([float(v) for v in vals])
    return E, np.array(F), Es, np.array(Fs)


def rms(F, R):
    d = F - R
    return float(np.sqrt((d * d).sum() / (R * R).sum()))


def test_program_builds_and_fails_cleanly_without_gpu(goldens, tmp_path):
    import torch
    prog = program()
    assert os.access(prog, os.X_OK)
    assert subprocess.run([prog], capture_output=True).returncode == 2
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    out = run(prog, "fp64", goldens["pair_L20_M20"], tmp_path)
    assert out.returncode == 1
    assert "GSE_ERR_UNSUPPORTED" in out.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["pair_L20_M20", "water300_noncubic", "water600_L18_M17_odd"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_dropin_classes_match_reference(goldens, tmp_path, case, precision, tol):
    g = goldens[case]
    out = run(program(), precision, g, tmp_path)
    assert out.returncode == 0, out.stderr
    E, F, Es, Fs = parse(out.stdout)
    Eref, Fref = float(g["E"]), g["F"]
    print(case, precision, abs(E - Eref) / abs(Eref), rms(F, Fref), abs(Es - Eref) / abs(Eref),
          rms(Fs, Fref))
    assert abs(E - Eref) <= tol * abs(Eref)
    assert rms(F, Fref) <= tol
    assert abs(Es - Eref) <= tol * abs(Eref)
    assert rms(Fs, Fref) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol,own", [("fp64", 1e-12, "1"), ("mixed", 1e-5, "0"),
                                               ("mixed", 1e-5, "1")])
def test_dropin_64cubed_green_multiply_inside_the_fft(tmp_path, precision, tol, own):
    """A process without PyTorch links the Green's multiply into the c2r
    transform (cuFFT load callback) for grids of 64^3 points and more; the
    mixed form on a cubic 16 N2 grid takes the library's own FFT instead
    unless GSE_B200_OWN_FFT=0.  The 23,559-charge water box (M = 64) checks
    each path against the reference."""
    from conftest import GOLDEN
    from gse_b200 import workloads as W
    z = np.load(os.path.join(GOLDEN, "water_23559.npz"))
    s = W.config_water_23k()
    g = {"M": np.array(s.grid), "box": np.array(s.boxes), "sigma": np.array(s.sigma),
         "xyzq": s.xyzq.astype(np.float64)}
    out = run(program(), precision, g, tmp_path, env={"GSE_B200_OWN_FFT": own})
    assert out.returncode == 0, out.stderr
    paths = int([ln for ln in out.stdout.splitlines() if ln.startswith("PATHS")][0].split()[1])
    if precision == "mixed" and own == "1":
        assert paths & 8 and not paths & 2, paths
    else:
        assert paths & 2, "Green's multiply not inside the FFT"
    E, F, Es, Fs = parse(out.stdout)
    print(precision, abs(E - float(z["E"])) / abs(float(z["E"])), rms(F, z["F"]))
    assert abs(E - float(z["E"])) <= tol * abs(float(z["E"]))
    assert rms(F, z["F"]) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision,dt", [("fp64", np.float64), ("mixed", np.float32)])
def test_dropin_grid_operations(goldens, tmp_path, precision, dt):
    """CpuGaussCharge::spreadChargeOnGrid (the real-space variant's second
    spreading, sigma2), calcElectricFieldOnGrid and calcDipoleSum called by
    a C++ caller on the grids of its own evaluation, against the oracle
    restatement of the same reference methods: the grids bit for bit, the
    dipole within 1e-12 of the sum of its |terms|."""
    import oracle
    g = goldens["water300_noncubic"]
    M = tuple(int(v) for v in g["M"])
    box = tuple(float(v) for v in g["box"])
    L = dict(os.environ, GSE_CHECK_GRID_OPS="1")
    path = tmp_path / "xyzq.txt"
    np.savetxt(path, g["xyzq"], fmt="%.17g")
    out = subprocess.run([program(), precision, *map(str, M), *map(repr, box),
                          repr(float(g["sigma"])), str(path)], capture_output=True, text=True,
                         timeout=300, env=L)
    assert out.returncode == 0, out.stderr
    dip = None
    rows = []
    for line in out.stdout.splitlines():
        tag, *vals = line.split()
        if tag == "DIP":
            dip = np.array([float(v) for v in vals])
        elif tag == "G":
            rows.append([float(v) for v in vals])
    G = np.array(rows).astype(dt)
    assert G.shape == (M[0] * M[1] * M[2], 6)
    rho, phi, rhoS, ex, ey, ez = (G[:, k].reshape(M[::-1]) for k in range(6))
    _, s2, _ = oracle.gse_params(float(g["sigma"]))
    rc2 = 3.0 * np.sqrt(2.0) * s2
    assert np.array_equal(rhoS, oracle.spread_on_grid(M, box, s2, rc2, rho, dt))
    for e, w in zip((ex, ey, ez), oracle.efield(M, box, phi, dt)):
        assert np.array_equal(e, w)
    ref = oracle.dipole_sum(M, box, rho, dt)
    h = np.array(box) / np.array(M)
    z, y, x = np.meshgrid(*(np.arange(m) for m in M[::-1]), indexing="ij")
    v = np.abs(rho.astype(np.float64)) * h.prod()
    scale = np.array([(v * x * h[0]).sum(), (v * y * h[1]).sum(), (v * z * h[2]).sum()])
    assert (np.abs(dip - ref) <= 1e-12 * scale).all()


@pytest.mark.gpu
def test_dropin_ewald_classes(goldens, tmp_path):
    """CpuEwaldRecip (kcut 12) and CpuEwaldDirect (rcut 9, with the exclusion
    lists of rigid 3-site molecules) called by a C++ caller, the sequence of
    cpu_gse.cpp:555-560, against the oracle restatements of the same methods."""
    import oracle
    from gse_b200 import workloads as W
    g = goldens["water300_noncubic"]
    box = tuple(float(v) for v in g["box"])
    sigma = float(g["sigma"])
    out = run(program(), "fp64", g, tmp_path, env={"GSE_CHECK_EWALD": "1"})
    assert out.returncode == 0, out.stderr
    vals = {"EWR": [], "FWR": [], "EWD": [], "FWD": []}
    for line in out.stdout.splitlines():
        tag, *v = line.split()
        if tag in vals:
            vals[tag].append([float(t) for t in v])
    x = np.asarray(g["xyzq"], dtype=np.float64)
    er, fr = oracle.ewald_recip(sigma, 12, box, x)
    ib, nb = W.triplet_exclusions(x.shape[0])
    ed, fd = oracle.ewald_direct(sigma, 9.0, box, x, iblo14=ib, inb14=nb)
    assert abs(vals["EWR"][0][0] - er) <= 1e-11 * abs(er)
    assert rms(np.array(vals["FWR"]), fr) <= 1e-11
    assert abs(vals["EWD"][0][0] - ed) <= 1e-12 * abs(ed)
    assert rms(np.array(vals["FWD"]), fd) <= 1e-12


CXX_INSTANCES = r"""
#include "gse_dropin.h"
using namespace gse_b200;
template <typename AT, typename CT>
int use(int n) {
  CpuGaussCharge<AT, CT> g(16, 16, 16);
  std::vector<xyzq_t<CT>> x(n, xyzq_t<CT>{1, 2, 3, 1});
  CpuGrid<CT> rho(16, 16, 16), phi(16, 16, 16);
  std::vector<AT> fx(n), fy(n), fz(n);
  g.spreadChargeToGrid(1.0, 4.0, n, x.data(), 16.0, 16.0, 16.0, rho);
  g.interpolateForce(1.0, 4.0, n, x.data(), 16.0, 16.0, 16.0, phi, fx.data(), fy.data(), fz.data());
  AT d[3];
  g.calcDipoleSum(16.0, 16.0, 16.0, rho, d[0], d[1], d[2]);
  return g.calcSupportSize(4.0, 16.0, 16.0, 16.0);
}
int main() {
  try {
    return use<double, double>(3) + use<double, float>(3) + use<float, float>(3) > 0 ? 0 : 1;
  } catch (const Error& e) {
    printf("error %d\n", (int)e.status);
    return 3;
  }
}
"""


def test_reference_instances_compile(tmp_path):
    """CpuGaussCharge<double,double>, <double,float> and <float,float> (the
    reference's instances, CpuGaussCharge.cpp:524-526) compile against the
    drop-in header and link; without a GPU the first call reports the
    library's error status instead of computing."""
    import torch
    from gse_b200 import build
    lib = build.build_lib()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "instances.cpp"
    src.write_text(CXX_INSTANCES)
    exe = tmp_path / "instances"
    libdir = os.path.dirname(lib)
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(root, "include"),
                    "-I", os.path.join(root, "gse_b200", "cxx"), str(src), "-o", str(exe),
                    "-L", libdir, "-lgse_b200", "-Wl,-rpath," + libdir], check=True)
    if torch.cuda.is_available():
        return
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 3 and out.stdout.startswith("error "), (out.returncode, out.stdout)


@pytest.mark.gpu
def test_dropin_float_float_instance(goldens, tmp_path):
    """The reference's third instance, CpuGaussCharge<float,float>
    (CpuGaussCharge.cpp:524-526), through the C++ drop-in on the GPU: its
    spread and its gather (float force arrays) against the oracle's float
    restatement of the reference, which equals the compiled reference's float
    instance bit for bit (test_oracle.py), within 1e-5."""
    import oracle
    g = goldens["water300_noncubic"]
    prog = program()
    out = run(prog, "mixed", g, tmp_path, env={"GSE_CHECK_FLOAT_FLOAT": "1"})
    assert out.returncode == 0, out.stderr
    rows = {"RFF": [], "FFF": [], "PHI": []}
    for line in out.stdout.splitlines():
        tag, *vals = line.split()
        if tag in rows:
            rows[tag].append([float(v) for v in vals])
    M = tuple(int(v) for v in g["M"])
    box = tuple(float(v) for v in g["box"])
    s1, _, rc = oracle.gse_params(float(g["sigma"]))
    x32 = np.asarray(g["xyzq"], dtype=np.float32)
    rho = np.array(rows["RFF"], dtype=np.float32).reshape(M[2], M[1], M[0])
    phi = np.array(rows["PHI"], dtype=np.float32).reshape(M[2], M[1], M[0])
    F = np.array(rows["FFF"])
    want_rho = oracle.spread(M, box, s1, rc, x32, dtype=np.float32)
    assert np.abs(rho - want_rho).max() <= 1e-5 * np.abs(want_rho).max()
    want_F = np.stack(oracle.gather(M, box, s1, rc, x32, phi, dtype=np.float32), axis=1)
    assert F.shape == want_F.shape and rms(F, want_F) <= 1e-5
