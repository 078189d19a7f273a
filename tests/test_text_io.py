"""The reference driver's text formats (CpuGrid::save, CpuGrid.h:76-106;
saveForce / readForce / loadArray / Erms, cpu_gse.cpp:128-196) in both
mirrors: a C++ caller of gse_dropin.h and the Python functions write the same
bytes, and the readers return what the writers wrote."""
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

VALUES = [1.0 / 3.0, -2.5e-7, 123456789.0, 0.0, -0.0, 1e30, -7.0, 0.000123456789, 65536.5]

CXX = r"""
#include "gse_dropin.h"
int main(int argc, char** argv) {
  const double v[] = {%s};
  const int n = sizeof(v) / sizeof(v[0]) / 3;
  gse_b200::saveForce(argv[1], n, v, v + n, v + 2 * n);
  std::vector<float> vf(v, v + 3 * n);
  gse_b200::saveForce(argv[2], n, vf.data(), vf.data() + n, vf.data() + 2 * n);
  gse_b200::CpuGrid<double> g(3, 1, 3);
  for (int i = 0; i < 9; i++) g.getDataPointer()[i] = v[i];
  g.save(argv[3]);
  std::vector<double> a(3 * n);
  gse_b200::loadArray<double>(3, n, argv[1], a.data());
  std::vector<double> fx(n), fy(n), fz(n);
  gse_b200::readForce<double>(argv[1], n, fx.data(), fy.data(), fz.data());
  printf("%%.17g %%.17g\n", a[4], fy[1]);
  printf("%%.17g\n", gse_b200::Erms(n, v, v + n, v + 2 * n, fx.data(), fy.data(), fz.data()));
  try {
    gse_b200::loadArray<double>(3, n + 1, argv[1], a.data());
  } catch (const gse_b200::Error& e) {
    printf("short file: %%d\n", (int)e.status);
  }
  return 0;
}
"""


def build_cxx(tmp_path):
    from gse_b200 import build
    lib = build.build_lib()
    src = tmp_path / "io_check.cpp"
    src.write_text(CXX % ", ".join(repr(v) for v in VALUES))
    exe = tmp_path / "io_check"
    libdir = os.path.dirname(lib)
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "gse_b200", "cxx"), str(src), "-o", str(exe),
                    "-L", libdir, "-lgse_b200", "-Wl,-rpath," + libdir], check=True)
    return exe


def test_text_formats_match_between_mirrors(tmp_path):
    from gse_b200.gse import CpuGrid, Erms, loadArray, readForce, saveForce
    exe = build_cxx(tmp_path)
    out = subprocess.run([str(exe), str(tmp_path / "f_cxx.txt"), str(tmp_path / "f32_cxx.txt"),
                          str(tmp_path / "g_cxx.txt")], capture_output=True, text=True, check=True)
    v = np.array(VALUES)
    n = len(VALUES) // 3
    saveForce(tmp_path / "f_py.txt", n, v[:n], v[n:2 * n], v[2 * n:])
    vf = v.astype(np.float32)
    saveForce(tmp_path / "f32_py.txt", n, vf[:n], vf[n:2 * n], vf[2 * n:])
    g = CpuGrid(3, 1, 3, dtype=np.float64)
    g.data[...] = v[:9].reshape(g.data.shape)
    g.save(tmp_path / "g_py.txt")
    for a, b in (("f_cxx.txt", "f_py.txt"), ("f32_cxx.txt", "f32_py.txt"), ("g_cxx.txt", "g_py.txt")):
        assert (tmp_path / a).read_bytes() == (tmp_path / b).read_bytes(), a
    # six significant digits, as iostream writes them
    assert (tmp_path / "f_py.txt").read_text().splitlines()[0] == "0.333333 0 -7"
    lines = out.stdout.splitlines()
    a4, fy1 = (float(t) for t in lines[0].split())
    fx, fy, fz = readForce(tmp_path / "f_cxx.txt", n)
    arr = loadArray(3, n, tmp_path / "f_cxx.txt")
    assert arr.reshape(-1)[4] == a4 and fy[1] == fy1
    assert float(lines[1]) == Erms(n, v[:n], v[n:2 * n], v[2 * n:], fx, fy, fz)
    assert lines[2] == "short file: 1"
    ib = loadArray(1, 3, tmp_path / "f_cxx.txt", np.float64)
    assert ib.shape == (3, 1)


def test_erms_is_the_oracle_force_rms():
    import oracle
    from gse_b200.gse import Erms
    rng = np.random.default_rng(3)
    R = rng.standard_normal((50, 3))
    F = R + 1e-3 * rng.standard_normal((50, 3))
    assert abs(Erms(50, *R.T, *F.T) - oracle.force_rms(F, R)) <= 1e-15


def _grid_values(dtype):
    rng = np.random.default_rng(11)
    v = rng.standard_normal(4 * 3 * 5) * 10.0 ** rng.integers(-8, 9, 4 * 3 * 5)
    v[:9] = VALUES
    v[9:13] = [1e-5, 1e-4, 99999.95, 100000.5]  # where %g switches notation / rounds up
    return v.astype(dtype).reshape(5, 3, 4)  # [z][y][x]: sizeX 4, sizeY 3, sizeZ 5


def test_grid_save_is_the_reference_writer(tmp_path, oracle_lib):
    """CpuGrid::save of the Python mirror writes the bytes of the reference's
    own header-only writer (CpuGrid.h:76-90, compiled into the oracle's
    reference build), in both calculation types, on a non-cubic grid."""
    if not oracle_lib.have_reference():
        import pytest
        pytest.skip("reference build not present")
    from gse_b200.gse import CpuGrid
    for dt in (np.float64, np.float32):
        v = _grid_values(dt)
        oracle_lib.ref_grid_save(v, tmp_path / "g_ref.txt")
        g = CpuGrid(4, 3, 5, dtype=dt)
        g.data[...] = v
        g.save(tmp_path / "g_py.txt")
        assert (tmp_path / "g_py.txt").read_bytes() == (tmp_path / "g_ref.txt").read_bytes(), dt
