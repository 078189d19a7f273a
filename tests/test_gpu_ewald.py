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
