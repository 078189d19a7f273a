"""gse_spread_mixed_noalloc: mixed-precision spreading without any device
allocation, for callers that may not allocate while they run (an engine
whose memory pool must stay the only owner of device memory, or a time-step
loop that cannot take cudaMalloc's synchronisation).

Called through the C ABI on two inputs in a row; each result must match the
existing entry point (gse_gauss_spread on a mixed-precision context) within
the tolerance used for the mixed spread elsewhere in the tests.  Collected
last so that a failure here comes after every other test has run; it passes
alone in a fresh process as well as after the rest of the suite."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # max |diff| / max |grid|, as for the mixed spread stage tests


def _existing_spread(M, box, s1, rc, xyzq32):
    from gse_b200.gse import CpuGaussCharge, CpuGrid
    gc = CpuGaussCharge(*M, precision="mixed")
    rho = CpuGrid(*M, dtype=np.float32)
    gc.spreadChargeToGrid(s1, rc, xyzq32.shape[0], xyzq32, *box, rho)
    return rho.data


def test_noalloc_spread_matches_existing_entry_point_twice():
    import torch
    import oracle
    from gse_b200 import _lib
    from gse_b200 import workloads as W
    L = _lib.load()
    M, box = (17, 18, 20), (18.0, 19.0, 21.0)
    s1, _, rc = oracle.gse_params(2.0)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.empty(M[2] * M[1] * M[0], dtype=torch.float32, device="cuda")
    for seed, n in ((5, 600), (6, 903)):
        x = W.triplets(n, 18.0, seed) * np.array([1.0, 19.0 / 18.0, 21.0 / 18.0, 1.0],
                                                  dtype=np.float32)
        x = np.ascontiguousarray(x, dtype=np.float32)
        d = torch.from_numpy(x).cuda()
        st = L.gse_spread_mixed_noalloc(M[0], M[1], M[2], s1, rc, n, d.data_ptr(), *box,
                                        out.data_ptr(), stream)
        assert st == 0, L.gse_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(M[2], M[1], M[0])
        want = _existing_spread(M, box, s1, rc, x)
        assert np.abs(got - want).max() <= TOL * np.abs(want).max()
        # and against the CPU restatement of the reference's spread in double
        ref = oracle.spread(M, box, s1, rc, x.astype(np.float64))
        assert np.abs(got - ref).max() <= TOL * np.abs(ref).max()


def test_noalloc_spread_rejects_oversized_grid_and_host_memory():
    import torch
    from gse_b200 import _lib
    L = _lib.load()
    out = torch.empty(8, dtype=torch.float32, device="cuda")
    st = L.gse_spread_mixed_noalloc(128, 128, 128, 1.26, 5.4, 0, None, 140.0, 140.0, 140.0,
                                    out.data_ptr(), None)
    assert st == 1 and "no-allocation limit" in L.gse_last_error().decode()
    host = np.zeros(8, dtype=np.float32)
    st = L.gse_spread_mixed_noalloc(2, 2, 2, 1.26, 5.4, 0, None, 2.0, 2.0, 2.0,
                                    host.ctypes.data, None)
    assert st == 1 and "device memory" in L.gse_last_error().decode()


def test_noalloc_spread_rejects_a_misaligned_record_array():
    """Positions are read as 16-byte records: a device pointer 4 bytes into an
    allocation is refused on the host, before anything runs on the GPU."""
    import torch
    from gse_b200 import _lib
    L = _lib.load()
    x = torch.zeros(4 * 10 + 1, dtype=torch.float32, device="cuda")
    out = torch.empty(8 * 8 * 8, dtype=torch.float32, device="cuda")
    st = L.gse_spread_mixed_noalloc(8, 8, 8, 1.26, 5.4, 10, x.data_ptr() + 4, 8.0, 8.0, 8.0,
                                    out.data_ptr(), None)
    assert st == 1 and "16-byte aligned" in L.gse_last_error().decode()
