"""Batched systems (gse_batch_*, mixed form) through the C ABI.

Every system of a batch must give what a mixed single-system context gives on
its own: energies within 1e-6 relative, forces within 1e-5 relative RMS (the
two paths round the grid differently: 64-bit fixed point with a global scale
in the batch, per-brick scales in the single-system spread), and both within
1e-5 of the FP64 form.  A batch's own results are bit-identical run to run,
and a replayed CUDA graph gives what the eager call gives."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIGMA = 2.0


def rms(F, R):
    d = np.asarray(F, np.float64) - np.asarray(R, np.float64)
    return float(np.sqrt((d * d).sum() / max((np.asarray(R, np.float64) ** 2).sum(), 1e-300)))


def mixed_systems():
    """Uneven systems: cubic ones as the batching workload builds them, plus
    odd, non-cubic, tiny (stencil wider than the grid) and empty systems."""
    from gse_b200 import workloads as W
    out = []
    for s in W.config_batch(10, seed=3, n_min=501, n_max=4001):
        out.append({"size": s.grid, "box": s.boxes, "xyzq": s.xyzq})
    out.append({"size": (17, 18, 20), "box": (17.5, 18.2, 19.9),
                "xyzq": W.triplets(900, 17.5, 5).astype(np.float32)
                * np.array([1.0, 18.2 / 17.5, 19.9 / 17.5, 1.0], np.float32)})
    out.append({"size": (10, 10, 10), "box": (10.0, 10.0, 10.0),
                "xyzq": W.triplets(99, 10.0, 6).astype(np.float32)})
    out.append({"size": (16, 16, 16), "box": (16.0, 16.0, 16.0),
                "xyzq": np.zeros((0, 4), np.float32)})
    return out


def make_batch(systems):
    from gse_b200.gse import Batch
    desc = [{"size": s["size"], "box": s["box"], "n": s["xyzq"].shape[0]} for s in systems]
    b = Batch(desc, sigma=SIGMA, kappa=0.4, lambdaSigma1=3.0)
    xyzq = np.concatenate([s["xyzq"] for s in systems]).astype(np.float32)
    return b, xyzq


def single(s, precision):
    from gse_b200.gse import Context
    M, box = s["size"], s["box"]
    ctx = Context(M[0], M[1], M[2], SIGMA, 0.4, 3.0, 3.0, box[0], box[1], box[2],
                  precision=precision)
    ct = np.float32 if precision == "mixed" else np.float64
    x = s["xyzq"].astype(ct)
    n = x.shape[0]
    fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
    E = ctx.forward(n, x, fx, fy, fz) if n else 0.0
    return ctx, E, np.stack([fx, fy, fz], 1)


@pytest.fixture(scope="module")
def batch_case():
    systems = mixed_systems()
    b, xyzq = make_batch(systems)
    return systems, b, xyzq


def test_batch_forward_matches_single_systems(batch_case):
    systems, b, xyzq = batch_case
    E, F = b.forward(xyzq)
    assert E.shape == (len(systems),) and F.shape == (b.n_total, 3)
    for k, s in enumerate(systems):
        lo, hi = b.first[k], b.first[k + 1]
        if hi == lo:
            assert E[k] == 0.0
            continue
        _, Em, Fm = single(s, "mixed")
        _, Ed, Fd = single(s, "fp64")
        print(k, s["size"], hi - lo, "E rel", abs(E[k] - Em) / abs(Em), "F rms", rms(F[lo:hi], Fm),
              "vs fp64", rms(F[lo:hi], Fd))
        assert abs(E[k] - Em) <= 1e-6 * abs(Em)
        assert rms(F[lo:hi], Fm) <= 1e-5
        assert rms(F[lo:hi], Fd) <= 1e-5
        assert abs(E[k] - Ed) <= 1e-5 * abs(Ed)


def test_batch_is_deterministic(batch_case):
    _, b, xyzq = batch_case
    E1, F1 = b.forward(xyzq)
    E2, F2 = b.forward(xyzq)
    assert np.array_equal(F1, F2)
    assert np.allclose(E1, E2, rtol=1e-13, atol=0.0)


def test_graph_replay_matches_eager(batch_case):
    import torch
    _, b, xyzq = batch_case
    E, F = b.forward(xyzq)
    bufs = b.buffers()
    b.capture(with_adjoint=False)
    bufs["forces"].zero_()
    bufs["energies"].zero_()
    for _ in range(3):
        b.launch()
    torch.cuda.synchronize()
    assert np.array_equal(bufs["forces"].cpu().numpy().T, F)
    assert np.allclose(bufs["energies"].cpu().numpy(), E, rtol=1e-13, atol=0.0)
    # new positions written into the batch's buffer are picked up by the graph
    x2 = xyzq.copy()
    x2[:, :3] += 0.37
    bufs["xyzq"].copy_(torch.from_numpy(x2))
    b.launch()
    torch.cuda.synchronize()
    E2, F2 = b.forward(x2)
    assert np.array_equal(bufs["forces"].cpu().numpy().T, F2)


def test_batch_adjoint_matches_single_systems(batch_case):
    systems, b, xyzq = batch_case
    rng = np.random.default_rng(4)
    G = rng.standard_normal((b.n_total, 3))
    dLdE = rng.uniform(0.5, 1.5, len(systems))
    dq, dx = b.adjoint(xyzq, dLdE, G)
    for k, s in enumerate(systems):
        lo, hi = int(b.first[k]), int(b.first[k + 1])
        n = hi - lo
        if n == 0:
            continue
        ctx, _, _ = single(s, "mixed")
        x = s["xyzq"].astype(np.float32)
        q, gx, gy, gz = (np.zeros(n) for _ in range(4))
        g = G[lo:hi]
        ctx.adjoint(n, x, float(dLdE[k]), np.ascontiguousarray(g[:, 0]),
                    np.ascontiguousarray(g[:, 1]), np.ascontiguousarray(g[:, 2]), q, gx, gy, gz)
        print(k, "dq rms", rms(dq[lo:hi], q), "dx rms", rms(dx[lo:hi], np.stack([gx, gy, gz], 1)))
        assert rms(dq[lo:hi], q) <= 1e-5
        assert rms(dx[lo:hi], np.stack([gx, gy, gz], 1)) <= 1e-5


def test_graph_with_adjoint_matches_eager(batch_case):
    import torch
    systems, b, xyzq = batch_case
    rng = np.random.default_rng(8)
    G = rng.standard_normal((b.n_total, 3))
    dLdE = np.ones(len(systems))
    dq, dx = b.adjoint(xyzq, dLdE, G)
    bufs = b.buffers()
    bufs["xyzq"].copy_(torch.from_numpy(xyzq))
    bufs["dLdE"].copy_(torch.from_numpy(dLdE))
    bufs["grad_forces"].copy_(torch.from_numpy(np.ascontiguousarray(G.T)))
    b.capture(with_adjoint=True)
    bufs["grad_out"].zero_()
    b.launch()
    torch.cuda.synchronize()
    out = bufs["grad_out"].cpu().numpy()
    # the reverse pass accumulates its source grid in 64-bit fixed point, so
    # it is as reproducible as the forward pass
    assert np.array_equal(out[0], dq)
    assert np.array_equal(out[1:].T, dx)


def test_autotune_and_cache(batch_case, tmp_path):
    _, b, xyzq = batch_case
    E0, F0 = b.forward(xyzq)
    cache = tmp_path / "tune.txt"
    b.autotune(cache, use_cache=False)
    i1 = b.info()
    text = cache.read_text().split()
    assert len(text) == 7 and text[0].startswith("batch-n") and text[2] == "0"
    E1, F1 = b.forward(xyzq)
    assert rms(F1, F0) <= 1e-12 and np.allclose(E1, E0, rtol=1e-12)
    b.autotune(cache, use_cache=True)  # taken from the file, no new line
    i2 = b.info()
    assert len(cache.read_text().splitlines()) == 1
    assert (i1.scatter_ctas, i1.gather_ctas, i1.largest_first) == \
        (i2.scatter_ctas, i2.gather_ctas, i2.largest_first)


def test_batch_of_256_systems_runs():
    """The batching workload's full size: 256 systems, N log-uniform in
    [501, 8001].  Spot-check three systems against single contexts."""
    from gse_b200 import workloads as W
    syst = [{"size": s.grid, "box": s.boxes, "xyzq": s.xyzq} for s in W.config_batch(256)]
    b, xyzq = make_batch(syst)
    E, F = b.forward(xyzq)
    assert np.isfinite(E).all() and np.isfinite(F).all()
    for k in (0, 100, 255):
        lo, hi = b.first[k], b.first[k + 1]
        _, Em, Fm = single(syst[k], "mixed")
        assert abs(E[k] - Em) <= 1e-6 * abs(Em)
        assert rms(F[lo:hi], Fm) <= 1e-5


# ---- the fused path: one persistent cooperative launch per direction ------
@pytest.fixture(scope="module")
def fused_case():
    """Systems as the batching workload builds them (every grid side a
    multiple of 8, at most 64): the batch takes the fused launches."""
    from gse_b200 import workloads as W
    systems = [{"size": s.grid, "box": s.boxes, "xyzq": s.xyzq}
               for s in W.config_batch(12, seed=7, n_min=501, n_max=8001)]
    b, xyzq = make_batch(systems)
    assert b.info().fused_available == 1 and b.info().fused == 0  # starts per stage
    b.set_schedule(fused=True, gather_lanes=16)
    return systems, b, xyzq


def test_fused_batch_forward_matches_single_systems(fused_case):
    """Each direction of the fused batch is one kernel; its small-grid FFT is
    the library's own (not cuFFT's), so results agree with single contexts to
    FP32 rounding: energies within 1e-6, forces within 1e-5, and both forms
    within 1e-5 of FP64."""
    systems, b, xyzq = fused_case
    assert b.info().fused == 1
    E, F = b.forward(xyzq)
    for k, s in enumerate(systems):
        lo, hi = b.first[k], b.first[k + 1]
        _, Em, Fm = single(s, "mixed")
        _, Ed, Fd = single(s, "fp64")
        print(k, s["size"], hi - lo, "E rel", abs(E[k] - Em) / abs(Em), "F rms",
              rms(F[lo:hi], Fm), "vs fp64", rms(F[lo:hi], Fd))
        assert abs(E[k] - Em) <= 1e-6 * abs(Em)
        assert rms(F[lo:hi], Fm) <= 1e-5
        assert rms(F[lo:hi], Fd) <= 1e-5
        assert abs(E[k] - Ed) <= 1e-5 * abs(Ed)


def test_fused_batch_is_deterministic(fused_case):
    """Grid sums in 64-bit fixed point and the energies summed slab by slab in
    a fixed order: two runs give the same bits, energies included."""
    _, b, xyzq = fused_case
    E1, F1 = b.forward(xyzq)
    E2, F2 = b.forward(xyzq)
    assert np.array_equal(F1, F2)
    assert np.array_equal(E1, E2)


def test_fused_batch_adjoint_matches_single_systems(fused_case):
    systems, b, xyzq = fused_case
    rng = np.random.default_rng(9)
    G = rng.standard_normal((b.n_total, 3))
    dLdE = rng.uniform(0.5, 1.5, len(systems))
    dq, dx = b.adjoint(xyzq, dLdE, G)
    for k in (0, len(systems) // 2, len(systems) - 1):
        s = systems[k]
        lo, hi = int(b.first[k]), int(b.first[k + 1])
        n = hi - lo
        ctx, _, _ = single(s, "mixed")
        x = s["xyzq"].astype(np.float32)
        q, gx, gy, gz = (np.zeros(n) for _ in range(4))
        g = G[lo:hi]
        ctx.adjoint(n, x, float(dLdE[k]), np.ascontiguousarray(g[:, 0]),
                    np.ascontiguousarray(g[:, 1]), np.ascontiguousarray(g[:, 2]), q, gx, gy, gz)
        print(k, "dq rms", rms(dq[lo:hi], q), "dx rms", rms(dx[lo:hi], np.stack([gx, gy, gz], 1)))
        assert rms(dq[lo:hi], q) <= 1e-5
        assert rms(dx[lo:hi], np.stack([gx, gy, gz], 1)) <= 1e-5


def test_fused_graph_is_one_kernel_per_direction(fused_case):
    """The captured forward + reverse graph holds exactly two kernel nodes,
    and its replay gives what the eager calls give, bit for bit."""
    import torch
    systems, b, xyzq = fused_case
    rng = np.random.default_rng(10)
    G = rng.standard_normal((b.n_total, 3))
    dLdE = np.ones(len(systems))
    E, F = b.forward(xyzq)
    dq, dx = b.adjoint(xyzq, dLdE, G)
    bufs = b.buffers()
    bufs["xyzq"].copy_(torch.from_numpy(xyzq))
    bufs["dLdE"].copy_(torch.from_numpy(dLdE))
    bufs["grad_forces"].copy_(torch.from_numpy(np.ascontiguousarray(G.T)))
    b.capture(with_adjoint=True)
    assert b.info().graph_kernels == 2
    bufs["grad_out"].zero_()
    bufs["forces"].zero_()
    b.launch()
    torch.cuda.synchronize()
    out = bufs["grad_out"].cpu().numpy()
    assert np.array_equal(bufs["forces"].cpu().numpy().T, F)
    assert np.array_equal(out[0], dq)
    assert np.array_equal(out[1:].T, dx)
    b.capture(with_adjoint=False)
    assert b.info().graph_kernels == 1


def test_fused_autotune_picks_a_schedule(fused_case, tmp_path):
    """The autotuner times the per-stage schedules and the fused ones (work-item
    order x lanes per atom of the gathers) on forward + reverse passes and keeps
    the fastest; the choice is cached (key, order, fused, lanes, CTAs, ms) and
    taken back from the file; results move by no more than the two paths'
    rounding differences; the schedule can be pinned back to fused."""
    _, b, xyzq = fused_case
    E0, F0 = b.forward(xyzq)
    cache = tmp_path / "tune.txt"
    b.autotune(cache, use_cache=False)
    i1 = b.info()
    text = cache.read_text().split()
    assert len(text) == 7 and text[0].startswith("batchf-n")
    assert int(text[2]) == i1.fused and (not i1.fused or int(text[3]) == i1.gather_lanes)
    E1, F1 = b.forward(xyzq)
    assert rms(F1, F0) <= 2e-6 and np.allclose(E1, E0, rtol=1e-6)
    b.set_schedule(fused=not i1.fused)
    b.autotune(cache, use_cache=True)
    assert len(cache.read_text().splitlines()) == 1 and b.info().fused == i1.fused
    b.set_schedule(fused=True, gather_lanes=8)
    E8, F8 = b.forward(xyzq)
    assert rms(F8, F0) <= 1e-6 and np.allclose(E8, E0, rtol=1e-12)
    b.set_schedule(fused=True, gather_lanes=16)


def test_fused_and_per_stage_batches_agree(monkeypatch):
    """The same systems through the per-stage launches (cuFFT transforms,
    GSE_B200_BATCH_FUSED=0 at creation) and the fused launch."""
    from gse_b200 import workloads as W
    systems = [{"size": s.grid, "box": s.boxes, "xyzq": s.xyzq}
               for s in W.config_batch(6, seed=11, n_min=501, n_max=8001)]
    bf, xyzq = make_batch(systems)
    bf.set_schedule(fused=True)
    monkeypatch.setenv("GSE_B200_BATCH_FUSED", "0")
    bs, _ = make_batch(systems)
    assert bf.info().fused == 1 and bs.info().fused_available == 0
    from gse_b200._lib import GseError
    with pytest.raises(GseError):
        bs.set_schedule(fused=True)
    Ef, Ff = bf.forward(xyzq)
    Es, Fs = bs.forward(xyzq)
    assert rms(Ff, Fs) <= 2e-6
    assert np.allclose(Ef, Es, rtol=1e-6, atol=0.0)
