"""Argument checks of the Python bindings that need no GPU: per-atom float64
arrays handed to the library as raw addresses must hold enough contiguous
doubles (gse_b200._lib.ptr_f64), or the call is refused before it reaches the
C ABI."""
import numpy as np
import pytest
import torch

from gse_b200._lib import GseError, ptr_f64


def test_good_arrays_pass():
    a = np.zeros(10)
    assert ptr_f64(a, 10, "fx") == a.ctypes.data
    t = torch.zeros(3, 10, dtype=torch.float64)
    assert ptr_f64(t[1], 10, "fy") == t[1].data_ptr()  # a row of a (3, n) tensor
    assert ptr_f64(np.zeros(12), 10, "fz") is not None  # longer is fine
    assert ptr_f64(None, 10, "fx") is None
    assert ptr_f64(12345, 10, "fx") == 12345  # raw address: the caller's responsibility
    assert ptr_f64(np.zeros(0), 0, "fx") is not None


@pytest.mark.parametrize("bad", [
    np.zeros(10, dtype=np.float32),          # wrong dtype: doubles would overrun it
    np.zeros(9),                             # too short
    np.zeros((10, 3))[:, 0],                 # strided column view
    torch.zeros(10, dtype=torch.float32),
    torch.zeros(10, 3, dtype=torch.float64)[:, 1],
    torch.zeros(5, dtype=torch.float64),
])
def test_bad_arrays_are_refused(bad):
    with pytest.raises(GseError) as ei:
        ptr_f64(bad, 10, "fx")
    assert ei.value.status == 1
    assert "fx" in str(ei.value)


class _FakeLib:
    """Records the C-ABI calls of a Context and returns GSE_OK."""

    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        def call(*args):
            self.calls.append((name, args))
            return 0
        return call


def _fake_context(n_grid=8):
    from gse_b200.gse import Context
    ctx = object.__new__(Context)
    ctx._L = _FakeLib()
    ctx.h = None
    ctx.precision, ctx.dtype, ctx.shape = "mixed", np.float32, (n_grid,) * 3
    return ctx


def test_wrappers_hand_valid_arrays_to_the_abi_and_refuse_bad_ones():
    n = 7
    ctx = _fake_context()
    x = np.zeros((n, 4), np.float32)
    f = [np.zeros(n) for _ in range(3)]
    t = torch.zeros(4, n, dtype=torch.float64)
    e = torch.zeros(1, dtype=torch.float64)
    ctx.forward(n, x, *f)
    ctx.forward(n, x, t[0], t[1], t[2], energy_out=e)
    ctx.interpolate_force(n, x, *f)
    ctx.interpolate_field(n, x, *f)
    ctx.gauss_interpolate(1.0, 4.0, n, x, 8.0, 8.0, 8.0, np.zeros((8, 8, 8), np.float32), *f)
    ctx.adjoint(n, x, 1.0, None, None, None, t[0], t[1], t[2], t[3])
    ctx.adjoint(n, x, 1.0, f[0], f[1], f[2], t[0], t[1], t[2], t[3])
    names = [c[0] for c in ctx._L.calls]
    assert names == ["gse_forward", "gse_forward", "gse_interpolate_force",
                     "gse_interpolate_field", "gse_gauss_interpolate", "gse_adjoint", "gse_adjoint"]
    assert ctx._L.calls[0][1][4] == f[0].ctypes.data  # fx reaches the ABI unchanged
    assert ctx._L.calls[1][1][3] == e.data_ptr()
    short = np.zeros(n - 1)
    for bad_call in (lambda: ctx.forward(n, x, short, f[1], f[2]),
                     lambda: ctx.forward(n, x, *f, energy_out=torch.zeros(1)),
                     lambda: ctx.interpolate_force(n, x, f[0], f[1], np.zeros(n, np.float32)),
                     lambda: ctx.adjoint(n, x, 1.0, None, None, None, short, *f)):
        with pytest.raises(GseError):
            bad_call()
    assert len(ctx._L.calls) == 7  # refused before any call


class _FakeCudaTensor:
    """Stands in for a CUDA tensor view that starts `offset` bytes into an
    allocation (no GPU needed): only the attributes the binding inspects."""

    def __init__(self, dtype, numel, offset):
        self.dtype, self._numel, self._offset = dtype, numel, offset
        self.is_cuda = True

    def data_ptr(self):
        return 0x7f0000000000 + self._offset

    def is_contiguous(self):
        return True

    def numel(self):
        return self._numel


@pytest.mark.parametrize("precision,dtype,offset,align", [
    ("mixed", torch.float32, 4, 16), ("mixed", torch.float32, 8, 16),
    ("fp64", torch.float64, 16, 32), ("fp64", torch.float64, 8, 32)])
def test_misaligned_device_positions_are_refused_before_the_abi(precision, dtype, offset, align):
    """Positions are read on the GPU as float4/double4 records: a CUDA view
    whose start is not 16/32-byte aligned is refused by every wrapper that
    takes positions, and nothing reaches the library (the library checks the
    same on the host for callers of the C ABI)."""
    n = 5
    ctx = _fake_context()
    ctx.precision, ctx.dtype = precision, (np.float32 if precision == "mixed" else np.float64)
    x = _FakeCudaTensor(dtype, 4 * n, offset)
    f = [np.zeros(n) for _ in range(3)]
    for call in (lambda: ctx.forward(n, x, *f), lambda: ctx.spread_charge(n, x),
                 lambda: ctx.interpolate_force(n, x, *f), lambda: ctx.interpolate_field(n, x, *f),
                 lambda: ctx.adjoint(n, x, 1.0, None, None, None, *f, np.zeros(n))):
        with pytest.raises(GseError) as ei:
            call()
        assert ei.value.status == 1 and f"{align}-byte aligned" in str(ei.value)
    assert ctx._L.calls == []
    ok = _FakeCudaTensor(dtype, 4 * n, 2 * align)  # aligned view: passes to the ABI
    ctx.spread_charge(n, ok)
    assert ctx._L.calls[0][1][2] == ok.data_ptr()


def test_positions_of_the_wrong_type_are_refused():
    n = 4
    ctx = _fake_context()  # mixed: float32 records
    with pytest.raises(GseError):
        ctx.spread_charge(n, np.zeros((n, 4), np.float64))
    with pytest.raises(GseError):
        ctx.spread_charge(n, np.zeros((n - 1, 4), np.float32))
    assert ctx._L.calls == []
