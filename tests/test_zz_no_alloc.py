"""ket_marginals_noalloc against an independent numpy marginal sum and against
ket_marginals on the same amplitudes.

The caller owns every device buffer (allocated here with torch, as a caller
with its own allocator would); the entry point itself allocates nothing and
keeps its scratch in a fixed device array shared by all calls.  Two calls in a
row check that leftovers of the previous call do not leak into the next.
Both precisions run through it: complex64 amplitudes are summed in FP64, so
the numpy sum over the same float32 values agrees to 1e-12 as well.  n = 24
fills 24 of the array's 40 qubit columns over 2048 blocks.
This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _numpy_marginals(n, a):
    p = np.abs(a.astype(np.complex128)) ** 2
    idx = np.arange(1 << n, dtype=np.int64)
    return np.array([p[(idx >> q) & 1 == 1].sum() for q in range(n)])


def _engine_marginals(n, a):
    from ket_b200.circuit import DeviceState
    st = DeviceState(n)
    st.set_amplitudes(a.astype(np.complex128))
    return np.asarray(st.marginals())


@pytest.mark.parametrize("precision", ["c128", "c64"])
@pytest.mark.parametrize("n", [9, 17, 24])
def test_marginals_noalloc_matches_marginals(n, precision):
    import torch
    from ket_b200 import _lib
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(n)
    prec = _lib.KET_C128 if precision == "c128" else _lib.KET_C64
    dt = np.float64 if precision == "c128" else np.float32
    outs = []
    for call in range(2):
        a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        if call == 1:
            a[::3] = 0  # a different state: the second call must not see the first one's sums
        a /= np.linalg.norm(a)
        if precision == "c64":
            a = a.astype(np.complex64)
        want = _numpy_marginals(n, a)
        inter = np.stack([a.real, a.imag], axis=1).reshape(-1).astype(dt)
        d_amp = torch.from_numpy(inter.copy()).to(dev)
        d_out = torch.full((n,), -1.0, dtype=torch.float64, device=dev)
        _lib.check(L.ket_marginals_noalloc(C.c_void_p(d_amp.data_ptr()), n, prec,
                                           C.c_void_p(d_out.data_ptr()), C.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize(dev)
        got = d_out.cpu().numpy()
        assert np.max(np.abs(got - want)) < TOL
        if precision == "c128":
            assert np.max(np.abs(got - _engine_marginals(n, a))) < TOL
        outs.append(got)
    assert not np.array_equal(outs[0], outs[1])


def test_marginals_noalloc_rejects_bad_arguments():
    import torch
    from ket_b200 import _lib
    L = _lib.lib()
    assert L.ket_marginals_noalloc(None, 10, _lib.KET_C128, None, None) == 2
    assert L.ket_marginals_noalloc(C.c_void_p(16), 41, _lib.KET_C128, C.c_void_p(16), None) == 1
    assert L.ket_marginals_noalloc(C.c_void_p(16), 10, 7, C.c_void_p(16), None) == 2
    # host memory is refused before anything reaches the GPU
    h_amp = torch.zeros(2 << 10, dtype=torch.float64)
    d_out = torch.zeros(10, dtype=torch.float64, device="cuda:0")
    assert L.ket_marginals_noalloc(C.c_void_p(h_amp.data_ptr()), 10, _lib.KET_C128,
                                   C.c_void_p(d_out.data_ptr()), None) == 2
    d_amp = torch.zeros(2 << 10, dtype=torch.float64, device="cuda:0")
    h_out = torch.zeros(10, dtype=torch.float64)
    assert L.ket_marginals_noalloc(C.c_void_p(d_amp.data_ptr()), 10, _lib.KET_C128,
                                   C.c_void_p(h_out.data_ptr()), None) == 2
