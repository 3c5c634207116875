"""ket_marginals_noalloc against ket_marginals on the same amplitudes.

The caller owns every device buffer (allocated here with torch, as a caller
with its own allocator would); the entry point itself allocates nothing and
keeps its scratch in a fixed device array shared by all calls.  Two calls in a
row check that leftovers of the previous call do not leak into the next.
This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _marginals_ref(n, amps):
    from ket_b200.circuit import DeviceState
    st = DeviceState(n)
    st.set_amplitudes(amps)
    return st.marginals()


@pytest.mark.parametrize("n", [9, 17, 22])
def test_marginals_noalloc_matches_marginals(n):
    import torch
    from ket_b200 import _lib
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(n)
    outs = []
    for call in range(2):
        a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        if call == 1:
            a[::3] = 0  # a different state: the second call must not see the first one's sums
        a /= np.linalg.norm(a)
        want = np.asarray(_marginals_ref(n, a))
        d_amp = torch.from_numpy(np.stack([a.real, a.imag], axis=1).reshape(-1).copy()).to(dev)
        d_out = torch.full((n,), -1.0, dtype=torch.float64, device=dev)
        _lib.check(L.ket_marginals_noalloc(C.c_void_p(d_amp.data_ptr()), n, _lib.KET_C128,
                                           C.c_void_p(d_out.data_ptr()), C.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize(dev)
        got = d_out.cpu().numpy()
        assert np.max(np.abs(got - want)) < 1e-12
        outs.append(got)
    assert not np.array_equal(outs[0], outs[1])


def test_marginals_noalloc_rejects_bad_arguments():
    from ket_b200 import _lib
    L = _lib.lib()
    assert L.ket_marginals_noalloc(None, 10, _lib.KET_C128, None, None) == 2
    assert L.ket_marginals_noalloc(C.c_void_p(16), 41, _lib.KET_C128, C.c_void_p(16), None) == 1
    assert L.ket_marginals_noalloc(C.c_void_p(16), 10, 7, C.c_void_p(16), None) == 2
