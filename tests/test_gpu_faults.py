"""Failure detection without a GPU fault.

* A device allocation that fails (injected on the host with
  ket_debug_fail_alloc) is reported as KET_ERR_OOM and leaves the context
  usable.
* The batched QAOA kernel waits on other CTAs with a bounded spin; the test
  hook drops one work item so that the tiles depending on it wait in vain.
  The wait gives up after a short limit, the call reports KET_ERR_TIMEOUT
  through the context's status word, and the next call runs normally.
* The staged pass kernels' wait for a tile's copies is bounded in time; the
  test hook skips one tile's copies and the call reports KET_ERR_TIMEOUT."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_alloc_failure_is_reported_and_context_survives():
    import ket_b200 as K
    from ket_b200 import _lib
    from ket_b200.circuit import DeviceState
    L = _lib.lib()
    L.ket_debug_fail_alloc(0)
    try:
        with pytest.raises(K.KetError) as ei:
            DeviceState(20)
        assert ei.value.code == _lib.KET_ERR_OOM
    finally:
        L.ket_debug_fail_alloc(-1)
    st = DeviceState(20)
    st.set_basis(0)
    st.apply(K.Circuit(20).h(0).cnot(0, 19).ops)
    a = st.amplitudes([0, 1 + (1 << 19)])
    assert abs(a[0] - 1 / math.sqrt(2)) < 1e-15 and abs(a[1] - 1 / math.sqrt(2)) < 1e-15


def test_batch_wait_times_out_and_recovers():
    import ket_b200 as K
    from ket_b200 import _lib
    from ket_b200.batch import batch_qaoa
    L = _lib.lib()
    edges = [(i, (i + 1) % 14) for i in range(14)]
    inst = [(14, edges, [0.3], [0.7])]
    L.ket_debug_batch_hook(0, 1 << 14)   # drop the first pass-0 tile: pass-1 tiles wait in vain
    try:
        with pytest.raises(K.KetError) as ei:
            batch_qaoa(inst, use_graph=False)
        assert ei.value.code == _lib.KET_ERR_TIMEOUT
    finally:
        L.ket_debug_batch_hook(-1, 0)
    got = batch_qaoa(inst, use_graph=False)
    from oracle import oracle as O
    c = O.qaoa(14, edges, [-0.6], [0.7])
    p = np.abs(c.simulate(mode=O.DENSE).dense()) ** 2
    x = np.arange(1 << 14)
    cut = np.zeros(1 << 14)
    for u, v in edges:
        cut += ((x >> u) ^ (x >> v)) & 1
    assert abs(got[0] - float(np.dot(p, cut))) < 1e-11


def test_staged_pass_wait_times_out_and_recovers():
    """The staged pass kernels' tile groups wait for each tile's copies with a
    bounded wait.  The test hook makes the issuing warp skip one tile, so that
    wait runs out (about two seconds), the group's threads stop together, the
    CTA waits for the copies it has in flight, and the call reports
    KET_ERR_TIMEOUT; the next call on the same context runs normally and
    matches the other form."""
    import ket_b200 as K
    from ket_b200 import _lib
    from ket_b200 import workloads as W
    from ket_b200.circuit import DeviceState, flatten_ops, ops_to_abi
    L = _lib.lib()
    c, _ = W.brickwork_circuit(16, 4, 3)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    st = DeviceState(16)
    st.set_basis(0)
    L.ket_debug_stage_drop(5)
    try:
        with pytest.raises(K.KetError) as ei:
            st.apply_abi(arr, m, k, specialize=1, stage=1)
        assert ei.value.code == _lib.KET_ERR_TIMEOUT
    finally:
        L.ket_debug_stage_drop(-1)
    st.set_basis(0)
    st.apply_abi(arr, m, k, specialize=1, stage=1)
    a = st.amplitudes_dense()
    st.set_basis(0)
    st.apply_abi(arr, m, k, specialize=1, stage=-1)
    assert np.array_equal(a, st.amplitudes_dense())
