"""The staged form of the compiled pass kernels (ket_exec_opts.stage = 1):
every tile is brought into shared memory by tensor-memory-accelerator copies
issued ahead of use, one CTA per SM with two tile groups sharing three
stages, instead of per-thread loads into registers.  The program, the layouts and the arithmetic are the same, so
the two forms must give equal states bit for bit -- over every op kind, with
and without the reference's pruning, in both precisions, down to a state of
one tile -- and the staged form must match the oracle to 1e-12."""
import ctypes as C

import numpy as np
import pytest

from test_gpu_parity import build_both, random_gates

pytestmark = pytest.mark.gpu


def _launches():
    from ket_b200 import _lib
    out, cs = (C.c_int64 * 4)(), C.c_double()
    _lib.check(_lib.lib().ket_jit_stats(out, C.byref(cs)))
    return out[3]


def _run(n, circ, stage, prune=True, precision=0, init=0, reg_bits=0):
    from ket_b200.circuit import DeviceState, flatten_ops, ops_to_abi
    arr, m, k = ops_to_abi(flatten_ops(circ.ops))
    st = DeviceState(n, precision=precision)
    st.set_basis(init)
    before = _launches()
    st.apply_abi(arr, m, k, prune=prune, specialize=1, reg_bits=reg_bits, stage=stage)
    assert _launches() > before, "no compiled pass kernel ran"
    out = st.amplitudes_dense()
    del st
    return out


@pytest.mark.parametrize("n,seed", [(12, 41), (13, 42), (15, 43), (17, 44)])
@pytest.mark.parametrize("prune", [True, False])
@pytest.mark.parametrize("reg_bits", [4, 5])
def test_staged_equals_register_loads_random(n, seed, prune, reg_bits):
    import ket_b200 as K
    c = K.Circuit(n)
    for name, qs, ps in random_gates(n, 160, seed):
        c = c.unitary(ps, *qs) if name == "unitary" else getattr(c, name)(*ps, *qs)
    init = seed * 131 % (1 << n)
    a = _run(n, c, 1, prune, init=init, reg_bits=reg_bits)
    b = _run(n, c, -1, prune, init=init, reg_bits=reg_bits)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("n,seed", [(14, 51), (16, 52)])
def test_staged_vs_sparse_oracle(n, seed):
    from oracle import oracle as O
    kc, oc = build_both(n, random_gates(n, 200, seed))
    want = oc.simulate(mode=O.SPARSE).dense()
    got = _run(n, kc, 1, reg_bits=4)
    assert np.max(np.abs(got - want)) < 1e-12


def test_staged_workload_family_26q():
    from ket_b200 import workloads as W
    c, _ = W.brickwork_qft(26, 8, 42)
    assert np.array_equal(_run(26, c, 1), _run(26, c, -1))


def test_staged_c64():
    from ket_b200 import workloads as W
    c, _ = W.brickwork_qft(20, 10, 9)
    assert np.array_equal(_run(20, c, 1, precision=1), _run(20, c, -1, precision=1))
