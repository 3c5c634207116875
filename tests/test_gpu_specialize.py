"""Pass kernels compiled per program (ket_exec_opts.specialize = 1) against the
interpreter k_fused2 (specialize = -1).  Below 26 qubits both run the same op
records with the same arithmetic, so the states must be equal bit for bit --
with the reference's pruning and without, in complex128 and complex64, over
every op kind the program generator emits (register, lane and warp targets,
register and thread controls, out-of-tile controls, phase fans, shared-memory
ops).  From 26 qubits on the compiled kernels' programs use 4 register bits."""
import ctypes as C

import numpy as np
import pytest

from test_gpu_parity import random_gates

pytestmark = pytest.mark.gpu


def _jit_stats():
    from ket_b200 import _lib
    out, cs = (C.c_int64 * 4)(), C.c_double()
    _lib.check(_lib.lib().ket_jit_stats(out, C.byref(cs)))
    return list(out)


def _run(n, arr, m, k, specialize, prune, precision=0, init=0):
    from ket_b200.circuit import DeviceState
    st = DeviceState(n, precision=precision)
    st.set_basis(init)
    st.apply_abi(arr, m, k, prune=prune, specialize=specialize)
    out = st.amplitudes_dense()
    del st
    return out


@pytest.mark.parametrize("n,seed", [(12, 1), (13, 2), (15, 3), (17, 4)])
@pytest.mark.parametrize("prune", [True, False])
def test_compiled_equals_interpreter_random(n, seed, prune):
    import ket_b200 as K
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c = K.Circuit(n)
    for name, qs, ps in random_gates(n, 160, seed):
        c = c.unitary(ps, *qs) if name == "unitary" else getattr(c, name)(*ps, *qs)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    before = _jit_stats()[3]
    got = _run(n, arr, m, k, 1, prune, init=seed * 977 % (1 << n))
    assert _jit_stats()[3] > before, "no compiled pass kernel ran"
    want = _run(n, arr, m, k, -1, prune, init=seed * 977 % (1 << n))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n", [20, 23])
def test_compiled_equals_interpreter_brickwork_qft(n):
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c, _ = W.brickwork_qft(n, 12, 42)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    got = _run(n, arr, m, k, 1, True)
    want = _run(n, arr, m, k, -1, True)
    assert np.array_equal(got, want)


def test_compiled_large_state_brickwork_bitwise():
    """From 26 qubits on compiled kernels run programs with 4 register bits
    (256 threads of 16 amplitudes), the interpreter keeps 5: the gates land
    on other roles, but a gate's register and lane forms round alike, so
    without phase fans the states are still equal bit for bit."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c, _ = W.brickwork_circuit(26, 6, 11)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    got = _run(26, arr, m, k, 1, True)
    want = _run(26, arr, m, k, -1, True)
    assert np.array_equal(got, want)


def test_compiled_large_state_brickwork_c64_bitwise():
    """The same at complex64 (FP32 gate arithmetic)."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c, _ = W.brickwork_circuit(26, 5, 13)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    got = _run(26, arr, m, k, 1, True, precision=1)
    want = _run(26, arr, m, k, -1, True, precision=1)
    assert np.array_equal(got, want)


def test_compiled_large_state_qft_to_rounding():
    """Merged phase fans group their factors by role, so with the QFT's fans
    the two register-bit counts agree to rounding."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c, _ = W.brickwork_qft(27, 3, 11)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    got = _run(27, arr, m, k, 1, False)
    want = _run(27, arr, m, k, -1, False)
    assert np.max(np.abs(got - want)) < 1e-13


def test_compiled_large_state_random_gates_to_rounding():
    """Every op kind at 4 register bits (shared-memory ops, controlled gates,
    multi-qubit unitaries) against the interpreter's 5-bit programs."""
    import ket_b200 as K
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c = K.Circuit(26)
    for name, qs, ps in random_gates(26, 90, 26):
        c = c.unitary(ps, *qs) if name == "unitary" else getattr(c, name)(*ps, *qs)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    # without pruning: a last-bit difference from a phase fan next to the
    # 1e-7 threshold could flip a prune decision
    got = _run(26, arr, m, k, 1, False, init=12345)
    want = _run(26, arr, m, k, -1, False, init=12345)
    assert np.max(np.abs(got - want)) < 1e-13


def test_compiled_equals_interpreter_c64():
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c, _ = W.brickwork_qft(18, 8, 7)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    got = _run(18, arr, m, k, 1, True, precision=1)
    want = _run(18, arr, m, k, -1, True, precision=1)
    assert np.array_equal(got, want)


def test_automatic_policy_uses_ready_kernels():
    """specialize = 0 runs a compiled kernel once one for the program's shape is
    in the cache (the first call compiled it), and the result is unchanged."""
    from ket_b200 import _lib
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c, _ = W.brickwork_qft(26, 2, 3)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    want = _run(26, arr, m, k, 1, True)
    _lib.check(_lib.lib().ket_jit_wait())
    before = _jit_stats()[3]
    got = _run(26, arr, m, k, 0, True)
    assert _jit_stats()[3] > before
    assert np.array_equal(got, want)


def test_kernels_compiled_ahead_serve_the_default_policy():
    """Below 26 qubits the default policy compiles nothing itself, but uses
    kernels compiled ahead of time (Circuit.compile_kernels)."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c, _ = W.brickwork_qft(15, 6, 77)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    want = _run(15, arr, m, k, -1, True)
    assert c.compile_kernels() >= 1
    before = _jit_stats()[3]
    got = _run(15, arr, m, k, 0, True)
    assert _jit_stats()[3] > before
    assert np.array_equal(got, want)
