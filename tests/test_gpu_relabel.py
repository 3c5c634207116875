"""Uncontrolled swaps of two qubits of a tile run as relabellings of the tile
layout (FO_RELAY): no data moves, the exchange offsets and the store layout
name the qubits anew.  Checked on a random dense state against a numpy
permutation of the amplitudes, on both forms of the pass (compiled kernels and
the interpreter), with swap patterns that touch the tile's lane bits (qubits
0-4), its high bits and both, alone and mixed with gates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _swap_np(a, n, p, q):
    t = a.reshape([2] * n)  # axis k is qubit n - 1 - k
    return np.swapaxes(t, n - 1 - p, n - 1 - q).reshape(-1)


def _apply(n, a0, circ, specialize, prune=True):
    from ket_b200.circuit import DeviceState, flatten_ops, ops_to_abi
    arr, m, k = ops_to_abi(flatten_ops(circ.ops))
    st = DeviceState(n)
    st.set_amplitudes(a0)
    st.apply_abi(arr, m, k, prune=prune, specialize=specialize)
    out = st.amplitudes_dense()
    del st
    return out


PATTERNS = {
    "qft_tail": lambda n: [(i, n - 1 - i) for i in range(n // 2)],
    "high_only": lambda n: [(6, 13), (9, n - 1), (7, 12)],
    "lane_high": lambda n: [(0, 9), (3, n - 2), (1, 2)],
    "chain": lambda n: [(5, 6), (6, 7), (7, 8), (0, 5)],
}


@pytest.mark.parametrize("n", [14, 18, 23])
@pytest.mark.parametrize("pattern", sorted(PATTERNS))
@pytest.mark.parametrize("specialize", [1, -1])
def test_swaps_permute_the_state(n, pattern, specialize):
    import ket_b200 as K
    rng = np.random.default_rng(n)
    a0 = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    a0 /= np.linalg.norm(a0)
    c = K.Circuit(n)
    want = a0.copy()
    for p, q in PATTERNS[pattern](n):
        c = c.swap(p, q)
        want = _swap_np(want, n, p, q)
    got = _apply(n, a0, c, specialize)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n", [16, 23])
def test_swaps_between_gates_both_forms(n):
    """Swaps interleaved with mixing gates and CNOTs on the swapped qubits:
    the compiled kernels equal the interpreter bit for bit and the oracle to
    1e-12."""
    import ket_b200 as K
    from oracle import oracle as O
    rng = np.random.default_rng(7)
    c = K.Circuit(n)
    oc = O.OCircuit(n)
    for layer in range(6):
        for q in range(n):
            th = float(rng.uniform(0, 6.28))
            c = c.ry(th, q)
            oc.add("ry", [q], [th])
        for q in range(layer % 2, n - 1, 2):
            c = c.cnot(q, q + 1)
            oc.add("cnot", [q, q + 1])
        for p, q in PATTERNS["qft_tail" if layer % 2 else "lane_high"](n):
            c = c.swap(p, q)
            oc.add("swap", [p, q])
    a0 = np.zeros(1 << n, complex)
    a0[3] = 1
    got = _apply(n, a0, c, 1)
    assert np.array_equal(got, _apply(n, a0, c, -1))
    want = oc.simulate(init=3, mode=O.DENSE_PRUNE).dense()
    assert np.max(np.abs(got - want)) < 1e-12
