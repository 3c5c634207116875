"""circuitMatrix() and blochAngles() on the engine: the reference's tests
(circuit.test.ts:6423-6513, :4745-4786) and parity with the oracle."""
import math

import numpy as np
import pytest

import ket_b200 as K
from ket_b200 import RangeError
from test_oracle_kats import BLOCH_KATS, MATRIX_KATS, _ocirc

pytestmark = pytest.mark.gpu


def kcirc(n, gates):
    c = K.Circuit(n)
    for name, qs, ps in gates:
        c = c.unitary(ps, *qs) if name == "unitary" else getattr(c, name)(*ps, *qs)
    return c


@pytest.mark.parametrize("kat", MATRIX_KATS, ids=[k[0] for k in MATRIX_KATS])
def test_circuit_matrix_kats(kat):
    _, n, gates, want = kat
    U = kcirc(n, gates).circuitMatrix()
    assert np.max(np.abs(U - want)) < 0.5e-10
    assert np.max(np.abs(U.conj().T @ U - np.eye(1 << n))) < 0.5e-10


def test_circuit_matrix_errors():
    with pytest.raises(TypeError):
        K.Circuit(1).h(0).creg("c", 1).measure(0, "c", 0).circuitMatrix()
    with pytest.raises(RangeError):
        K.Circuit(13).circuitMatrix()


def random_gates(n, depth, seed):
    rng = np.random.default_rng(seed)
    g = []
    for _ in range(depth):
        q = int(rng.integers(n))
        q2 = int((q + 1 + rng.integers(max(1, n - 1))) % n) if n > 1 else q
        r = rng.integers(5)
        if r == 0 or n == 1:
            g.append((["h", "t", "s", "x"][rng.integers(4)], [q], []))
        elif r == 1:
            g.append((["rx", "ry", "rz"][rng.integers(3)], [q], [float(rng.uniform(0, 2 * math.pi))]))
        elif r == 2:
            g.append(("cnot", [q, q2], []))
        elif r == 3:
            g.append(("cu3", [q, q2], [float(x) for x in rng.uniform(0, 2 * math.pi, 3)]))
        else:
            g.append(("xx", [q, q2], [float(rng.uniform(0, 2 * math.pi))]))
    return g


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 9])
def test_circuit_matrix_matches_oracle(n):
    g = random_gates(n, 6 * n, 100 + n)
    U = kcirc(n, g).circuitMatrix()
    V = _ocirc(n, g).circuit_matrix()
    assert np.max(np.abs(U - V)) < 1e-12


def test_circuit_matrix_12_qubits():
    """The largest size: sampled columns equal the oracle's one-column
    simulations, and the matrix is unitary up to the reference's per-gate
    pruning, which drops amplitudes below 1e-7 along the way (about 1e-7 of
    U^dagger U - I on this circuit, as in the reference)."""
    n = 12
    g = random_gates(n, 60, 7)
    U = kcirc(n, g).circuitMatrix()
    oc = _ocirc(n, g)
    flip = lambda i: int(format(i, f"0{n}b")[::-1], 2)  # noqa: E731
    perm = [flip(r) for r in range(1 << n)]
    for col in (0, 1, 777, 4095):
        want = oc.simulate(init=flip(col)).dense()[perm]
        d = np.max(np.abs(U[:, col] - want))
        assert d < 1e-12, (col, d)
    dev = np.max(np.abs(U.conj().T @ U - np.eye(1 << n)))
    assert dev < 1e-6, dev


@pytest.mark.parametrize("kat", BLOCH_KATS, ids=[k[0] for k in BLOCH_KATS])
def test_bloch_kats(kat):
    _, n, gates, theta, td, phi, pd = kat
    b = kcirc(n, gates).blochAngles(0)
    assert abs(b["theta"] - theta) < 0.5 * 10 ** -td
    if phi is not None:
        assert abs(b["phi"] - phi) < 0.5 * 10 ** -pd


def test_bloch_errors_and_parity():
    with pytest.raises(TypeError):
        K.Circuit(1).measure(0, "c", 0).blochAngles(0)
    n = 14
    g = random_gates(n, 80, 3)
    c = kcirc(n, g)
    st = _ocirc(n, g).simulate()
    for q in (0, 5, 13):
        b = c.blochAngles(q)
        o = st.bloch(q)
        assert abs(b["theta"] - o[4]) < 1e-12 and abs(b["phi"] - o[5]) < 1e-12
    with pytest.raises(RangeError):
        c.blochAngles(14)
