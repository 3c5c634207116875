"""The oracle pinned against the reference's own known answers.

Every case in tests/golden/reference_kats.json restates a test of the
reference suite (dmvjs/ket src/circuit.test.ts) with its expected value and
digit count; the oracle must reproduce all of them in its sparse mode (the
reference's own data structure and pruning) and in its dense modes.
"""
import math

import numpy as np
import pytest

from harness import (bit_index, check_pershot, init_index, load_kats, load_pershot_kats, oracle_circuit,
                     pershot_oracle_raw, summarize, tol)
from oracle import oracle as O

CASES = load_kats()


def eval_oracle(case, mode):
    c = oracle_circuit(case)
    st = c.simulate(init=init_index(case), mode=mode)
    idx, p = st.exact_probs()
    probs = {format(int(i), "b").zfill(case["n"])[::-1]: float(v) for i, v in zip(idx, p)}
    for chk in case["checks"]:
        kind = chk[0]
        if kind == "amp":
            a = st.amplitude(bit_index(chk[1]))
            assert abs(a.real - chk[2]) < tol(chk[4]), (case["id"], chk, a)
            assert abs(a.imag - chk[3]) < tol(chk[4]), (case["id"], chk, a)
        elif kind == "prob":
            assert abs(probs.get(chk[1], 0.0) - chk[2]) < tol(chk[3]), (case["id"], chk, probs)
        elif kind == "nkeys":
            assert len(probs) == chk[1], (case["id"], probs)
        elif kind == "uniform":
            assert all(abs(v - chk[1]) < tol(chk[2]) for v in probs.values())
        elif kind == "marg":
            m = st.marginals()
            assert abs(m[chk[1]] - chk[2]) < tol(chk[3])
        elif kind == "norm":
            assert abs(sum(probs.values()) - 1.0) < tol(chk[1])
        elif kind == "vqe":
            e = c.vqe([(t[0], t[1]) for t in chk[1]], mode=mode)
            assert abs(e - chk[2]) < tol(chk[3]), (case["id"], e)
        elif kind == "expect":
            # the reference's expectation() starts from |0..0>
            e = c.expectation(chk[1], mode=mode)
            assert abs(e - chk[2]) < tol(chk[3]), (case["id"], e)
        else:
            raise AssertionError(kind)


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_kat_sparse(case):
    eval_oracle(case, O.SPARSE)


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_kat_dense(case):
    eval_oracle(case, O.DENSE)


def test_gradient_kats():
    """gradient() parameter-shift KATs (circuit.test.ts:4168-4219)."""
    Z = [(1.0, "Z")]
    # realAmplitudes(1, 0) is exactly ry(p0, 0)
    for theta, want in [(0.0, 0.0), (math.pi / 4, -math.sin(math.pi / 4)), (math.pi, 0.0)]:
        g = O.gradient(O.ANS_REAL_AMPLITUDES, 1, 0, [theta], Z)
        assert abs(g[0] - want) < tol(10)
    p0, p1 = math.pi / 3, math.pi / 6
    g = O.gradient(O.ANS_REAL_AMPLITUDES, 2, 0, [p0, p1], [(1.0, "ZI"), (1.0, "IZ")])
    assert abs(g[0] + math.sin(p0)) < tol(10) and abs(g[1] + math.sin(p1)) < tol(10)
    g1 = O.gradient(O.ANS_REAL_AMPLITUDES, 1, 0, [math.pi / 5], [(1.0, "Z")])
    g2 = O.gradient(O.ANS_REAL_AMPLITUDES, 1, 0, [math.pi / 5], [(2.0, "Z")])
    assert abs(g2[0] - 2 * g1[0]) < tol(10)


def test_minimize_kats():
    """minimize() KATs (circuit.test.ts:4239-4262)."""
    r = O.minimize(O.ANS_REAL_AMPLITUDES, 1, 0, [0.1], [(1.0, "Z")])
    assert abs(r["energy"] + 1) < tol(4) and r["converged"]
    r = O.minimize(O.ANS_REAL_AMPLITUDES, 2, 0, [0.1, 0.1], [(1.0, "ZZ"), (0.5, "ZI")], lr=0.2, steps=500)
    assert abs(r["energy"] + 1.5) < tol(3) and r["converged"]
    r = O.minimize(O.ANS_REAL_AMPLITUDES, 1, 0, [0.1], [(1.0, "Z")], steps=1)
    assert not r["converged"] and r["steps"] == 1
    r = O.minimize(O.ANS_REAL_AMPLITUDES, 1, 0, [math.pi], [(1.0, "Z")])
    assert r["converged"] and r["steps"] == 0


def test_qaoa_4cycle():
    """qaoa + maxCutHamiltonian on the 4-cycle (circuit.test.ts:6373-6421)."""
    edges = [(0, 1), (1, 2), (2, 3), (3, 0)]
    H = O.maxcut_hamiltonian(4, edges)
    assert H[0] == (2.0, "IIII") and len(H) == 5
    idx, p = O.qaoa(4, edges, [], []).simulate().exact_probs()
    assert len(idx) == 16 and all(abs(v - 1 / 16) < tol(10) for v in p)
    st = O.qaoa(4, edges, [math.pi / 4], [0.15 * math.pi]).simulate()
    probs = dict(zip([int(i) for i in st.exact_probs()[0]], st.exact_probs()[1]))
    assert probs.get(0b0101, 0) > 0.20 and probs.get(0b1010, 0) > 0.20   # '1010' and '0101'
    assert O.qaoa(4, edges, [math.pi / 4], [0.15 * math.pi]).vqe(H) > 2.5
    assert abs(O.OCircuit(4).vqe(H)) < tol(10)
    assert O.maxcut_hamiltonian(3, []) == []


def test_bigint_indices_sparse():
    """Qubits 30, 31 and 40 (circuit.test.ts:482-505) on the sparse oracle."""
    c = O.OCircuit(31).add("h", [0]).add("cnot", [0, 30])
    idx, p = c.simulate().exact_probs()
    assert list(idx) == [0, (1 << 30) | 1]
    c = O.OCircuit(32).add("h", [0]).add("cnot", [0, 31])
    idx, _ = c.simulate().exact_probs()
    assert list(idx) == [0, (1 << 31) | 1]
    c = O.OCircuit(41).add("x", [40])
    idx, p = c.simulate().exact_probs()
    assert list(idx) == [1 << 40] and p[0] == 1.0


def test_bounds_errors():
    """#checkOp errors (circuit.test.ts:507-552)."""
    with pytest.raises(O.OracleRangeError):
        O.OCircuit(2).add("h", [-1])
    with pytest.raises(O.OracleRangeError):
        O.OCircuit(2).add("x", [2])
    with pytest.raises(O.OracleRangeError):
        O.OCircuit(2).add("cnot", [5, 1])
    with pytest.raises(O.OracleRangeError):
        O.OCircuit(3).add("ccx", [0, 1, 3])
    with pytest.raises(O.OracleTypeError):
        O.OCircuit(2).add("cnot", [1, 1])
    with pytest.raises(O.OracleTypeError):
        O.OCircuit(2).add("crx", [0, 0], [0.5])


PERSHOT = load_pershot_kats()


def pure_oracle_probs(case):
    """run()'s pure fast path on the case's gates with the same seed."""
    c = O.OCircuit(case["n"])
    for op in case["ops"]:
        c.add(op[0], op[1], op[2])
    idx = c.simulate().run(case["run"]["shots"], case["run"]["seed"])
    probs = {}
    for i in idx.tolist():
        k = format(int(i), "b").zfill(case["n"])[::-1]
        probs[k] = probs.get(k, 0) + 1 / len(idx)
    return probs


@pytest.mark.parametrize("case", PERSHOT, ids=[c["id"] for c in PERSHOT])
def test_pershot_kat_oracle(case):
    """run()'s per-shot path (circuit.ts:3455-3481) on the oracle against the
    reference's measure / reset / if / noise tests."""
    idx, bits, regs = pershot_oracle_raw(case)
    probs, cregs = summarize(case["n"], idx, bits, regs)
    clean = pure_oracle_probs(case) if any(c[0] == "like_clean" for c in case["checks"]) else None
    check_pershot(case, probs, cregs, clean)


def _xorshift(s, k):
    for _ in range(k):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
    return s


def test_pershot_draw_order():
    """Draws per shot follow applyOps: one per measure / reset, one more per
    measure when pMeas != 0, one per noisy gate, one for sampleSV, then n
    readout draws when pMeas != 0; an if-body draws only when it runs."""
    c = O.OCircuit(2).add("h", [0]).add("cnot", [0, 1])
    c.measure(0, 0)
    c.reset(1)
    _, _, st = c.run_pershot(10, 7, 0.0, 0.0, 0.0, 1)
    assert st == _xorshift(7, 10 * 3)
    _, _, st = c.run_pershot(10, 7, 0.1, 0.2, 0.3, 1)
    assert st == _xorshift(7, 10 * (1 + 1 + 1 + 1 + 1 + 1 + 2))
    # if-body with a noisy gate: x(1) runs only when bit 0 reads 1
    d = O.OCircuit(2)
    d.measure(0, 0)
    d.if_(0, 1, 1, O.OCircuit(2).add("x", [1]))
    _, _, st = d.run_pershot(5, 9, 0.5, 0.0, 0.0, 1, init=1)  # q0 = 1: always taken
    assert st == _xorshift(9, 5 * (1 + 1 + 1))
    _, _, st = d.run_pershot(5, 9, 0.5, 0.0, 0.0, 1, init=0)  # never taken
    assert st == _xorshift(9, 5 * (1 + 1))


# circuitMatrix() / blochAngles() (circuit.test.ts:6423-6513, :4745-4786), restated
S2 = 1 / math.sqrt(2)
MATRIX_KATS = [
    ("identity", 2, [], np.eye(4)),
    ("h", 1, [("h", [0], [])], np.array([[S2, S2], [S2, -S2]])),
    ("x", 1, [("x", [0], [])], np.array([[0, 1], [1, 0]])),
    ("s", 1, [("s", [0], [])], np.array([[1, 0], [0, 1j]])),
    ("cnot_unitary", 2, [("unitary", [0, 1], np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]]))],
     np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]])),
    ("h_unitary", 1, [("unitary", [0], np.array([[S2, S2], [S2, -S2]]))], np.array([[S2, S2], [S2, -S2]])),
]
BLOCH_KATS = [  # (id, n, gates, theta, theta digits, phi or None, phi digits)
    ("zero", 1, [], 0.0, 10, None, 0),
    ("one", 1, [("x", [0], [])], math.pi, 10, None, 0),
    ("plus", 1, [("h", [0], [])], math.pi / 2, 8, 0.0, 8),
    ("rx", 1, [("rx", [0], [math.pi / 2])], math.pi / 2, 8, -math.pi / 2, 8),
    ("ry", 1, [("ry", [0], [math.pi / 3])], math.pi / 3, 8, None, 0),
    ("bell", 2, [("h", [0], []), ("cnot", [0, 1], [])], math.pi / 2, 8, None, 0),
]


def _ocirc(n, gates):
    c = O.OCircuit(n)
    for name, qs, ps in gates:
        if name == "unitary":
            c.unitary(ps, qs)
        else:
            c.add(name, qs, ps)
    return c


@pytest.mark.parametrize("kat", MATRIX_KATS, ids=[k[0] for k in MATRIX_KATS])
def test_circuit_matrix_kats_oracle(kat):
    _, n, gates, want = kat
    U = _ocirc(n, gates).circuit_matrix()
    assert np.max(np.abs(U - want)) < tol(10)
    assert np.max(np.abs(U.conj().T @ U - np.eye(1 << n))) < tol(10)


@pytest.mark.parametrize("kat", BLOCH_KATS, ids=[k[0] for k in BLOCH_KATS])
def test_bloch_kats_oracle(kat):
    _, n, gates, theta, td, phi, pd = kat
    out = _ocirc(n, gates).simulate().bloch(0)
    assert abs(out[4] - theta) < tol(td)
    if phi is not None:
        assert abs(out[5] - phi) < tol(pd)


# dm() (circuit.test.ts:5017-5245), restated: (id, n, gates, noise {p1, p2}, checks)
#   ("purity", x, digits) ("purity_lt", x) ("prob", bits, x, digits) ("absent", bits)
#   ("entropy", x, digits) ("entropy_in", lo, hi) ("theta", x, digits) ("phi", x, digits)
#   ("get", row, col, re, digits) ("total", x, digits)
H0 = ("h", [0], [])
BELL = [H0, ("cnot", [0, 1], [])]
DM_KATS = [
    ("pure0", 1, [], None, [("purity", 1, 10), ("prob", "0", 1, 10), ("absent", "1"), ("entropy", 0, 10),
                            ("theta", 0, 10), ("get", 0, 0, 1, 10), ("get", 1, 1, 0, 10), ("get", 0, 1, 0, 10)]),
    ("pure1", 1, [("x", [0], [])], None, [("purity", 1, 10), ("absent", "0"), ("prob", "1", 1, 10),
                                          ("theta", math.pi, 10)]),
    ("plus", 1, [H0], None, [("purity", 1, 10), ("prob", "0", 0.5, 10), ("prob", "1", 0.5, 10), ("entropy", 0, 10),
                             ("theta", math.pi / 2, 10), ("phi", 0, 10)]),
    ("bell", 2, BELL, None, [("purity", 1, 10), ("prob", "00", 0.5, 10), ("prob", "11", 0.5, 10), ("absent", "01"),
                             ("absent", "10"), ("entropy", 0, 10)]),
    ("hhh", 3, [H0, ("h", [1], []), ("h", [2], [])], None, [("prob", "000", 0.125, 10), ("prob", "111", 0.125, 10)]),
    ("noisy_h", 1, [H0], {"p1": 0.1}, [("purity_lt", 1), ("get", 0, 1, (1 - 4 * 0.1 / 3) * 0.5, 8)]),
    ("p1_zero", 1, [H0], {"p1": 0}, [("purity", 1, 10)]),
    ("noisy_bell", 2, BELL, {"p2": 0.05}, [("purity_lt", 1)]),
    ("dep_02", 1, [H0], {"p1": 0.2}, [("entropy_in", 0, 1)]),
    ("max_mixed", 1, [H0], {"p1": 0.75}, [("entropy", 1, 6)]),
    ("noisy_total", 2, BELL, {"p1": 0.05, "p2": 0.05}, [("total", 1, 8)]),
    ("ccx", 3, [("x", [0], []), ("x", [1], []), ("ccx", [0, 1, 2], [])], None, [("purity", 1, 10), ("prob", "111", 1, 10)]),
    ("ccx_off", 3, [("x", [2], []), ("ccx", [0, 1, 2], [])], None, [("prob", "001", 1, 10)]),
    ("cswap", 3, [("x", [0], []), ("x", [2], []), ("cswap", [0, 1, 2], [])], None, [("prob", "110", 1, 10)]),
    ("cswap_off", 3, [("x", [2], []), ("cswap", [0, 1, 2], [])], None, [("prob", "001", 1, 10)]),
]


def check_dm(case, probs, purity, entropy, bloch, get):
    for chk in case[4]:
        k = chk[0]
        if k == "purity":
            assert abs(purity - chk[1]) < tol(chk[2]), (case[0], purity)
        elif k == "purity_lt":
            assert purity < chk[1], (case[0], purity)
        elif k == "prob":
            assert abs(probs.get(chk[1], 0.0) - chk[2]) < tol(chk[3]), (case[0], probs)
        elif k == "absent":
            assert chk[1] not in probs, (case[0], probs)
        elif k == "entropy":
            assert abs(entropy() - chk[1]) < tol(chk[2]), case[0]
        elif k == "entropy_in":
            assert chk[1] < entropy() < chk[2], case[0]
        elif k == "theta":
            assert abs(bloch(0)[0] - chk[1]) < tol(chk[2]), case[0]
        elif k == "phi":
            assert abs(bloch(0)[1] - chk[1]) < tol(chk[2]), case[0]
        elif k == "get":
            assert abs(get(chk[1], chk[2]).real - chk[3]) < tol(chk[4]), case[0]
        elif k == "total":
            assert abs(sum(probs.values()) - chk[1]) < tol(chk[2]), case[0]
        else:
            raise AssertionError(k)


@pytest.mark.parametrize("case", DM_KATS, ids=[c[0] for c in DM_KATS])
def test_dm_kats_oracle(case):
    _, n, gates, noise, _ = case
    nz = noise or {}
    d = _ocirc(n, gates).dm(nz.get("p1", 0.0), nz.get("p2", 0.0))
    dense = d.dense()
    check_dm(case, d.probabilities(), d.purity(), d.entropy, d.bloch, lambda r, c: dense[r, c])


def test_dm_noise_ordering_oracle():
    """circuit.test.ts:5147-5153, :5175-5186: purity falls with noise; forte-1 is
    cleaner than harmony; aria-1 is noisier than none."""
    ps = [_ocirc(1, [H0]).dm(p, 0).purity() for p in (0.01, 0.1, 0.3)]
    assert ps[0] > ps[1] > ps[2]
    forte = _ocirc(2, BELL).dm(0.0001, 0.002).purity()
    harmony = _ocirc(2, BELL).dm(0.001, 0.015).purity()
    assert forte > harmony
    assert _ocirc(2, BELL).dm(0.0003, 0.005).purity() < _ocirc(2, BELL).dm().purity()


def test_sparse_oracle_agrees_with_dense_prune_on_the_family():
    """DENSE_PRUNE is the reference's pruning on a dense array: on the
    workload's family it gives the sparse map's amplitudes, so it stands in
    for the sparse mode where a Map of 2^26 entries is too slow."""
    from oracle import oracle as O
    oc, _ = O.brickwork(16, 20, 42, with_qft=True)
    a = oc.simulate(mode=O.SPARSE).dense()
    b = oc.simulate(mode=O.DENSE_PRUNE).dense()
    assert np.array_equal(a, b)
