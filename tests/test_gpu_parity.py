"""GPU engine against the oracle on seeded random circuits and on the
benchmark circuit families, through the public Circuit API.

Tolerances: complex128 amplitudes and probabilities within 1e-12 of the
oracle (the bar the engine is held to); shot indices bit-exact where the
reference's summation order is reproduced (2^n <= 2^20)."""
import math
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AMP_TOL = 1e-12

GATES1 = ["h", "x", "y", "z", "s", "si", "t", "ti", "v", "vi", "r2", "r4", "r8", "id"]
GATES1P = {"rx": 1, "ry": 1, "rz": 1, "u1": 1, "p": 1, "u2": 2, "u3": 3, "gpi": 1, "gpi2": 1, "vz": 1}
GATES2 = ["cnot", "swap", "iswap", "srswap", "cy", "cz", "ch", "cs", "ct", "csdg", "ctdg", "csrn", "cr2", "cr4", "cr8"]
GATES2P = {"xx": 1, "yy": 1, "zz": 1, "xy": 1, "ms": 2, "crx": 1, "cry": 1, "crz": 1, "cu1": 1, "cu2": 2, "cu3": 3}
GATES3 = ["ccx", "cswap", "csrswap"]


def random_gates(n, count, seed, unitary=True):
    rnd = random.Random(seed)
    out = []
    for _ in range(count):
        r = rnd.random()
        if r < 0.35:
            out.append((rnd.choice(GATES1), [rnd.randrange(n)], []))
        elif r < 0.6:
            g = rnd.choice(list(GATES1P))
            out.append((g, [rnd.randrange(n)], [rnd.uniform(-math.pi, 2 * math.pi) for _ in range(GATES1P[g])]))
        elif r < 0.75 and n >= 2:
            a, b = rnd.sample(range(n), 2)
            out.append((rnd.choice(GATES2), [a, b], []))
        elif r < 0.9 and n >= 2:
            g = rnd.choice(list(GATES2P))
            a, b = rnd.sample(range(n), 2)
            out.append((g, [a, b], [rnd.uniform(0, 2 * math.pi) for _ in range(GATES2P[g])]))
        elif r < 0.97 and n >= 3:
            out.append((rnd.choice(GATES3), rnd.sample(range(n), 3), []))
        elif unitary and n >= 3:
            k = rnd.choice([1, 2, 3])
            qs = rnd.sample(range(n), k)
            m = np.linalg.qr(np.random.default_rng(rnd.randrange(1 << 30)).normal(size=(2 ** k, 2 ** k))
                             + 1j * np.random.default_rng(rnd.randrange(1 << 30)).normal(size=(2 ** k, 2 ** k)))[0]
            out.append(("unitary", qs, m))
    return out


def build_both(n, gates):
    import ket_b200 as K
    from oracle import oracle as O
    kc, oc = K.Circuit(n), O.OCircuit(n)
    for name, qs, ps in gates:
        if name == "unitary":
            kc = kc.unitary(ps, *qs)
            oc.unitary(ps, qs)
        else:
            kc = getattr(kc, name)(*ps, *qs)
            oc.add(name, qs, ps)
    return kc, oc


@pytest.mark.parametrize("n,seed", [(1, 1), (2, 2), (3, 3), (5, 4), (7, 5), (9, 6), (11, 7), (12, 8), (13, 9),
                                    (14, 10), (15, 11)])
def test_random_circuits_vs_oracle(n, seed):
    from oracle import oracle as O
    gates = random_gates(n, 60 + 10 * n, seed)
    kc, oc = build_both(n, gates)
    init = random.Random(seed).randrange(1 << n)
    want = oc.simulate(init=init, mode=O.SPARSE).dense()
    bs = format(init, "b").zfill(n)[::-1]
    got = kc.statevector_array(initialState=bs)
    assert np.max(np.abs(got - want)) < AMP_TOL
    # every fusion setting and the unfused path give the same state
    for fusion in (0, 6, 8, 10):
        st = kc._state(bs, fusion=fusion)
        assert np.max(np.abs(st.amplitudes_dense() - want)) < AMP_TOL, fusion


@pytest.mark.parametrize("n,seed", [(10, 21), (13, 22), (16, 23)])
def test_prune_off_matches_dense_oracle(n, seed):
    from oracle import oracle as O
    gates = random_gates(n, 120, seed, unitary=False)
    kc, oc = build_both(n, gates)
    want = oc.simulate(mode=O.DENSE).dense()
    got = kc._state(None, prune=False).amplitudes_dense()
    assert np.max(np.abs(got - want)) < AMP_TOL


def test_config1_brickwork16_exactprobs_and_shots():
    """16q brickwork, 20 layers, seed 42: exactProbs and 4096 shots at seed 42
    equal the reference algorithm's (sparse oracle) -- shots index for index."""
    from ket_b200 import workloads as W
    from oracle import oracle as O
    kc, _ = W.brickwork_circuit(16, 20, 42)
    oc, _ = O.brickwork(16, 20, 42)
    st = oc.simulate(mode=O.SPARSE)
    oidx, op = st.exact_probs()
    probs = kc.exactProbs()
    assert len(probs) == len(oidx)
    got = np.array([probs[format(int(i), "b").zfill(16)[::-1]] for i in oidx])
    assert np.max(np.abs(got - op)) < AMP_TOL
    shots_ref = st.run(4096, 42)
    dist = kc.run(shots=4096, seed=42)
    counts = {}
    for i in shots_ref.tolist():
        counts[i] = counts.get(i, 0) + 1
    want = {format(i, "b").zfill(16)[::-1]: c / 4096 for i, c in counts.items()}
    assert dist.probs == want


def test_brickwork_qft_20q_vs_oracle():
    """The 30-qubit workload's family at 20 qubits: brickwork(40) + qft(20)."""
    from ket_b200 import workloads as W
    from oracle import oracle as O
    kc, idx = W.brickwork_qft(20, 40, 42)
    oc, _ = O.brickwork(20, 40, 42, with_qft=True)
    want = oc.simulate(mode=O.DENSE_PRUNE).dense()
    got = kc.statevector_array()
    assert np.max(np.abs(got - want)) < AMP_TOL
    amps = kc.amplitudes(idx)
    assert np.max(np.abs(amps - want[np.array(idx)])) < AMP_TOL
    p = np.abs(want) ** 2
    md = kc.marginal_dist(list(range(10)))
    want_md = np.bincount(np.arange(1 << 20) & 1023, weights=p, minlength=1024)
    assert np.max(np.abs(md - want_md)) < 1e-13
    m = np.array(kc.marginals())
    want_m = np.array([p[(np.arange(1 << 20) >> q) & 1 == 1].sum() for q in range(20)])
    assert np.max(np.abs(m - want_m)) < 1e-12


def test_readouts_dense_and_sparse_probs():
    from oracle import oracle as O
    gates = random_gates(12, 150, 77)
    kc, oc = build_both(12, gates)
    st = oc.simulate(mode=O.SPARSE)
    oidx, op = st.exact_probs()
    dst = kc._state()
    idx, p = dst.probs_sparse()
    assert np.array_equal(idx, oidx) and np.max(np.abs(p - op)) < AMP_TOL
    pd = dst.probs_dense()
    full = np.zeros(1 << 12)
    full[oidx.astype(np.int64)] = op
    assert np.max(np.abs(pd - full)) < AMP_TOL
    assert abs(dst.norm2() - 1.0) < 1e-12


def test_sampling_large_state_reference_order():
    """A 25-qubit state: every shot equals the reference's, whose running sum
    numpy's sequential cumsum reproduces bit for bit."""
    from ket_b200 import workloads as W
    from harness import reference_draws
    kc, _ = W.brickwork_circuit(25, 6, 42)
    st = kc._state()
    a = st.amplitudes_dense()
    sel = np.random.default_rng(25).integers(0, 1 << 25, 20000)
    want, r = reference_draws(a, draws_at=sel, rng_seed=25)
    assert np.array_equal(st.sample(r), want)


def test_expectation_and_pauli_sum_vs_oracle():
    from oracle import oracle as O
    from ket_b200 import vqe
    gates = random_gates(6, 80, 5)
    kc, oc = build_both(6, gates)
    rnd = random.Random(3)
    for _ in range(10):
        pauli = "".join(rnd.choice("IXYZ") for _ in range(6))
        assert abs(kc.expectation(pauli) - oc.expectation(pauli)) < 1e-12
    terms = [(rnd.uniform(-1, 1), "".join(rnd.choice("IXYZ") for _ in range(6))) for _ in range(12)]
    assert abs(vqe(kc, terms) - oc.vqe(terms)) < 1e-12


def test_ghz_on_qubit_30_and_31():
    """Indices above 2^31 (circuit.test.ts:482-493): 31- and 32-qubit dense states."""
    import ket_b200 as K
    d = K.Circuit(31).h(0).cnot(0, 30).run(shots=256, seed=42)
    assert set(d.probs) <= {"0" * 31, "1" + "0" * 29 + "1"} and len(d.probs) == 2
    c = K.Circuit(32).h(0).cnot(0, 31)
    a = c.amplitudes([0, (1 << 31) | 1, 1, 1 << 31])
    assert abs(a[0] - 1 / math.sqrt(2)) < 1e-15 and abs(a[1] - 1 / math.sqrt(2)) < 1e-15
    assert a[2] == 0 and a[3] == 0


def test_c64_state_close_to_c128():
    from ket_b200 import KET_C64, workloads as W
    kc, _ = W.brickwork_circuit(14, 10, 42)
    a128 = kc._state(None, precision=0).amplitudes_dense()
    a64 = kc._state(None, precision=KET_C64).amplitudes_dense()
    n64 = np.vdot(a64, a64).real
    fid = abs(np.vdot(a128, a64)) ** 2 / n64           # a128 has unit norm
    assert abs(n64 - 1) < 1e-5                           # FP32 gate entries drift the norm
    assert fid > 1 - 1e-9 and np.max(np.abs(a128 - a64)) < 1e-5


def test_state_compare_matches_host():
    """ket_state_compare: <a|b> and max |a - b| across precisions, against numpy."""
    from ket_b200 import KET_C64, workloads as W
    kc, _ = W.brickwork_circuit(15, 8, 7)
    s128 = kc._state(None, precision=0)
    s64 = kc._state(None, precision=KET_C64)
    a128, a64 = s128.amplitudes_dense(), s64.amplitudes_dense()
    ov, mx = s128.compare(s64)
    assert abs(ov - np.vdot(a128, a64)) < 1e-12
    assert abs(mx - np.max(np.abs(a128 - a64))) < 1e-15
    ov2, mx2 = s128.compare(s128)
    assert abs(ov2 - 1) < 1e-13 and mx2 == 0.0


def test_invalid_ops_leave_state_untouched():
    import ket_b200 as K
    from ket_b200.circuit import DeviceState, ops_to_abi
    st = DeviceState(3)
    st.apply(K.Circuit(3).h(0).ops)
    before = st.amplitudes_dense()
    arr, m, k = ops_to_abi(K.Circuit(3).x(1).x(2).ops)
    arr[1].q[0] = 9
    with pytest.raises(K.RangeError):
        st.apply_abi(arr, m, k)
    assert np.array_equal(st.amplitudes_dense(), before)


@pytest.mark.parametrize("n", [21, 22, 24, 26])
def test_fused_equals_unfused_many_tiles(n):
    """States with many tiles per CTA (the persistent loop's later iterations):
    the fused passes give the unfused per-gate result, run twice on each form
    of the pass (a race would show up as a difference between runs).  Each
    form is pinned: under the default policy a pass of a 26+ qubit state runs
    on the interpreter until its compiled kernel is ready, and the two forms
    agree to rounding only where merged phase ops are present."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import DeviceState, flatten_ops, ops_to_abi
    c, _ = W.brickwork_qft(n, 10, 42)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    st = DeviceState(n)
    st.apply_abi(arr, m, k, fusion=0, prune=False)
    unfused = st.amplitudes_dense()
    del st
    for specialize in (-1, 1):
        res = []
        for _ in range(2):
            st = DeviceState(n)
            st.apply_abi(arr, m, k, fusion=-1, prune=False, specialize=specialize)
            res.append(st.amplitudes_dense())
            del st
        assert np.max(np.abs(res[0] - unfused)) < 1e-13, specialize
        assert np.array_equal(res[0], res[1]), specialize
