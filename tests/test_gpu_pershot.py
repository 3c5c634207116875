"""run()'s per-shot path on the device (ket_run_shots) against the oracle.

* Every restated reference test of measure / reset / if / noise
  (tests/golden/pershot_kats.json) holds for the engine's Circuit.run.
* Per shot, the engine's sampled index, classical bits and the stream state
  after the last draw equal the oracle's for the same seed: both walk the
  reference's draw order, and the trajectories agree to rounding (P(q=1) is
  summed in a different order, so an outcome could differ only if a draw fell
  within rounding of it).
* Random circuits with mid-circuit measurement, reset, nested if and noise
  at 10-16 qubits agree shot by shot with the oracle.
"""
import ctypes as C
import math

import numpy as np
import pytest

from harness import (case_registers, check_pershot, ket_pershot_circuit, load_pershot_kats, pershot_noise,
                     pershot_oracle_raw, summarize)

pytestmark = pytest.mark.gpu

CASES = load_pershot_kats()


def engine_raw(circ, shots, seed, nz, init=0):
    from ket_b200 import _lib
    from ket_b200.circuit import DeviceState, make_prng, shots_to_abi
    arr, m, k, nb, layout = shots_to_abi(circ.ops, circ._cregs)
    st = DeviceState(circ.qubits)
    noise = _lib.ket_noise(*(nz or (0.0, 0.0, 0.0)))
    state = C.c_uint32(make_prng(seed).state[0])
    idx = np.zeros(max(shots, 1), dtype=np.uint64)
    bits = np.zeros(max(shots * nb, 1), dtype=np.uint8)
    mv = np.ascontiguousarray(m).view(np.float64)
    _lib.check(_lib.lib().ket_run_shots(st.h, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                                        C.byref(noise), init, shots, C.byref(state), nb,
                                        idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                        bits.ctypes.data_as(C.POINTER(C.c_uint8))))
    return idx[:shots], bits[: shots * nb].reshape(shots, nb), int(state.value), layout


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_pershot_kat_engine(case):
    c = ket_pershot_circuit(case)
    r = c.run(shots=case["run"]["shots"], seed=case["run"]["seed"], noise=case["run"]["noise"])
    clean = None
    if any(k[0] == "like_clean" for k in case["checks"]):
        clean = c.run(shots=case["run"]["shots"], seed=case["run"]["seed"]).probs
    check_pershot(case, r.probs, r.cregs, clean)


@pytest.fixture(params=[1, 0], ids=["one_at_a_time", "automatic"])
def path(request):
    """ket_run_shots' path: 1 = one trajectory at a time through the fused
    engine; 0 = automatic (every KAT and the small random circuits below
    then run as batched trajectories in shared memory)."""
    from ket_b200 import _lib
    _lib.check(_lib.lib().ket_debug_pershot_path(request.param))
    yield request.param
    _lib.lib().ket_debug_pershot_path(0)


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_pershot_matches_oracle_shot_by_shot(case, path):
    from ket_b200.circuit import make_prng
    c = ket_pershot_circuit(case)
    shots, seed = case["run"]["shots"], case["run"]["seed"]
    idx, bits, state, layout = engine_raw(c, shots, seed, pershot_noise(case))
    oidx, obits, regs = pershot_oracle_raw(case)
    assert layout == regs
    assert np.array_equal(idx, oidx), case["id"]
    assert np.array_equal(bits, obits), case["id"]
    # the oracle's final stream state, recomputed from its own draw count
    from oracle import oracle as O
    oc = O.OCircuit(case["n"])
    from harness import _oracle_ops
    _oracle_ops(oc, case["ops"], regs, case["n"])
    nz = pershot_noise(case) or (0.0, 0.0, 0.0)
    _, _, ostate = oc.run_pershot(shots, make_prng(seed).state[0], nz[0], nz[1], nz[2], case_registers(case)[1])
    assert state == ostate


def random_case(n, depth, seed, noise, if_draws=True):
    """A seeded circuit with gates of every kind, measurements, resets and a
    nested if, as a case spec (see tests/golden/make_pershot_kats.py).
    if_draws=False keeps every draw out of the if-bodies (only noiseless
    permutation gates there), so that each shot draws a fixed number of times."""
    rng = np.random.default_rng(seed)
    singles = ["h", "x", "y", "z", "s", "t", "v"]
    rots = ["rx", "ry", "rz", "u1"]

    def gates(k):
        ops = []
        for _ in range(k):
            r = rng.integers(7)
            q = int(rng.integers(n))
            q2 = int((q + 1 + rng.integers(n - 1)) % n)
            if r == 0:
                ops.append([singles[rng.integers(len(singles))], [q], []])
            elif r == 1:
                ops.append([rots[rng.integers(len(rots))], [q], [float(rng.uniform(0, 2 * math.pi))]])
            elif r == 2:
                ops.append(["cnot", [q, q2], []])
            elif r == 3:
                ops.append(["crz", [q, q2], [float(rng.uniform(0, 2 * math.pi))]])
            elif r == 4:
                ops.append(["swap", [q, q2], []])
            elif r == 5:
                ops.append(["xx", [q, q2], [float(rng.uniform(0, 2 * math.pi))]])
            else:
                q3 = int((q2 + 1 + rng.integers(n - 2)) % n)
                if q3 == q:
                    q3 = (q3 + 1) % n
                if q3 == q2:
                    q3 = (q3 + 1) % n
                ops.append(["ccx", [q, q2, q3], []]) if len({q, q2, q3}) == 3 else ops.append(["h", [q], []])
        return ops

    ops = [["creg", "c", 3]] + gates(depth)
    ops += [["measure", 0, "c", 0], ["measure", n - 1, "c", 1]]
    ops += gates(depth // 2)
    if if_draws:
        ops += [["if", "c", 1, gates(3) + [["measure", 1, "c", 2], ["if", "c", 5, [["x", [2], []]]]]]]
    else:
        ops += [["if", "c", 1, [["ccx", [0, 1, 2], []], ["if", "c", 3, [["cswap", [2, 0, 1], []]]]]]]
        ops += [["unitary", [1, 3], _random_unitary(rng, 4)], ["csrswap", [0, 2, 3], []]]
    ops += [["reset", n // 2, 0]] + gates(depth // 2) + [["measure", 2, "m", 0]]
    return {"id": f"rand{n}", "n": n, "ops": ops, "run": {"shots": 0, "seed": 0, "noise": noise}, "checks": []}


def _random_unitary(rng, d):
    z = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    q, r = np.linalg.qr(z)
    q = q * (np.diag(r) / np.abs(np.diag(r)))
    return [[float(v) for c in row for v in (c.real, c.imag)] for row in q]


@pytest.mark.parametrize("n,depth,shots,noise,if_draws", [
    (10, 40, 200, None, True), (12, 40, 100, "aria-1", True), (16, 24, 12, {"p1": 0.05, "p2": 0.1, "pMeas": 0.02}, True),
    (5, 40, 2000, {"p1": 0.05, "p2": 0.1, "pMeas": 0.02}, False), (10, 40, 500, "h1-1", False),
    (12, 30, 200, {"p1": 0.02, "p2": 0.05, "pMeas": 0.01}, False)])
def test_pershot_random_circuits(n, depth, shots, noise, if_draws, path):
    case = random_case(n, depth, 1000 + n, noise, if_draws)
    c = ket_pershot_circuit(case)
    idx, bits, state, layout = engine_raw(c, shots, 77, pershot_noise(case))
    oidx, obits, regs = pershot_oracle_raw(case, shots=shots, seed=77)
    assert layout == regs
    assert np.array_equal(bits, obits)
    assert np.array_equal(idx, oidx)
    assert len(set(idx.tolist())) > 1  # the trajectories differ


def test_pershot_errors_leave_state_alone():
    from ket_b200 import _lib
    from ket_b200.circuit import DeviceState
    L = _lib.lib()
    st = DeviceState(3)
    st.set_basis(5)
    before = st.amplitudes_dense()

    def call(ops, ncbits=1, shots=1):
        arr = (_lib.ket_op * len(ops))()
        for i, (kind, qs) in enumerate(ops):
            arr[i].kind, arr[i].nq, arr[i].mat = kind, len(qs), -1
            for j, v in enumerate(qs):
                arr[i].q[j] = v
        state = C.c_uint32(1)
        idx = np.zeros(shots, dtype=np.uint64)
        bits = np.zeros(shots * max(ncbits, 1), dtype=np.uint8)
        return L.ket_run_shots(st.h, arr, len(ops), None, 0, None, 0, shots, C.byref(state), ncbits,
                               idx.ctypes.data_as(C.POINTER(C.c_uint64)), bits.ctypes.data_as(C.POINTER(C.c_uint8)))

    assert call([(_lib.OP_MEASURE, (0, 1))]) == _lib.KET_ERR_RANGE          # classical bit past the registers
    assert call([(_lib.OP_RESET, (3,))]) == _lib.KET_ERR_RANGE              # reset checks its qubit
    assert call([(_lib.OP_IF, (0, 1, 1, 2)), (_lib.OP_BARRIER, (0,))]) == _lib.KET_ERR_TYPE  # body past the end
    assert call([(_lib.OP_IF, (0, 40, 1, 0))], ncbits=40) == _lib.KET_ERR_UNSUPPORTED
    assert call([(_lib.OP_CNOT, (1, 1))]) == _lib.KET_ERR_TYPE              # control == target, via lower_ops
    assert np.array_equal(st.amplitudes_dense(), before)
    # a measured qubit outside the state reads 0 and leaves the state alone
    assert call([(_lib.OP_MEASURE, (7, 0))]) == 0


def test_pershot_c64_statistics():
    """The c64 workspace gives the same statistics (its probabilities are
    FP32, so shots may differ from the c128 run)."""
    from ket_b200 import _lib
    from ket_b200.circuit import DeviceState, shots_to_abi, make_prng
    from ket_b200 import Circuit
    c = Circuit(2).h(0).cnot(0, 1).measure(0, "c", 0)
    arr, m, k, nb, layout = shots_to_abi(c.ops, c._cregs)
    st = DeviceState(2, _lib.KET_C64)
    shots = 4000
    state = C.c_uint32(make_prng(3).state[0])
    idx = np.zeros(shots, dtype=np.uint64)
    bits = np.zeros(shots * nb, dtype=np.uint8)
    mv = np.ascontiguousarray(m).view(np.float64)
    _lib.check(_lib.lib().ket_run_shots(st.h, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, None, 0,
                                        shots, C.byref(state), nb, idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                        bits.ctypes.data_as(C.POINTER(C.c_uint8))))
    assert set(idx.tolist()) <= {0, 3}
    assert abs(bits.mean() - 0.5) < 0.05
    assert np.array_equal(bits.astype(np.int64) * 3, idx.astype(np.int64))
