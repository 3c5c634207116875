"""Host-side logic without a GPU: the Python mirror of the reference API
(builder validation, PRNG, bitstrings, gate matrices, workload generators),
the C-ABI library's exports, and the fusion planner's statistics."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import ket_b200 as K
from ket_b200 import _lib, gates as G, workloads as W
from ket_b200.circuit import bitstring_to_index, flatten_ops, index_to_bitstring, make_prng, ops_to_abi, prng_draws
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "ket_sv.h")).read()
    return sorted(set(re.findall(r"KET_API\s+[\w\s\*]+?\b(ket_\w+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    L = _lib.lib()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert L.ket_abi_version() == 1


def test_prng_matches_reference_xorshift():
    """makePrng (circuit.ts:813-819): xorshift32, seed 0 -> 1."""
    st = 42
    rng = make_prng(42)
    for _ in range(100):
        v, st = O.prng_next(st)
        assert rng() == v / 4294967296.0
    assert make_prng(0)() == make_prng(1)()
    d = prng_draws(42, 50)
    r2 = make_prng(42)
    assert all(d[i] == r2() for i in range(50))


def test_bitstrings():
    assert bitstring_to_index("10", 2) == 1 and bitstring_to_index("01", 2) == 2
    assert index_to_bitstring(1, 3) == "100"
    assert index_to_bitstring((1 << 40), 41) == "0" * 40 + "1"
    with pytest.raises(TypeError):
        bitstring_to_index("0", 2)
    with pytest.raises(TypeError):
        bitstring_to_index("0x", 2)


def test_builder_validation():
    """#checkOp (circuit.ts:1113-1146) and the bounds tests (circuit.test.ts:507-552)."""
    with pytest.raises(K.RangeError):
        K.Circuit(2).h(-1)
    with pytest.raises(K.RangeError):
        K.Circuit(2).x(2)
    with pytest.raises(K.RangeError):
        K.Circuit(3).z(99)
    with pytest.raises(K.RangeError):
        K.Circuit(2).cnot(5, 1)
    with pytest.raises(K.RangeError):
        K.Circuit(2).xx(math.pi / 4, 0, 5)
    with pytest.raises(K.RangeError):
        K.Circuit(3).ccx(0, 1, 3)
    with pytest.raises(TypeError):
        K.Circuit(2).cnot(1, 1)
    with pytest.raises(TypeError):
        K.Circuit(2).crz(0.3, 0, 0)
    with pytest.raises(TypeError):
        K.Circuit(1).unitary([[1, 0, 0], [0, 1, 0]], 0)
    with pytest.raises(K.RangeError, match="5"):
        K.Circuit(3).h(5)
    K.Circuit(3).h(0).h(1).h(2)


def test_immutability_and_params():
    a = K.Circuit(1)
    b = a.h(0)
    assert len(a) == 0 and len(b) == 1
    c = K.Circuit(1).h(0).rx("theta", 0).rz("phi", 0)
    assert c.params == ["phi", "theta"]
    with pytest.raises(TypeError):
        flatten_ops(c.ops)
    d = c.bind({"theta": 0.3, "phi": 0.5})
    assert d.params == [] and d.ops[1].gate == G.Rx(0.3)
    with pytest.raises(TypeError):
        c.bind({"theta": 0.3})


def test_named_gates_flatten():
    bell = K.Circuit(2).h(0).cnot(0, 1)
    c = K.Circuit(4).defineGate("bell", bell).gate("bell", 2, 3)
    flat = flatten_ops(c.ops)
    assert [o.kind for o in flat] == ["single", "cnot"]
    assert flat[0].qubits == (2,) and flat[1].qubits == (2, 3)
    with pytest.raises(TypeError):
        K.Circuit(4).gate("nope", 0)


def test_gate_matrices_match_oracle():
    """gates.py against the oracle's restatement of gates.ts, bit for bit."""
    cases = [("h", [0], []), ("t", [0], []), ("v", [0], []), ("rx", [0], [0.7]), ("ry", [0], [1.3]),
             ("rz", [0], [2.1]), ("u1", [0], [0.4]), ("u2", [0], [0.1, 0.2]), ("u3", [0], [0.3, 0.4, 0.5]),
             ("gpi", [0], [0.6]), ("gpi2", [0], [0.8]), ("xx", [0, 1], [0.9]), ("yy", [0, 1], [1.1]),
             ("zz", [0, 1], [1.2]), ("xy", [0, 1], [1.4]), ("ms", [0, 1], [0.2, 0.7]), ("iswap", [0, 1], []),
             ("srswap", [0, 1], []), ("crx", [0, 1], [0.5]), ("cu3", [0, 1], [0.1, 0.2, 0.3]), ("r8", [0], [])]
    for name, qs, ps in cases:
        oc = O.OCircuit(2).add(name, qs, ps)
        kind, oq, m = oc.op_info(0)
        kc = getattr(K.Circuit(2), name)(*ps, *qs)
        op = kc.ops[0]
        mine = np.array(op.gate, dtype=np.complex128).reshape(-1)
        assert kind == op.kind and oq == list(op.qubits)
        assert np.array_equal(mine, m), name


def test_workload_generators_match_oracle():
    """The seeded brickwork stream is identical in Python and in the oracle."""
    c, rng = W.brickwork_circuit(8, 6, 42)
    oc, st = O.brickwork(8, 6, 42)
    assert len(c) == len(oc)
    for i, op in enumerate(c.ops):
        kind, qs, m = oc.op_info(i)
        assert kind == op.kind and qs == list(op.qubits)
        if op.gate is not None:
            assert np.array_equal(np.array(op.gate, dtype=np.complex128).reshape(-1), m)
    assert rng.s == st
    # qft appended; amplitude indices continue the stream
    c2, idx = W.brickwork_qft(8, 6, 42, n_amps=5)
    oc2, st2 = O.brickwork(8, 6, 42, with_qft=True)
    assert len(c2) == len(oc2)
    s = st2
    for k in range(5):
        v, s = O.prng_next(s)
        assert idx[k] == v >> 24
    # random 3-regular graphs
    r = W.Xorshift32(7)
    e1 = W.regular3(10, r)
    e2, s2 = O.regular3(10, 7)
    assert e1 == e2 and r.s == s2
    deg = np.zeros(10, int)
    for u, v in e1:
        deg[u] += 1
        deg[v] += 1
    assert (deg == 3).all()


def test_qaoa_batch_and_vqe_workloads():
    inst = W.qaoa_batch(64, p=4)
    assert len(inst) == 64
    for n, e, g, b in inst:
        assert n in (10, 12, 14, 16, 18, 20, 22) and len(e) == 3 * n // 2 and len(g) == 4
        assert all(0 <= x < math.pi for x in g + b)
    ansatz, H, params = W.tfim_vqe(6, 2, 3)
    assert ansatz.paramCount == 24 and len(params) == 3 and len(H) == 11
    assert len(ansatz(params[0])) == 2 * (12 + 5)


def test_ops_to_abi():
    c = K.Circuit(3).h(0).cnot(0, 2).ccx(0, 1, 2).xx(0.3, 1, 2).unitary(np.eye(8), 0, 1, 2).barrier()
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    assert k == 6
    assert [arr[i].kind for i in range(k)] == [0, 1, 5, 3, 8, 9]
    assert arr[4].nq == 3 and m.size == 4 + 16 + 64


def plan(c, fusion=-1, prec=0):
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    mv = np.ascontiguousarray(m).view(np.float64)
    o = _lib.exec_opts(fusion, True)
    out = (C.c_int64 * 3)()
    rc = _lib.lib().ket_plan_stats(c.qubits, prec, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                                   C.byref(o), out)
    _lib.check(rc)
    return list(out)


def test_planner_pass_counts_on_the_bench_workload():
    """The tile planner on the 30-qubit bench circuit (no GPU needed): with
    the reference's pruning, mixing gates keep their order and a candidate
    tile scores first by the mixing gates it takes (106 passes; 90 is a lower
    bound for the mixing gates alone); without pruning, 42 passes."""
    c, _ = W.brickwork_qft(30, 40, 42)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    mv = np.ascontiguousarray(m).view(np.float64)
    for prune, most in ((True, 106), (False, 42)):
        o = _lib.exec_opts(-1, prune)
        out = (C.c_int64 * 3)()
        _lib.check(_lib.lib().ket_plan_stats(30, 0, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                                             C.byref(o), out))
        assert 90 <= out[0] <= most if prune else out[0] <= most, (prune, list(out))
        assert out[1] == 0 and out[2] <= k


def test_program_statistics_stay_in_their_array():
    """ket_plan_program_stats on the 30-qubit bench circuit writes its 16 counts
    and nothing past them, whatever op types the programs hold (the QFT's
    phase polynomials included)."""
    c, _ = W.brickwork_qft(30, 40, 42)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    mv = np.ascontiguousarray(m).view(np.float64)
    for reg_bits in (4, 5):
        o = _lib.exec_opts(prune=True, specialize=1, reg_bits=reg_bits)
        buf = (C.c_int64 * 24)(*([-7] * 24))
        _lib.check(_lib.lib().ket_plan_program_stats(30, 0, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)),
                                                     m.size, C.byref(o), buf))
        assert list(buf)[16:] == [-7] * 8
        assert buf[14] == 106 and buf[15] == 0
        assert buf[11] > 0  # phase fans and phase polynomials of the QFT
        assert buf[12] + buf[13] == buf[1] + buf[2]  # every 2x2 op has one matrix form


def test_planner_statistics():
    c, _ = W.brickwork_circuit(16, 20, 42)
    fused = plan(c)
    unf = plan(c, fusion=0)
    assert unf[0] == 0 and unf[1] == unf[2]
    # folding merges diagonals into neighbouring single-qubit gates on the same qubit
    assert unf[2] * 0.6 < fused[2] <= unf[2]
    assert fused[0] < unf[1] / 5, fused
    # validation runs in the planner without a GPU
    bad = K.Circuit(2).h(0)
    arr, m, k = ops_to_abi(bad.ops)
    arr[0].q[0] = 7
    o = _lib.exec_opts()
    out = (C.c_int64 * 3)()
    mv = np.ascontiguousarray(m).view(np.float64)
    rc = _lib.lib().ket_plan_stats(2, 0, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, C.byref(o), out)
    assert rc == _lib.KET_ERR_RANGE


def test_no_gpu_reports_cuda_error():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = C.c_void_p()
    rc = _lib.lib().ket_ctx_create(0, C.byref(h))
    assert rc == _lib.KET_ERR_CUDA


def test_program_generator_on_the_bench_workload():
    """The cost-model layouts on the 30-qubit bench circuit (4 register bits,
    pruning on): 2x2 gates on lane bits, which cost a shuffle per amplitude,
    nearly all become register gates (145 under the greedy rule), and no swap
    is left as a shared-memory op (the QFT's closing swaps are relabellings)."""
    c, _ = W.brickwork_qft(30, 40, 42)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    mv = np.ascontiguousarray(m).view(np.float64)
    o = _lib.exec_opts(prune=True, specialize=1, reg_bits=4)
    cnt = (C.c_int64 * 16)()
    _lib.check(_lib.lib().ket_plan_program_stats(30, 0, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                                                 C.byref(o), cnt))
    assert cnt[14] == 106
    assert cnt[2] <= 32, list(cnt)   # 2x2 on lane bits
    assert cnt[5] == 0, list(cnt)    # swaps through shared memory
    assert 150 <= cnt[0] <= 260, list(cnt)  # layout exchanges
