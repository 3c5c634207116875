"""The fusion planner and the register-tiled program generator, checked on the
CPU: the programs are executed by an emulator of the k_fused2 kernel's op
semantics (tests/cpp/emulate_program.cpp) and compared with the oracle."""
import random

import numpy as np
import pytest

from emulator import emu_apply
from test_gpu_parity import build_both, random_gates


@pytest.mark.parametrize("n,seed", [(12, 1), (13, 2), (14, 3), (15, 4), (16, 5)])
@pytest.mark.parametrize("prune", [False, True])
@pytest.mark.parametrize("nreg", [5, 4])
@pytest.mark.parametrize("deferred", [True, False])
def test_emulated_programs_match_oracle(n, seed, prune, nreg, deferred):
    from oracle import oracle as O
    gates = random_gates(n, 90, seed, unitary=False)
    kc, oc = build_both(n, gates)
    init = random.Random(seed).randrange(1 << n)
    st0 = np.zeros(1 << n, complex)
    st0[init] = 1
    from ket_b200.circuit import flatten_ops
    rc, got, passes = emu_apply(n, flatten_ops(kc.ops), st0, prune=prune, nreg=nreg, deferred=deferred)
    assert rc == 0 and passes[0] > 0
    want = oc.simulate(init=init, mode=O.DENSE_PRUNE if prune else O.DENSE).dense()
    assert np.max(np.abs(got - want)) < 1e-12


@pytest.mark.parametrize("n", [14, 16])
@pytest.mark.parametrize("nreg", [5, 4])
@pytest.mark.parametrize("deferred", [True, False])
def test_emulated_brickwork_qft(n, nreg, deferred):
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops
    from oracle import oracle as O
    c, _ = W.brickwork_qft(n, 8, 42)
    st0 = np.zeros(1 << n, complex)
    st0[0] = 1
    rc, got, passes = emu_apply(n, flatten_ops(c.ops), st0, prune=False, nreg=nreg, deferred=deferred)
    oc, _ = O.brickwork(n, 8, 42, with_qft=True)
    assert rc == 0
    assert np.max(np.abs(got - oc.simulate(mode=O.DENSE).dense())) < 1e-12


FO_CPHASE, FO_PPOLY = 11, 16


@pytest.mark.parametrize("n", [14, 16])
@pytest.mark.parametrize("nreg", [5, 4])
def test_emulated_brickwork_qft_pruned_phase_runs(n, nreg):
    """With pruning on, the QFT's runs of controlled phases become merged
    phase ops (FO_PPOLY and FO_CPHASE); the result still equals the
    reference algorithm with its per-gate pruning."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops
    from emulator import type_count
    from oracle import oracle as O
    c, _ = W.brickwork_qft(n, 8, 42)
    st0 = np.zeros(1 << n, complex)
    st0[0] = 1
    rc, got, passes = emu_apply(n, flatten_ops(c.ops), st0, prune=True, nreg=nreg)
    assert rc == 0
    assert type_count(FO_PPOLY) > 0
    oc, _ = O.brickwork(n, 8, 42, with_qft=True)
    assert np.max(np.abs(got - oc.simulate(mode=O.DENSE_PRUNE).dense())) < 1e-12


FO_REAL = 17


@pytest.mark.parametrize("n", [14, 16])
@pytest.mark.parametrize("nreg", [5, 4])
@pytest.mark.parametrize("prune", [True, False])
def test_emulated_deferred_register_swaps(n, nreg, prune):
    """CNOTs whose control sits on a thread bit or outside the tile and whose
    target is a register bit are deferred (FOF_SW), and so are X gates on lane
    bits with no lane op after them before the next exchange: the brickwork's
    programs hold both, and the compiled kernels' semantics (per-thread swap
    flags and logical thread ids, matrix entries exchanged, FO_REAL,
    logical-slot and logical-lane exchanges and stores) give the reference
    algorithm's state, as the interpreter's eager moves do."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops
    from emulator import lane_defer_count, sw_count
    from oracle import oracle as O
    c, _ = W.brickwork_qft(n, 12, 7)
    st0 = np.zeros(1 << n, complex)
    st0[0] = 1
    oc, _ = O.brickwork(n, 12, 7, with_qft=True)
    want = oc.simulate(mode=O.DENSE_PRUNE if prune else O.DENSE).dense()
    outs = []
    for deferred in (True, False):
        rc, got, passes = emu_apply(n, flatten_ops(c.ops), st0, prune=prune, nreg=nreg, deferred=deferred)
        assert rc == 0
        assert sw_count() > 0 and lane_defer_count() > 0
        assert np.max(np.abs(got - want)) < 1e-12
        outs.append(got)
    assert np.array_equal(outs[0], outs[1])  # swaps are exact: both orders give the same bits



FO_SWAPS, FO_RELAY = 5, 18


@pytest.mark.parametrize("n", [13, 16])
@pytest.mark.parametrize("nreg", [5, 4])
@pytest.mark.parametrize("prune", [True, False])
def test_emulated_swaps_as_relabellings(n, nreg, prune):
    """The QFT's closing swaps, uncontrolled and with both qubits in the tile,
    run as relabellings of the layout (FO_RELAY: no data moves, no
    shared-memory round trip); controlled swaps stay shared-memory ops.  The
    state is the reference algorithm's."""
    import ket_b200 as K
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops
    from emulator import type_count
    from oracle import oracle as O
    c, _ = W.brickwork_qft(n, 6, 3)
    c = c.cswap(0, 1, n - 1).swap(2, n - 2)
    st0 = np.zeros(1 << n, complex)
    st0[5] = 1
    rc, got, passes = emu_apply(n, flatten_ops(c.ops), st0, prune=prune, nreg=nreg)
    assert rc == 0
    assert type_count(FO_RELAY) >= n // 2
    assert type_count(FO_SWAPS) >= 1  # the controlled one
    oc, _ = O.brickwork(n, 6, 3, with_qft=True)
    oc.add("cswap", [0, 1, n - 1])
    oc.add("swap", [2, n - 2])
    want = oc.simulate(init=5, mode=O.DENSE_PRUNE if prune else O.DENSE).dense()
    assert np.max(np.abs(got - want)) < 1e-12


FO_EXCH, FO_SYNC = 0, 19


@pytest.mark.parametrize("nreg", [5, 4])
def test_relabelling_programs_keep_loads_before_stores(nreg):
    """A pass of swaps only: the relabellings change which qubits the warp and
    register roles hold, so the store writes amplitudes that other threads
    loaded; the program then holds a barrier (FO_SYNC, or an exchange) between
    the loads and the store."""
    import ket_b200 as K
    from ket_b200.circuit import flatten_ops
    from emulator import type_count
    n = 16
    c = K.Circuit(n).swap(6, 13).swap(9, 15).swap(7, 12)
    rng = np.random.default_rng(1)
    a0 = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    rc, got, passes = emu_apply(n, flatten_ops(c.ops), a0, prune=False, nreg=nreg)
    assert rc == 0 and passes[0] == 1
    assert type_count(FO_RELAY) == 3
    assert type_count(FO_SYNC) + type_count(FO_EXCH) >= 1
    want = a0.reshape([2] * n)
    for p, q in ((6, 13), (9, 15), (7, 12)):
        want = np.swapaxes(want, n - 1 - p, n - 1 - q)
    assert np.array_equal(got, want.reshape(-1))


# Digests of the programs the planner makes for fixed circuits.  A change to
# the planner that is meant to leave its output alone (a faster search, a
# refactor) must leave these alone; one that changes the programs on purpose
# updates them, after the emulated and GPU parity tests pass.  They also pin
# that planning is deterministic: every byte of every op is defined.
PINNED_DIGESTS = [
    # (circuit, n, precision, prune, register bits) -> (digest, tiled passes, program ops)
    (("brickwork_qft", 30, 40, 42), "c128", True, 4, (0xeeddb0f01fc22c8b, 106, 1819)),
    (("random", 14, 200, 2), "c128", True, 4, (0xdca14723c9e04af2, None, None)),
    (("random", 14, 200, 2), "c64", False, 5, (0xca49d847b18b1794, None, None)),
    (("brickwork_qft", 24, 12, 7), "c64", True, 4, (0xb1d93486d5347078, None, None)),
]


@pytest.mark.parametrize("circ,prec,prune,nreg,want", PINNED_DIGESTS)
def test_pinned_program_digests(circ, prec, prune, nreg, want):
    import ket_b200 as K
    from ket_b200 import _lib, workloads as W
    from ket_b200.circuit import flatten_ops
    from emulator import plan_digest
    if circ[0] == "brickwork_qft":
        c, _ = W.brickwork_qft(circ[1], circ[2], circ[3])
    else:
        c = K.Circuit(circ[1])
        for name, qs, ps in random_gates(circ[1], circ[2], circ[3]):
            c = c.unitary(ps, *qs) if name == "unitary" else getattr(c, name)(*ps, *qs)
    precision = _lib.KET_C128 if prec == "c128" else _lib.KET_C64
    got = plan_digest(circ[1], flatten_ops(c.ops), precision, prune=prune, nreg=nreg)
    assert got[0] == want[0], hex(got[0])
    for g, w in zip(got[1:], want[1:]):
        if w is not None:
            assert g == w


# The same for adjoint-style reverse plans (the ancilla on qubit n, probes
# after the one-qubit matrix and diagonal gates): the probe passes' programs.
PINNED_ADJOINT_DIGESTS = [
    (("tfim_vqe", 24), (0x84d88aee9de27529, 30, 1068)),
    (("random", 15, 250, 11), (0x77d05877904d3a2b, 11, 459)),
]


@pytest.mark.parametrize("circ,want", PINNED_ADJOINT_DIGESTS)
def test_pinned_adjoint_program_digests(circ, want):
    import ket_b200 as K
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops
    from emulator import adjoint_plan_digest
    if circ[0] == "tfim_vqe":
        ans, _, params = W.tfim_vqe(circ[1], 8, 1)
        c = ans(params[0])
    else:
        c = K.Circuit(circ[1])
        for name, qs, ps in random_gates(circ[1], circ[2], circ[3]):
            c = c.unitary(ps, *qs) if name == "unitary" else getattr(c, name)(*ps, *qs)
    got = adjoint_plan_digest(circ[1], flatten_ops(c.ops))
    assert got == want, (hex(got[0]), got[1:])
