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
