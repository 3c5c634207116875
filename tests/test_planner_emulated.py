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
    target is a register bit are deferred (FOF_SW): the brickwork's programs
    hold such ops, and the compiled kernels' semantics (per-thread swap flags,
    matrix entries exchanged, FO_REAL, logical-slot exchanges and stores) give
    the reference algorithm's state, as the interpreter's eager swaps do."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops
    from emulator import sw_count
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
        assert sw_count() > 0
        assert np.max(np.abs(got - want)) < 1e-12
        outs.append(got)
    assert np.array_equal(outs[0], outs[1])  # swaps are exact: both orders give the same bits

