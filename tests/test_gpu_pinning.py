"""The programs the 30-qubit workload runs, pinned to the reference algorithm.

From 26 qubits the engine runs pass kernels compiled for 4-register-bit
programs (256 threads of 16 amplitudes), with merged phase fans and the
reference's per-gate pruning (accumulate(), statevector.ts:19-27).  Those
programs are checked here against the oracle directly, not against another
path of the engine:

* at 12-20 qubits through ket_exec_opts.reg_bits = 4, which gives small
  states the large states' programs: the random-gate suite (every gate kind)
  against the SPARSE oracle (the reference's sorted map with pruning), and the
  workload's own family, brickwork(40) + qft(20), against DENSE_PRUNE;
* at 26 qubits with the workload's exact options (compiled kernels, automatic
  register bits, pruning on) against the DENSE_PRUNE oracle on the host cores;
* the 24-qubit, 8-layer VQE gradient (adjoint against parameter shift on the
  same engine and against central differences, both without pruning), and
  the batched QAOA at its widest size, n = 22.

Tolerances: amplitudes and probabilities 1e-12 (complex128), the q0-q9
distribution 1e-13, gradients 1e-10 against parameter shift and 1e-8 against
central differences with eps = 1e-6 (the difference quotient's own rounding)."""
import ctypes as C

import numpy as np
import pytest

from test_gpu_parity import build_both, random_gates

pytestmark = pytest.mark.gpu

AMP_TOL = 1e-12


def _launches():
    from ket_b200 import _lib
    out, cs = (C.c_int64 * 4)(), C.c_double()
    _lib.check(_lib.lib().ket_jit_stats(out, C.byref(cs)))
    return out[3]


def _run(n, circ, reg_bits, specialize=1, init=0, prune=True):
    from ket_b200.circuit import DeviceState, flatten_ops, ops_to_abi
    arr, m, k = ops_to_abi(flatten_ops(circ.ops))
    st = DeviceState(n)
    st.set_basis(init)
    before = _launches()
    st.apply_abi(arr, m, k, prune=prune, specialize=specialize, reg_bits=reg_bits)
    ran = _launches() - before
    return st, ran


@pytest.mark.parametrize("n,seed", [(12, 31), (13, 32), (14, 33), (15, 34), (16, 35), (17, 36)])
def test_four_bit_programs_random_gates_vs_sparse_oracle(n, seed):
    from oracle import oracle as O
    gates = random_gates(n, 80 + 10 * n, seed)
    kc, oc = build_both(n, gates)
    init = (seed * 7919) % (1 << n)
    want = oc.simulate(init=init, mode=O.SPARSE).dense()
    st, ran = _run(n, kc, 4, init=init)
    assert ran > 0, "no compiled pass kernel ran"
    assert np.max(np.abs(st.amplitudes_dense() - want)) < AMP_TOL


@pytest.mark.parametrize("reg_bits", [4, 5])
def test_programs_brickwork40_qft20_vs_oracle(reg_bits):
    """The workload's family at 20 qubits, on 4- and 5-register-bit programs,
    read out as the workload reads: 1024 amplitudes and the q0-q9 distribution."""
    from ket_b200 import workloads as W
    from oracle import oracle as O
    kc, idx = W.brickwork_qft(20, 40, 42)
    oc, _ = O.brickwork(20, 40, 42, with_qft=True)
    want = oc.simulate(mode=O.DENSE_PRUNE).dense()
    st, ran = _run(20, kc, reg_bits)
    assert ran > 0
    assert np.max(np.abs(st.amplitudes_dense() - want)) < AMP_TOL
    assert np.max(np.abs(st.amplitudes(idx) - want[np.array(idx)])) < AMP_TOL
    p = np.abs(want) ** 2
    want_md = np.bincount(np.arange(1 << 20) & 1023, weights=p, minlength=1024)
    assert np.max(np.abs(st.marginal_dist(list(range(10))) - want_md)) < 1e-13


def test_workload_path_26q_vs_dense_prune_oracle():
    """brickwork(10) + qft(26) at 26 qubits through the workload's own options:
    compiled kernels (specialize = 1), automatic register bits (4 from 26
    qubits), merged phase fans, pruning on."""
    from ket_b200 import workloads as W
    from oracle import oracle as O
    n = 26
    kc, idx = W.brickwork_qft(n, 10, 42)
    oc, _ = O.brickwork(n, 10, 42, with_qft=True)
    st, ran = _run(n, kc, 0)
    assert ran > 0
    got = st.amplitudes_dense()
    amps = st.amplitudes(idx)
    md = st.marginal_dist(list(range(10)))
    del st
    want = oc.simulate(mode=O.DENSE_PRUNE).dense()
    assert np.max(np.abs(got - want)) < AMP_TOL
    assert np.max(np.abs(amps - want[np.array(idx)])) < AMP_TOL
    p = np.abs(want) ** 2
    want_md = np.bincount(np.arange(1 << n) & 1023, weights=p, minlength=1024)
    assert np.max(np.abs(md - want_md)) < 1e-13


def test_adjoint_vqe24_8_layers():
    """The differentiation workload at its own size: 24 qubits, 8 layers, 384
    parameters, TFIM Hamiltonian; one parameter vector of the seeded batch.

    The adjoint differentiates the exact energy (no pruning): it is held to
    parameter shift of the same energy at 1e-10 and to central differences at
    1e-8.  The reference's gradient() shifts energies simulated with its
    per-gate pruning; on this ansatz the first layers leave many amplitudes
    below 1e-7, so the pruned energy sits about 1e-6 from the exact one, and
    the pruned shift gradient is checked only to that order."""
    from ket_b200 import workloads as W
    from ket_b200.adjoint import adjoint_gradient, shift_gradient
    ans, H, params = W.tfim_vqe(24, 8, 1)
    P = np.asarray(params)
    e_adj, g_adj = adjoint_gradient(ans, H, P)
    e_sh, g_sh = shift_gradient(ans, H, P, prune=False)
    assert abs(e_adj[0] - e_sh[0]) < 1e-11
    assert np.max(np.abs(g_adj - g_sh)) < 1e-10

    def energy(p):
        return ans(list(p))._state(None, prune=False).expect_pauli_sum([(t.coeff, t.ops) for t in H])

    eps = 1e-6
    for k in (0, 191, 383):
        pp, pm = P[0].copy(), P[0].copy()
        pp[k] += eps
        pm[k] -= eps
        fd = (energy(pp) - energy(pm)) / (2 * eps)
        assert abs(fd - g_adj[0, k]) < 1e-8, k
    e_pr, g_pr = shift_gradient(ans, H, P, prune=True)
    assert abs(e_pr[0] - e_adj[0]) < 1e-4
    assert np.max(np.abs(g_pr - g_adj)) < 1e-4


def test_batch_qaoa_widest_instances():
    """n = 22, the largest size of the batch workload, against the oracle."""
    from ket_b200 import workloads as W
    from ket_b200.batch import batch_qaoa
    from test_gpu_batch import oracle_cut
    inst = W.qaoa_batch(2, p=4, seed=19, sizes=(22,))
    got = batch_qaoa(inst)
    for (n, e, g, b), v in zip(inst, got):
        assert n == 22
        assert abs(v - oracle_cut(n, e, g, b)) < 1e-10


@pytest.mark.parametrize("n,layers", [(1, 3), (2, 3), (3, 4), (11, 6), (20, 12)])
def test_shots_sequential_cdf_vs_oracle(n, layers):
    """run()'s sampler on the sequential CDF (states up to 20 qubits): the
    reference's running sum in index order, so shot indices equal the
    oracle's one for one, down to states smaller than one unrolled step."""
    from ket_b200 import workloads as W
    from oracle import oracle as O
    kc, _ = W.brickwork_circuit(n, layers, 5 + n)
    oc, _ = O.brickwork(n, layers, 5 + n)
    want = oc.simulate(mode=O.SPARSE).run(4096, 42)
    dist = kc.run(shots=4096, seed=42)
    counts = {}
    for i in want.tolist():
        counts[i] = counts.get(i, 0) + 1
    assert dist.probs == {format(i, "b").zfill(n)[::-1]: c / 4096 for i, c in counts.items()}


def _sample_vs_numpy_cdf(n, amps, draws_at=None, rng_seed=0):
    """Shots from ket_sample against a lower bound on numpy's sequential
    cumulative sum (np.cumsum adds left to right, rounding each step, as the
    reference's loop does).  Draws sit exactly on CDF values and one ulp above
    them, so any last-bit difference in the device CDF changes an index."""
    from ket_b200.circuit import DeviceState
    st = DeviceState(n)
    st.set_amplitudes(amps)
    from harness import reference_draws
    want, r = reference_draws(amps, draws_at, rng_seed)
    got = st.sample(r)
    assert np.array_equal(got, want)


def test_sequential_cdf_ties_and_binades():
    """Entries whose probability lies exactly halfway between two multiples of
    the running sum's ulp (a tie the reference's rounding breaks by the sum's
    parity), a binade crossing at the start, entries below the pruning
    threshold and exact zeros."""
    n = 14
    a = np.zeros(1 << n, dtype=np.complex128)
    a[0] = 0.6 ** 0.5                      # the sum starts in [0.5, 1): ulp 2^-53
    a[1:] = 2.0 ** -23 + 1j * 2.0 ** -27   # p = 2^-46 + 2^-54: every addition is a tie
    a[5::7] = 1e-8                         # p = 1e-16: below the threshold, not kept
    a[9::11] = 0.0
    _sample_vs_numpy_cdf(n, a)


def test_sampling_rejects_draws_outside_unit_interval():
    from ket_b200.circuit import DeviceState
    from ket_b200 import RangeError
    st = DeviceState(4)
    for bad in (-1e-300, 1.0000000000000002, float("nan")):
        with pytest.raises(RangeError):
            st.sample(np.array([0.5, bad]))


def test_sequential_cdf_leading_zeros_and_single_entry():
    """Nothing kept before the last entry (every draw, 0 included, lands on
    it), and a block of zeros between two kept entries."""
    n = 16
    a = np.zeros(1 << n, dtype=np.complex128)
    a[-1] = 1.0
    _sample_vs_numpy_cdf(n, a, draws_at=np.array([0, 1 << 15, (1 << n) - 1]))
    a[:] = 0.0
    a[3] = 0.5 ** 0.5
    a[(1 << n) - 5] = 0.5 ** 0.5
    _sample_vs_numpy_cdf(n, a, draws_at=np.array([0, 3, 4, 1 << 15, (1 << n) - 5]))


@pytest.mark.parametrize("n", [10, 16, 20, 24])
def test_sequential_cdf_random_states(n):
    rng = np.random.default_rng(n)
    a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    a[rng.random(1 << n) < 0.1] = 0.0
    a /= np.linalg.norm(a)
    sel = np.unique(rng.integers(0, 1 << n, 20000))
    _sample_vs_numpy_cdf(n, a, draws_at=sel, rng_seed=n)
