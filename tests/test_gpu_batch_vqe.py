"""Batched vqe() energies (ket_batch_vqe) against the oracle's vqe(), the
reference algorithm: a re-simulation per Pauli term of the sparse map with
per-gate pruning (algorithms.ts:301-336).  Tolerance 1e-12."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_energy(ansatz_kind, n, layers, params, ham):
    from oracle import oracle as O
    c = O.ansatz(ansatz_kind, n, layers, params)
    return c.vqe([(t.coeff, t.ops) for t in ham], mode=O.SPARSE)


def test_batch_vqe_uneven_widths_vs_oracle():
    from ket_b200 import workloads as W
    from ket_b200.batch import batch_vqe
    from oracle import oracle as O
    templates, inst = W.vqe_batch(96, sizes=(4, 7, 10, 13), layers=3, seed=5)
    got = batch_vqe(templates, inst)
    sizes = (4, 7, 10, 13)
    for i in range(0, 96, 5):
        t, p = inst[i]
        want = _oracle_energy(O.ANS_HEA_LADDER, sizes[t], 3, p, templates[t][1])
        assert abs(got[i] - want) < 1e-12, (i, sizes[t])


def test_batch_vqe_matches_engine_vqe_every_gate_kind():
    """Templates with fixed gates of every supported kind (controlled,
    two-qubit, toffoli, cswap, csrswap, 2-qubit unitary) and every parametric
    family, against the engine's own single-circuit vqe()."""
    import ket_b200 as K
    from ket_b200.batch import batch_vqe
    rng = np.random.default_rng(3)
    u2 = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]

    def ans(p):
        c = K.Circuit(6)
        for q in range(6):
            c = c.h(q)
        c = c.rx(p[0], 0).ry(p[1], 1).rz(p[2], 2).u1(p[3], 3).gpi(p[4], 4).gpi2(p[5], 5)
        c = c.crx(p[6], 0, 1).cry(p[7], 2, 3).crz(p[8], 4, 5).cu1(p[9], 1, 4)
        c = c.xx(p[10], 0, 3).yy(p[11], 1, 5).zz(p[12], 2, 4).xy(p[13], 3, 0)
        c = c.cnot(0, 5).swap(1, 2).ccx(0, 1, 3).cswap(2, 4, 5).csrswap(5, 0, 1).cz(3, 4).ch(2, 0)
        c = c.unitary(u2, 4, 1).t(3).s(2)
        return c

    H = [(0.7, "ZZIIII"), (-0.3, "XIYIIZ"), (0.25, "IIIIII"), (1.1, "YYYYYY"), (0.4, "IXIXIX")]
    inst = [(0, list(rng.uniform(0, 2 * math.pi, 14))) for _ in range(12)]
    got = batch_vqe([(ans, H)], inst)
    for (t, p), g in zip(inst, got):
        assert abs(g - K.vqe(ans(p), H)) < 1e-12


def test_batch_vqe_graph_replay_and_new_parameters():
    from ket_b200 import workloads as W
    from ket_b200.batch import batch_vqe
    templates, inst = W.vqe_batch(40, sizes=(5, 9), layers=2, seed=8)
    a = batch_vqe(templates, inst, use_graph=True)
    b = batch_vqe(templates, inst, use_graph=False)
    assert np.array_equal(a, b)
    inst2 = [(t, [v + 0.1 for v in p]) for t, p in inst]
    c = batch_vqe(templates, inst2, use_graph=True)      # replays the kept graph with new angles
    d = batch_vqe(templates, inst2, use_graph=False)
    assert np.array_equal(c, d) and not np.array_equal(a, c)


def test_batch_vqe_rejects():
    import ket_b200 as K
    from ket_b200._lib import KetError
    from ket_b200.batch import batch_vqe
    wide = (lambda p: K.Circuit(14).ry(p[0], 0), [(1.0, "Z" * 14)])
    with pytest.raises(KetError):
        batch_vqe([wide], [(0, [0.1])])
    bad = (lambda p: K.Circuit(3).ry(p[0], 0), [(1.0, "ZZ")])
    with pytest.raises(Exception):
        batch_vqe([bad], [(0, [0.1])])
