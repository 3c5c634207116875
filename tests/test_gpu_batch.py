"""Batched QAOA against the reference algorithm: the oracle's qaoa() +
maxCutHamiltonian() + vqe() (sparse map, pruning) with gamma_ref = -2 gamma."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def oracle_cut(n, edges, gamma, beta):
    """vqe() of the reference for small n; above that one oracle simulation
    and the diagonal MaxCut energy sum_x p(x) cut(x) (the same quantity the
    reference's per-term Z expectations add up to)."""
    from oracle import oracle as O
    c = O.qaoa(n, edges, [-2 * g for g in gamma], beta)
    if n <= 10:
        return c.vqe(O.maxcut_hamiltonian(n, edges), mode=O.SPARSE)
    p = np.abs(c.simulate(mode=O.DENSE).dense()) ** 2
    x = np.arange(1 << n)
    cut = np.zeros(1 << n)
    for u, v in edges:
        cut += ((x >> u) ^ (x >> v)) & 1
    return float(np.dot(p, cut))


def test_batch_qaoa_vs_oracle_mixed_sizes():
    from ket_b200 import workloads as W
    from ket_b200.batch import batch_qaoa
    inst = W.qaoa_batch(40, p=3, seed=7, sizes=(10, 12, 14, 16))
    got = batch_qaoa(inst)
    for (n, e, g, b), v in zip(inst, got):
        assert abs(v - oracle_cut(n, e, g, b)) < 1e-11, n


def test_batch_qaoa_graph_replay_and_4cycle():
    """The reference's 4-cycle KAT (circuit.test.ts:6373-6421): p=1 at
    gamma_ref = pi/4, beta = 0.15 pi gives an expected cut above 2.5."""
    from ket_b200.batch import batch_qaoa
    edges = [(0, 1), (1, 2), (2, 3), (3, 0)]
    inst = [(4, edges, [-math.pi / 8], [0.15 * math.pi])] * 3 + [(4, [], [0.3], [0.2])]
    a = batch_qaoa(inst, use_graph=True)
    b = batch_qaoa(inst, use_graph=False)
    assert np.array_equal(a, b)
    assert a[0] > 2.5 and abs(a[0] - oracle_cut(4, edges, [-math.pi / 8], [0.15 * math.pi])) < 1e-12
    assert abs(a[3]) < 1e-15


def test_batch_qaoa_wide_instances():
    from ket_b200 import workloads as W
    from ket_b200.batch import batch_qaoa
    inst = W.qaoa_batch(4, p=2, seed=11, sizes=(18, 20))
    got = batch_qaoa(inst)
    for (n, e, g, b), v in zip(inst, got):
        assert abs(v - oracle_cut(n, e, g, b)) < 1e-10


def test_every_launch_shape_gives_the_same_cuts(tmp_path, monkeypatch):
    """The autotuner's candidates (threads per CTA x tile width) change how the
    work is cut, not the result; the tuner caches its pick per batch shape."""
    from ket_b200 import autotune, workloads as W
    from ket_b200.batch import batch_qaoa
    monkeypatch.setenv("KET_B200_CACHE", str(tmp_path))
    inst = W.qaoa_batch(48, p=2, seed=5, sizes=(10, 12, 14, 16, 18))
    try:
        ref = None
        for nt, tb in autotune.CANDIDATES:
            autotune.set_batch_config(nt, tb)
            got = batch_qaoa(inst, use_graph=True)
            if ref is None:
                ref = got
            assert np.max(np.abs(got - ref)) < 1e-11, (nt, tb)
        for (n, e, g, b), v in list(zip(inst, ref))[:6]:
            assert abs(v - oracle_cut(n, e, g, b)) < 1e-11
        res = autotune.tune_batch_qaoa(inst, repeats=1)
        assert (res["block_threads"], res["tile_bits"]) in autotune.CANDIDATES
        assert autotune.cached_batch_config(inst)["block_threads"] == res["block_threads"]
        tuned = batch_qaoa(inst, tune=True)
        assert np.max(np.abs(tuned - ref)) < 1e-11
    finally:
        autotune.set_batch_config(0, 0)
