"""Adjoint gradients (ket_adjoint_gradient) against the engine's parameter
shift, central finite differences, the reference's gradient KATs and the
oracle's parameter shift (the reference algorithm).

Tolerances: adjoint vs parameter shift on the same engine 1e-10 (the target
bar); vs central differences with eps = 1e-6, 1e-7 (the difference quotient's
own rounding error is ~1e-9 * |E|/eps^2 ... ~1e-8)."""
import math
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def tfim(n, seed=3):
    from ket_b200 import workloads as W
    rnd = random.Random(seed)
    return W.tfim_hamiltonian(n, [0.5 + rnd.random() for _ in range(n)])


def test_gradient_kats_via_adjoint():
    """gradient() KATs of the reference suite (circuit.test.ts:4168-4219) on the adjoint path."""
    import ket_b200 as K
    Z = [(1.0, "Z")]
    ans = lambda p: K.Circuit(1).ry(p[0], 0)
    for theta, want in [(0.0, 0.0), (math.pi / 4, -math.sin(math.pi / 4)), (math.pi, 0.0)]:
        (g,) = K.gradient(ans, Z, [theta], method="adjoint")
        assert abs(g - want) < 0.5e-10
    ans2 = lambda p: K.Circuit(2).ry(p[0], 0).ry(p[1], 1)
    p0, p1 = math.pi / 3, math.pi / 6
    g = K.gradient(ans2, [(1.0, "ZI"), (1.0, "IZ")], [p0, p1], method="adjoint")
    assert abs(g[0] + math.sin(p0)) < 0.5e-10 and abs(g[1] + math.sin(p1)) < 0.5e-10
    (g,) = K.gradient(lambda p: K.Circuit(1).h(0).rz(p[0], 0), [(1.0, "X")], [math.pi / 4], method="adjoint")
    assert abs(g + math.sin(math.pi / 4)) < 0.5e-10
    (g,) = K.gradient(lambda p: K.Circuit(1).rx(p[0], 0), [(1.0, "Y")], [math.pi / 4], method="adjoint")
    assert abs(g + math.cos(math.pi / 4)) < 0.5e-10
    g = K.gradient(lambda p: K.Circuit(2).ry(p[0], 0).cnot(0, 1).ry(p[1], 1), [(1.0, "ZZ")], [0.5, math.pi / 4],
                   method="adjoint")
    assert abs(g[0]) < 0.5e-10 and abs(g[1] + math.sin(math.pi / 4)) < 0.5e-10
    assert K.gradient(lambda p: K.Circuit(1).h(0), Z, []) == []


def test_adjoint_matches_shift_and_finite_differences():
    from ket_b200 import workloads as W
    from ket_b200.adjoint import adjoint_gradient, shift_gradient
    n, layers = 12, 3
    ans = W.hea_ladder(n, layers)
    H = tfim(n)
    rnd = np.random.default_rng(5)
    P = rnd.uniform(0, 2 * np.pi, size=(2, ans.paramCount))
    e_adj, g_adj = adjoint_gradient(ans, H, P)
    e_sh, g_sh = shift_gradient(ans, H, P)
    assert np.max(np.abs(e_adj - e_sh)) < 1e-11
    assert np.max(np.abs(g_adj - g_sh)) < 1e-10
    # central differences on a few parameters
    import ket_b200 as K
    eps = 1e-6
    for k in (0, 7, ans.paramCount - 1):
        pp, pm = P[0].copy(), P[0].copy()
        pp[k] += eps
        pm[k] -= eps
        fd = (K.vqe(ans(list(pp)), H) - K.vqe(ans(list(pm)), H)) / (2 * eps)
        assert abs(fd - g_adj[0, k]) < 1e-7


def test_adjoint_vs_oracle_parameter_shift():
    """The oracle runs the reference's own gradient(): parameter shift over
    vqe(), each energy a re-simulation per Pauli term with pruning."""
    from ket_b200.adjoint import adjoint_gradient
    from ket_b200.algorithms import efficientSU2
    from oracle import oracle as O
    n, reps = 12, 1
    ans = efficientSU2(n, reps)
    H = [(t.coeff, t.ops) for t in tfim(n)][:6] + [(0.3, "X" * n)]
    rnd = np.random.default_rng(9)
    p = rnd.uniform(0, 2 * np.pi, size=ans.paramCount)
    _, g = adjoint_gradient(ans, H, [p])
    g_ref = O.gradient(O.ANS_EFFICIENT_SU2, n, reps, p, H, mode=O.DENSE)
    assert np.max(np.abs(g[0] - g_ref)) < 1e-10


def test_adjoint_gate_families_and_controls():
    """Controlled, two-qubit and IonQ-native parametric gates, affine angles."""
    import ket_b200 as K
    from ket_b200.adjoint import adjoint_gradient, shift_gradient

    def ans(p):
        c = K.Circuit(12)
        for q in range(12):
            c = c.h(q)
        c = c.crx(p[0], 0, 5).cry(2 * p[1] + 0.3, 6, 1).crz(-p[2], 11, 3).cu1(p[3] / 2, 2, 9)
        c = c.xx(p[4], 1, 7).yy(p[5], 8, 2).zz(p[6], 3, 10).xy(p[7], 4, 11)
        c = c.gpi(p[8], 5).gpi2(p[9], 6).rz(p[0], 7).u1(p[1], 8).ry(p[2] - 1.0, 9)
        return c

    H = tfim(12) + [(0.4, "Y" * 12), (0.2, "XYZ" * 4)]
    p = list(np.random.default_rng(1).uniform(0, 2 * np.pi, 10))
    _, ga = adjoint_gradient(ans, H, [p])
    # the parameter-shift rule is exact only for exp(-i a P / 2) gates; compare
    # to central differences for all, shift where exact
    import ket_b200 as KK
    eps = 1e-6
    for k in range(10):
        pp, pm = list(p), list(p)
        pp[k] += eps
        pm[k] -= eps
        fd = (KK.vqe(ans(pp), H) - KK.vqe(ans(pm), H)) / (2 * eps)
        assert abs(fd - ga[0, k]) < 1e-7, k


def test_trace_errors_fall_back_to_shift():
    import ket_b200 as K
    from ket_b200.adjoint import TraceError, trace

    def bad(p):
        return K.Circuit(1).ry(math.cos(p[0]), 0)  # untraceable dependence

    with pytest.raises(TraceError):
        trace(bad, [0.3])
    g_auto = K.gradient(bad, [(1.0, "Z")], [0.3])              # falls back to parameter shift
    g_shift = K.gradient_shift(bad, [(1.0, "Z")], [0.3])
    assert abs(g_auto[0] - g_shift[0]) < 1e-15


def test_minimize_kat_adjoint():
    """minimize() KAT (circuit.test.ts:4240-4244) with adjoint gradients."""
    import ket_b200 as K
    r = K.minimize(lambda p: K.Circuit(1).ry(p[0], 0), [(1.0, "Z")], [0.1])
    assert abs(r.energy + 1) < 0.5e-4 and r.converged


def test_host_checkpoints_match_device_checkpoints():
    """With no device memory allowed for checkpoints (a host-side budget, no
    fault), every checkpoint of psi goes to pinned host memory; the gradients
    are the same bit for bit as with device checkpoints."""
    from ket_b200 import _lib
    from ket_b200 import workloads as W
    from ket_b200.adjoint import adjoint_gradient
    ans = W.hea_ladder(14, 4)
    H = tfim(14)
    P = np.random.default_rng(21).uniform(0, 2 * np.pi, size=(3, ans.paramCount))
    e_dev, g_dev = adjoint_gradient(ans, H, P)
    L = _lib.lib()
    try:
        L.ket_debug_adjoint_budget(0)
        e_host, g_host = adjoint_gradient(ans, H, P)
    finally:
        L.ket_debug_adjoint_budget(-1)
    assert np.array_equal(e_dev, e_host) and np.array_equal(g_dev, g_host)


def test_adjoint_batch_on_compiled_kernels_matches_single_vectors():
    """A batch of 8 or more runs its passes on compiled kernels with every
    vector queued without a host wait; each vector's gradient equals the one
    computed alone (interpreter passes) to rounding."""
    from ket_b200 import workloads as W
    from ket_b200.adjoint import adjoint_gradient
    ans = W.hea_ladder(13, 3)
    H = tfim(13)
    P = np.random.default_rng(33).uniform(0, 2 * np.pi, size=(9, ans.paramCount))
    e_b, g_b = adjoint_gradient(ans, H, P)
    for k in (0, 4, 8):
        e1, g1 = adjoint_gradient(ans, H, P[k:k + 1])
        assert abs(e1[0] - e_b[k]) < 1e-12
        assert np.max(np.abs(g1[0] - g_b[k])) < 1e-12
