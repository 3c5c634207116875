"""Batched circuits in one persistent GPU launch, replayed from a CUDA graph:
QAOA MaxCut instances of uneven width (ket_batch_qaoa) and vqe() energies of
parameterised circuits of uneven width (ket_batch_vqe).

Instance i is (n, edges, gamma[p], beta[p]); the circuit is H on every qubit,
then per layer exp(-i gamma Z_u Z_v) on every edge and Rx(2 beta) on every
qubit, and the result is <C> = sum_edges (1 - <Z_u Z_v>)/2.  In the reference's
terms that is vqe(qaoa(n, edges, -2*gamma, beta), maxCutHamiltonian(n, edges))
(algorithms.ts:231-276).
"""
from __future__ import annotations

import ctypes as C
import weakref
from typing import Sequence, Tuple

import numpy as np

from ._lib import RangeError, check, default_ctx, ket_batch_template, ket_param_binding, lib


def batch_qaoa(instances: Sequence[Tuple[int, Sequence[Tuple[int, int]], Sequence[float], Sequence[float]]],
               use_graph: bool = True, tune: bool = False) -> np.ndarray:
    """Expected cut <C> of every instance (n, edges, gamma, beta).  tune: pick
    the launch shape with the autotuner (ket_b200/autotune.py), timing the
    candidates on this batch the first time a batch of its shape is seen."""
    if not instances:
        return np.zeros(0)
    if tune:
        from . import autotune
        cfg = autotune.cached_batch_config(instances) or autotune.tune_batch_qaoa(instances)
        autotune.set_batch_config(cfg["block_threads"], cfg["tile_bits"])
    return _run(instances, use_graph)


def _run(instances, use_graph: bool) -> np.ndarray:
    p = len(instances[0][2])
    ns, nes, eoff, edges, gam, bet = [], [], [], [], [], []
    for n, e, g, b in instances:
        if len(g) != p or len(b) != p:
            raise TypeError("every instance needs the same number of gamma and beta angles")
        ns.append(n)
        nes.append(len(e))
        eoff.append(len(edges) // 2)
        for u, v in e:
            edges += [u, v]
        gam += list(g)
        bet += list(b)
    N = len(instances)
    n_a = np.ascontiguousarray(ns, dtype=np.int32)
    ne_a = np.ascontiguousarray(nes, dtype=np.int32)
    eo_a = np.ascontiguousarray(eoff, dtype=np.int64)
    ed_a = np.ascontiguousarray(edges or [0, 0], dtype=np.int32)
    g_a = np.ascontiguousarray(gam or [0.0], dtype=np.float64)
    b_a = np.ascontiguousarray(bet or [0.0], dtype=np.float64)
    out = np.zeros(N)
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    check(lib().ket_batch_qaoa(default_ctx(), N, ip(n_a), ip(ne_a), eo_a.ctypes.data_as(C.POINTER(C.c_int64)),
                               ip(ed_a), p, dp(g_a), dp(b_a), 1 if use_graph else 0, dp(out)))
    return out


def batch_vqe(templates, instances, use_graph: bool = True) -> np.ndarray:
    """vqe() energies of many parameterised circuits in one launch.

    templates: [(ansatz, hamiltonian)], an ansatz being a function params ->
    Circuit (AnsatzFn or any callable) on at most 13 qubits and a hamiltonian
    a PauliTerm list, as vqe(ansatz(params), hamiltonian) takes them
    (algorithms.ts:301-336).  instances: [(template index, params)].  Returns
    energy[i] = vqe(ansatz_t(params_i), H_t) for every instance, computed with
    the reference's per-gate pruning; instances of different templates may
    differ in width, gates and Hamiltonian.  Each ansatz is traced once and
    kept while the ansatz object lives, so it must build the same gate list
    on every call (as the adjoint's trace requires)."""
    from .adjoint import _terms
    if not instances:
        return np.zeros(0)
    nparams = max(len(p) for _, p in instances)
    first = {}
    for t, p in instances:
        if not 0 <= t < len(templates):
            raise RangeError(f"instance template index {t} out of range")
        first.setdefault(t, p)
    tmpl = (ket_batch_template * max(1, len(templates)))()
    all_ops, all_mats, all_binds, coeffs, pauli = [], [], [], [], []
    for j, (ansatz, ham) in enumerate(templates):
        p0 = first.get(j)
        if p0 is None:
            p0 = [0.3] * getattr(ansatz, "paramCount", nparams)
        n, arr, m, k, binds = _traced(ansatz, p0)
        terms = _terms(ham, n)
        moff = len(all_mats)
        tmpl[j].nqubits, tmpl[j].nops, tmpl[j].nbinds, tmpl[j].nterms = n, k, len(binds), len(terms)
        tmpl[j].op_first, tmpl[j].bind_first = len(all_ops), len(all_binds)
        tmpl[j].term_first, tmpl[j].pauli_first = len(coeffs), sum(len(x) for x in pauli)
        for i in range(k):
            if arr[i].mat >= 0:
                arr[i].mat += moff
            all_ops.append(arr[i])
        all_mats.extend(m.tolist())
        all_binds.extend(binds)
        for c, o in terms:
            coeffs.append(c)
            pauli.append(o)
    ops_a = (type(all_ops[0]) * max(1, len(all_ops)))(*all_ops) if all_ops else None
    mats = np.ascontiguousarray(np.asarray(all_mats or [0j], dtype=np.complex128)).view(np.float64)
    barr = (ket_param_binding * max(1, len(all_binds)))()
    for i, (op, gate, prm, scale, shift) in enumerate(all_binds):
        barr[i].op, barr[i].gate, barr[i].param, barr[i].scale, barr[i].shift = op, gate, prm, scale, shift
    cf = np.ascontiguousarray(coeffs or [0.0], dtype=np.float64)
    ps = "".join(pauli).encode()
    it = np.ascontiguousarray([t for t, _ in instances], dtype=np.int32)
    if all(len(p) == nparams for _, p in instances):
        th = np.ascontiguousarray(np.asarray([p for _, p in instances], dtype=np.float64).reshape(-1))
    else:
        th = np.zeros((len(instances), max(nparams, 1)))
        for i, (_, p) in enumerate(instances):
            th[i, : len(p)] = p
        th = np.ascontiguousarray(th.reshape(-1))
    out = np.zeros(len(instances))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    check(lib().ket_batch_vqe(default_ctx(), len(templates), tmpl, ops_a, dp(mats), mats.size // 2, barr, dp(cf), ps,
                              len(instances), it.ctypes.data_as(C.POINTER(C.c_int)), dp(th), max(nparams, 1),
                              1 if use_graph else 0, dp(out)))
    return out


# Traced templates, kept per ansatz function while it lives: a parameter sweep
# calls batch_vqe again and again with the same ansatze, and tracing (two
# builds of the circuit) costs more host time than the batch's kernel.
_TRACE_CACHE = weakref.WeakKeyDictionary()


def _traced(ansatz, p0):
    """(n, ket_op array, matrices, count, bindings) of an ansatz, traced once."""
    from .adjoint import trace
    from .circuit import ops_to_abi
    key = len(p0)
    try:
        hit = _TRACE_CACHE.get(ansatz, {}).get(key)
    except TypeError:  # not weak-referenceable: trace every time
        hit = None
    if hit is None:
        n, ops, binds = trace(ansatz, [float(v) for v in p0])
        arr, m, k = ops_to_abi(ops)
        hit = (n, arr, m, k, binds)
        try:
            _TRACE_CACHE.setdefault(ansatz, {})[key] = hit
        except TypeError:
            pass
    n, arr, m, k, binds = hit
    arr2 = (type(arr[0]) * max(1, k))()
    C.memmove(arr2, arr, C.sizeof(arr2))  # the caller shifts matrix offsets in its copy
    return n, arr2, m, k, binds
