"""Batched QAOA MaxCut: thousands of instances of uneven width in one
persistent GPU launch (ket_batch_qaoa), replayed from a CUDA graph.

Instance i is (n, edges, gamma[p], beta[p]); the circuit is H on every qubit,
then per layer exp(-i gamma Z_u Z_v) on every edge and Rx(2 beta) on every
qubit, and the result is <C> = sum_edges (1 - <Z_u Z_v>)/2.  In the reference's
terms that is vqe(qaoa(n, edges, -2*gamma, beta), maxCutHamiltonian(n, edges))
(algorithms.ts:231-276).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence, Tuple

import numpy as np

from ._lib import check, default_ctx, lib


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
