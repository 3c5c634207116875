"""Algorithms on the statevector path: the circuit builders and variational
loops of the reference's src/algorithms.ts, over the GPU engine.

qft / iqft / qaoa / maxCutHamiltonian / realAmplitudes / efficientSU2 build the
same op lists as the reference.  vqe() returns the same energy but computes it
from one simulation (the reference re-simulates once per Pauli term with a
basis rotation).  gradient() offers the reference's parameter shift and an
adjoint reverse sweep (ket_adjoint_gradient) that gives all P derivatives from
one forward and one backward pass.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence, Tuple, Union

import numpy as np

from .circuit import Circuit


# ---------------------------------------------------------------- QFT (algorithms.ts:16-38)
def qft(n: int) -> Circuit:
    c = Circuit(n)
    for j in range(n - 1, -1, -1):
        c = c.h(j)
        for k in range(j - 1, -1, -1):
            c = c.cu1(math.pi / 2 ** (j - k), k, j)
    for i in range(n // 2):
        c = c.swap(i, n - 1 - i)
    return c


def iqft(n: int) -> Circuit:
    c = Circuit(n)
    for i in range(n // 2):
        c = c.swap(i, n - 1 - i)
    for j in range(n):
        for k in range(j - 1, -1, -1):
            c = c.cu1(-math.pi / 2 ** (j - k), k, j)
        c = c.h(j)
    return c


# ---------------------------------------------------------------- Pauli terms
@dataclass(frozen=True)
class PauliTerm:
    """coeff * (P_{n-1} ⊗ ... ⊗ P_0): ops[0] acts on qubit n-1 (algorithms.ts:278-288)."""
    coeff: float
    ops: str


TermLike = Union[PauliTerm, Tuple[float, str], dict]


def _terms(hamiltonian) -> List[Tuple[float, str]]:
    out = []
    for t in hamiltonian:
        if isinstance(t, PauliTerm):
            out.append((float(t.coeff), t.ops))
        elif isinstance(t, dict):
            out.append((float(t["coeff"]), t["ops"]))
        else:
            out.append((float(t[0]), t[1]))
    return out


# ---------------------------------------------------------------- QAOA (algorithms.ts:231-276)
def maxCutHamiltonian(n: int, edges: Sequence[Tuple[int, int]]) -> List[PauliTerm]:
    if len(edges) == 0:
        return []
    terms = [PauliTerm(len(edges) / 2, "I" * n)]
    for u, v in edges:
        arr = ["I"] * n
        arr[n - 1 - u] = "Z"
        arr[n - 1 - v] = "Z"
        terms.append(PauliTerm(-0.5, "".join(arr)))
    return terms


def qaoa(n: int, edges: Sequence[Tuple[int, int]], gamma: Sequence[float], beta: Sequence[float]) -> Circuit:
    if len(gamma) != len(beta):
        raise TypeError(f"gamma and beta must have equal length (got {len(gamma)} vs {len(beta)})")
    c = Circuit(n)
    for q in range(n):
        c = c.h(q)
    for l in range(len(gamma)):
        for u, v in edges:
            c = c.cnot(u, v).rz(-gamma[l], v).cnot(u, v)
        for q in range(n):
            c = c.rx(2 * beta[l], q)
    return c


# ---------------------------------------------------------------- VQE (algorithms.ts:301-336)
def vqe(ansatz: Circuit, hamiltonian) -> float:
    """<ansatz|H|ansatz>: terms with |coeff| < 1e-15 are skipped and identity
    terms add their coefficient, as in the reference."""
    n = ansatz.qubits
    terms = _terms(hamiltonian)
    for coeff, ops in terms:
        if len(ops) != n:
            raise TypeError(f"ops '{ops}' length must equal ansatz.qubits ({n})")
    if not terms:
        return 0.0
    if all(abs(c) < 1e-15 or not any(ch in "XYZ" for ch in o.upper()) for c, o in terms):
        return float(sum(c for c, o in terms if abs(c) >= 1e-15))
    ansatz._require_pure("exactProbs()")
    return ansatz._state().expect_pauli_sum(terms)


# ---------------------------------------------------------------- ansatz families (algorithms.ts:341-399)
class AnsatzFn:
    """An ansatz function with its parameter count (AnsatzFn, algorithms.ts:341-349)."""

    def __init__(self, param_count: int, fn: Callable[[Sequence[float]], Circuit]):
        self.paramCount = param_count
        self._fn = fn

    def __call__(self, params):
        return self._fn(params)


def realAmplitudes(n: int, reps: int = 3) -> AnsatzFn:
    pc = n * (reps + 1)

    def fn(params):
        if len(params) != pc:
            raise ValueError(f"realAmplitudes({n}, {reps}) needs {pc} params, got {len(params)}")
        c, p = Circuit(n), 0
        for _ in range(reps):
            for q in range(n):
                c = c.ry(params[p], q); p += 1
            for q in range(n - 1):
                c = c.cnot(q, q + 1)
        for q in range(n):
            c = c.ry(params[p], q); p += 1
        return c

    return AnsatzFn(pc, fn)


def efficientSU2(n: int, reps: int = 3) -> AnsatzFn:
    pc = 2 * n * (reps + 1)

    def fn(params):
        if len(params) != pc:
            raise ValueError(f"efficientSU2({n}, {reps}) needs {pc} params, got {len(params)}")
        c, p = Circuit(n), 0
        for _ in range(reps):
            for q in range(n):
                c = c.ry(params[p], q).rz(params[p + 1], q); p += 2
            for q in range(n - 1):
                c = c.cnot(q, q + 1)
        for q in range(n):
            c = c.ry(params[p], q).rz(params[p + 1], q); p += 2
        return c

    return AnsatzFn(pc, fn)


# ---------------------------------------------------------------- gradients (algorithms.ts:536-609)
def gradient_shift(ansatz, hamiltonian, params: Sequence[float]) -> List[float]:
    """Parameter shift, exactly the reference's gradient(): 2P energy evaluations."""
    shift = math.pi / 2
    out = []
    for i in range(len(params)):
        plus = [p + shift if j == i else p for j, p in enumerate(params)]
        minus = [p - shift if j == i else p for j, p in enumerate(params)]
        out.append(0.5 * (vqe(ansatz(plus), hamiltonian) - vqe(ansatz(minus), hamiltonian)))
    return out


def gradient(ansatz, hamiltonian, params: Sequence[float], method: str = "auto") -> List[float]:
    """gradient() (algorithms.ts:536-547).  method: 'adjoint' (one reverse
    sweep), 'shift' (the reference's parameter shift) or 'auto' (adjoint when
    the ansatz can be traced, else shift)."""
    if method == "shift":
        return gradient_shift(ansatz, hamiltonian, params)
    from .adjoint import adjoint_gradient, TraceError
    if len(params) == 0:
        return []
    try:
        _, g = adjoint_gradient(ansatz, hamiltonian, [list(params)])
        return [float(v) for v in g[0]]
    except TraceError:
        if method == "adjoint":
            raise
        return gradient_shift(ansatz, hamiltonian, params)


@dataclass
class MinimizeResult:
    params: List[float]
    energy: float
    steps: int
    converged: bool
    truncated: bool = False


def minimize(ansatz, hamiltonian, initialParams: Sequence[float], lr: float = 0.1, steps: int = 200,
             tol: float = 1e-6, method: str = "auto") -> MinimizeResult:
    """minimize() (algorithms.ts:591-609): gradient descent until the gradient
    norm drops below tol."""
    params = list(initialParams)
    for step in range(steps):
        grad = gradient(ansatz, hamiltonian, params, method=method)
        norm = math.sqrt(sum(g * g for g in grad))
        if norm < tol:
            return MinimizeResult(params, vqe(ansatz(params), hamiltonian), step, True)
        params = [p - lr * g for p, g in zip(params, grad)]
    return MinimizeResult(params, vqe(ansatz(params), hamiltonian), steps, False)
