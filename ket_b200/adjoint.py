"""Adjoint gradients for ket's variational API (gradient() / minimize(),
algorithms.ts:536-609) on the GPU engine.

An ansatz is a Python function params -> Circuit, as in the reference.  To
differentiate it in one reverse sweep, the ansatz is traced once: it is called
with parameter stand-ins (float subclasses that remember `scale * params[k] +
shift`), and every rotation built from one becomes a parametric binding of the
circuit template.  A second build with different parameter values checks that
no other gate depends on the parameters (e.g. through math.cos), in which case
TraceError is raised and gradient() falls back to the reference's parameter
shift.
"""
from __future__ import annotations

import ctypes as C
import math
import random
from typing import List, Sequence, Tuple

import numpy as np

from ._lib import PG, check, default_ctx, ket_param_binding, lib
from .circuit import Circuit, flatten_ops, ops_to_abi


class TraceError(Exception):
    """The ansatz cannot be traced into a parametric template."""


class Sym(float):
    """scale * params[index] + shift, carried through affine arithmetic."""

    def __new__(cls, value, index, scale=1.0, shift=0.0):
        o = float.__new__(cls, value)
        o.index, o.scale, o.shift = index, scale, shift
        return o

    def _affine(self, mul, add):
        return Sym(float(self) * mul + add, self.index, self.scale * mul, self.shift * mul + add)

    def __neg__(self):
        return self._affine(-1.0, 0.0)

    def __pos__(self):
        return self

    def __mul__(self, o):
        if isinstance(o, Sym):
            raise TraceError("product of two parameters")
        if isinstance(o, (int, float)):
            return self._affine(float(o), 0.0)
        return NotImplemented

    __rmul__ = __mul__

    def __truediv__(self, o):
        if isinstance(o, Sym):
            raise TraceError("quotient of two parameters")
        if isinstance(o, (int, float)):
            return self._affine(1.0 / float(o), 0.0)
        return NotImplemented

    def __add__(self, o):
        if isinstance(o, Sym):
            raise TraceError("sum of two parameters")
        if isinstance(o, (int, float)):
            return self._affine(1.0, float(o))
        return NotImplemented

    __radd__ = __add__

    def __sub__(self, o):
        if isinstance(o, Sym):
            raise TraceError("difference of two parameters")
        if isinstance(o, (int, float)):
            return self._affine(1.0, -float(o))
        return NotImplemented

    def __rsub__(self, o):
        if isinstance(o, (int, float)):
            return self._affine(-1.0, float(o))
        return NotImplemented


def trace(ansatz, params: Sequence[float]):
    """Template op list + bindings of `ansatz` at `params`."""
    syms = [Sym(float(v), i) for i, v in enumerate(params)]
    circ = ansatz(syms)
    ops = flatten_ops(circ.ops)
    binds = []
    for i, op in enumerate(ops):
        sp = [p for p in op.params if isinstance(p, Sym)]
        if not sp:
            continue
        if len(op.params) != 1 or op.name not in PG:
            raise TraceError(f"parameter used in gate '{op.name}' (only one-angle rotations are differentiable)")
        s = sp[0]
        binds.append((i, PG[op.name], s.index, s.scale, s.shift))
    # any other dependence on the parameters shows up as a changed matrix
    other = [float(v) + 0.37 + 0.11 * random.random() for v in params]
    ops2 = flatten_ops(ansatz(other).ops)
    bound = {b[0] for b in binds}
    if len(ops2) != len(ops):
        raise TraceError("the ansatz's gate list depends on the parameter values")
    for i, (a, b) in enumerate(zip(ops, ops2)):
        if a.kind != b.kind or a.qubits != b.qubits:
            raise TraceError("the ansatz's gate list depends on the parameter values")
        if i not in bound and a.gate != b.gate:
            raise TraceError(f"gate {i} ('{a.name}') depends on the parameters in an untraceable way")
    return circ.qubits, ops, binds


MIN_QUBITS = 12  # one register tile: smaller circuits are padded with idle qubits


def _abi(n, ops, binds, hamiltonian):
    arr, m, k = ops_to_abi(ops)
    nb = len(binds)
    barr = (ket_param_binding * max(1, nb))()
    for j, (op, gate, p, scale, shift) in enumerate(binds):
        barr[j].op, barr[j].gate, barr[j].param = op, gate, p
        barr[j].scale, barr[j].shift = scale, shift
    terms = hamiltonian
    coeffs = np.ascontiguousarray([t[0] for t in terms] or [0.0], dtype=np.float64)
    opsb = "".join(t[1] for t in terms).encode()
    return arr, m, k, barr, nb, coeffs, opsb, len(terms)


def _terms(hamiltonian, n, pad_to=None):
    from .algorithms import _terms as tt
    terms = tt(hamiltonian)
    for c, o in terms:
        if len(o) != n:
            raise TypeError(f"ops '{o}' length must equal ansatz.qubits ({n})")
    if pad_to and pad_to > n:  # ops[0] acts on the top qubit: idle qubits are prepended as I
        terms = [(c, "I" * (pad_to - n) + o) for c, o in terms]
    return terms


def adjoint_gradient(ansatz, hamiltonian, params_batch, init: int = 0, checkpoint_every: int = 0):
    """(energies[B], gradients[B][P]) for each parameter vector of the batch."""
    pb = [list(map(float, p)) for p in params_batch]
    n, ops, binds = trace(ansatz, pb[0])
    P = len(pb[0])
    N = max(n, MIN_QUBITS)
    arr, m, k, barr, nb, coeffs, opsb, nt = _abi(n, ops, binds, _terms(hamiltonian, n, N))
    theta = np.ascontiguousarray(pb, dtype=np.float64).reshape(-1) if P else np.zeros(1)
    B = len(pb)
    energy = np.zeros(max(B, 1))
    grad = np.zeros(max(B * P, 1))
    mv = np.ascontiguousarray(m).view(np.float64)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    n = N
    check(lib().ket_adjoint_gradient(default_ctx(), n, init, arr, k, dp(mv), m.size, barr, nb, dp(theta), P, B, nt,
                                     dp(coeffs), opsb, checkpoint_every, dp(energy), dp(grad)))
    return energy[:B], grad[: B * P].reshape(B, P)


def shift_gradient(ansatz, hamiltonian, params_batch, init: int = 0, prune: bool = False):
    """The reference's parameter-shift gradient, computed by the engine."""
    pb = [list(map(float, p)) for p in params_batch]
    n, ops, binds = trace(ansatz, pb[0])
    P = len(pb[0])
    arr, m, k, barr, nb, coeffs, opsb, nt = _abi(n, ops, binds, _terms(hamiltonian, n))
    theta = np.ascontiguousarray(pb, dtype=np.float64).reshape(-1) if P else np.zeros(1)
    B = len(pb)
    energy = np.zeros(max(B, 1))
    grad = np.zeros(max(B * P, 1))
    mv = np.ascontiguousarray(m).view(np.float64)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    check(lib().ket_shift_gradient(default_ctx(), n, init, arr, k, dp(mv), m.size, barr, nb, dp(theta), P, B, nt,
                                   dp(coeffs), opsb, 1 if prune else 0, dp(energy), dp(grad)))
    return energy[:B], grad[: B * P].reshape(B, P)
