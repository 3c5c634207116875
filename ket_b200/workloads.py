"""Seeded synthetic workloads (all inputs synthetic; no dataset is involved).

Every generator draws from makePrng (xorshift32, circuit.ts:813-819) seeded
with 42, in a fixed draw order:

* brickwork(n, layers): per layer, per qubit g = floor(rng()*5) picks
  {0:H, 1:T, 2:Rx, 3:Ry, 4:Rz}; rotations then draw theta = rng()*2*pi; then
  CNOT(q, q+1) for even q on even layers and odd q on odd layers.
* brickwork_qft(n, layers): the same circuit followed by qft(n); the stream
  then continues with the amplitude indices idx = u32 >> (32 - n).
* qaoa_batch: n = 10 + 2*floor(rng()*7) (uniform on {10,...,22}); a random
  3-regular graph by the pairing model with rejection (Fisher-Yates shuffle of
  the 3n half-edges, reject self-loops and multi-edges); then per layer
  gamma = rng()*pi, beta = rng()*pi.
* tfim_vqe: fields h_i = 0.5 + rng() for i = 0..n-1, then batch parameter
  vectors theta = rng()*2*pi.
* vqe_batch: per template width n (ascending), fields h_i = 0.5 + rng() for
  the TFIM; then per instance a template t = floor(rng()*T) and its
  parameters theta = rng()*2*pi.
* midcircuit_brickwork(n, layers): brickwork(n, layers), measure q0 into c[0],
  reset q0, then brickwork(n, layers // 2) on the same stream (run() with
  noise exercises the per-shot path on it).

oracle/ket_oracle.cpp draws the identical streams for the parity tests.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

from .algorithms import PauliTerm, qft
from .circuit import Circuit


class Xorshift32:
    def __init__(self, seed: int = 42):
        self.s = (int(seed) & 0xFFFFFFFF) or 1

    def next_u32(self) -> int:
        x = self.s
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        self.s = x
        return x

    def __call__(self) -> float:
        return self.next_u32() / 4294967296.0


def brickwork(n: int, layers: int, rng: Xorshift32, c: Circuit = None) -> Circuit:
    c = Circuit(n) if c is None else c
    for l in range(layers):
        for q in range(n):
            g = math.floor(rng() * 5)
            if g == 0:
                c = c.h(q)
            elif g == 1:
                c = c.t(q)
            else:
                th = rng() * 2 * math.pi
                c = (c.rx if g == 2 else c.ry if g == 3 else c.rz)(th, q)
        for q in range(l & 1, n - 1, 2):
            c = c.cnot(q, q + 1)
    return c


def brickwork_circuit(n: int, layers: int, seed: int = 42) -> Tuple[Circuit, Xorshift32]:
    rng = Xorshift32(seed)
    return brickwork(n, layers, rng), rng


def midcircuit_brickwork(n: int, layers: int, seed: int = 42) -> Circuit:
    """The per-shot path's workload: brickwork(n, layers) from the seeded
    stream, then measure q0 into c[0] and reset q0, then brickwork(n,
    layers // 2) continuing the stream."""
    rng = Xorshift32(seed)
    c = brickwork(n, layers, rng)
    c = c.measure(0, "c", 0).reset(0)
    return brickwork(n, layers // 2, rng, c)


def brickwork_qft(n: int, layers: int, seed: int = 42, n_amps: int = 1024):
    """Brickwork + qft(n); returns (circuit, amplitude indices)."""
    rng = Xorshift32(seed)
    c = brickwork(n, layers, rng)
    c = c.append(qft(n))
    idx = [rng.next_u32() >> (32 - n) for _ in range(n_amps)]
    return c, idx


def regular3(n: int, rng: Xorshift32) -> List[Tuple[int, int]]:
    while True:
        pts = [i // 3 for i in range(3 * n)]
        for i in range(3 * n - 1, 0, -1):
            j = math.floor(rng() * (i + 1))
            pts[i], pts[j] = pts[j], pts[i]
        edges, seen, ok = [], set(), True
        for k in range(3 * n // 2):
            u, v = pts[2 * k], pts[2 * k + 1]
            if u == v:
                ok = False
                break
            if u > v:
                u, v = v, u
            if (u, v) in seen:
                ok = False
                break
            seen.add((u, v))
            edges.append((u, v))
        if ok:
            return edges


def qaoa_batch(ninst: int = 4096, p: int = 4, seed: int = 42, sizes: Sequence[int] = (10, 12, 14, 16, 18, 20, 22)):
    """Instances (n, edges, gamma[p], beta[p]) of the QAOA MaxCut batch."""
    rng = Xorshift32(seed)
    out = []
    for _ in range(ninst):
        n = sizes[math.floor(rng() * len(sizes))]
        edges = regular3(n, rng)
        gamma, beta = [], []
        for _ in range(p):
            gamma.append(rng() * math.pi)
            beta.append(rng() * math.pi)
        out.append((n, edges, gamma, beta))
    return out


def hea_ladder(n: int, layers: int):
    """Layers of (Ry(theta), Rz(theta) on every qubit, then CNOT(q, q+1) for q = 0..n-2);
    layer l, qubit q uses params 2(n*l + q) (Ry) and 2(n*l + q) + 1 (Rz)."""
    from .algorithms import AnsatzFn
    pc = 2 * n * layers

    def fn(params):
        if len(params) != pc:
            raise ValueError(f"hea_ladder({n}, {layers}) needs {pc} params, got {len(params)}")
        c, k = Circuit(n), 0
        for _ in range(layers):
            for q in range(n):
                c = c.ry(params[k], q).rz(params[k + 1], q)
                k += 2
            for q in range(n - 1):
                c = c.cnot(q, q + 1)
        return c

    return AnsatzFn(pc, fn)


def tfim_hamiltonian(n: int, h: Sequence[float]) -> List[PauliTerm]:
    """H = -sum_i Z_i Z_{i+1} - sum_i h_i X_i as PauliTerms (ops[0] = qubit n-1)."""
    terms = []
    for i in range(n - 1):
        arr = ["I"] * n
        arr[n - 1 - i] = "Z"
        arr[n - 1 - (i + 1)] = "Z"
        terms.append(PauliTerm(-1.0, "".join(arr)))
    for i in range(n):
        arr = ["I"] * n
        arr[n - 1 - i] = "X"
        terms.append(PauliTerm(-h[i], "".join(arr)))
    return terms


def tfim_vqe(n: int = 24, layers: int = 8, batch: int = 64, seed: int = 42):
    """(ansatz, hamiltonian, params[batch][2*n*layers]) of the adjoint-gradient workload."""
    rng = Xorshift32(seed)
    h = [0.5 + rng() for _ in range(n)]
    ansatz = hea_ladder(n, layers)
    params = [[rng() * 2 * math.pi for _ in range(ansatz.paramCount)] for _ in range(batch)]
    return ansatz, tfim_hamiltonian(n, h), params


def vqe_batch(ninst: int = 1024, sizes: Sequence[int] = (8, 9, 10, 11, 12, 13), layers: int = 4, seed: int = 42):
    """The batched VQE workload: templates [(hea_ladder(n, layers), TFIM(n))] for
    every n in sizes, and ninst instances (template index, parameters) drawn
    uniformly over the templates -- a parameter sweep over circuits of uneven
    width."""
    rng = Xorshift32(seed)
    templates = []
    for n in sizes:
        h = [0.5 + rng() for _ in range(n)]
        templates.append((hea_ladder(n, layers), tfim_hamiltonian(n, h)))
    inst = []
    for _ in range(ninst):
        t = math.floor(rng() * len(sizes))
        pc = templates[t][0].paramCount
        inst.append((t, [rng() * 2 * math.pi for _ in range(pc)]))
    return templates, inst
