"""Shared helpers: build one case on the oracle (CPU checker) or on the GPU
engine's Circuit API, and evaluate the reference-style read-outs."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_kats():
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        return json.load(f)["cases"]


def tol(digits):
    """vitest toBeCloseTo(x, d): |got - x| < 0.5 * 10^-d."""
    return 0.5 * 10.0 ** (-digits)


def unitary_matrix(rows):
    return [[complex(r[2 * j], r[2 * j + 1]) for j in range(len(r) // 2)] for r in rows]


def oracle_circuit(case):
    from oracle import oracle as O
    c = O.OCircuit(case["n"])
    for name, qs, ps in case["gates"]:
        if name == "unitary":
            c.unitary(unitary_matrix(ps), qs)
        else:
            c.add(name, qs, ps)
    return c


def ket_circuit(case):
    from ket_b200 import Circuit
    c = Circuit(case["n"])
    for name, qs, ps in case["gates"]:
        if name == "unitary":
            c = c.unitary(unitary_matrix(ps), *qs)
        else:
            c = getattr(c, name)(*ps, *qs)
    return c


def bit_index(bs):
    return int(bs[::-1], 2)


def init_index(case):
    return bit_index(case["init"]) if case.get("init") else 0
