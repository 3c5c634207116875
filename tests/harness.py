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


# ---------------------------------------------------------------- run()'s per-shot path
def load_pershot_kats():
    with open(os.path.join(GOLDEN, "pershot_kats.json")) as f:
        return json.load(f)["cases"]


def case_registers(case):
    """{name: (first bit, size)}: the circuit's classical registers in the
    order the reference's #cregs Map holds them (creg() and measure()
    register at the top level only; an if-body's builder circuit is
    discarded)."""
    sizes = {}
    for op in case["ops"]:
        if op[0] == "creg":
            sizes[op[1]] = op[2]
        elif op[0] == "measure":
            sizes[op[2]] = max(sizes.get(op[2], 0), op[3] + 1)
    out, nb = {}, 0
    for name, size in sizes.items():
        out[name] = (nb, size)
        nb += size
    return out, nb


def _oracle_ops(c, ops, regs, n):
    from oracle import oracle as O
    for op in ops:
        if op[0] == "creg":
            continue
        if op[0] == "measure":
            reg = regs.get(op[2])
            c.measure(op[1], reg[0] + op[3] if reg is not None and op[3] < reg[1] else -1)
        elif op[0] == "reset":
            c.reset(op[1])
            if op[2] == 1:
                c.add("x", [op[1]])
        elif op[0] == "if":
            body = O.OCircuit(n)
            _oracle_ops(body, op[3], regs, n)
            first, size = regs.get(op[1], (0, 0))
            c.if_(first, size, op[2], body)
        elif op[0] == "unitary":
            c.unitary(unitary_matrix(op[2]), op[1])
        else:
            c.add(op[0], op[1], op[2])


def pershot_noise(case):
    from ket_b200.circuit import resolve_noise
    return resolve_noise(case["run"]["noise"])


def pershot_oracle_raw(case, shots=None, seed=None):
    """The oracle's per-shot run: (index per shot, bits [shots, ncbits], registers)."""
    from oracle import oracle as O
    from ket_b200.circuit import make_prng
    regs, nb = case_registers(case)
    c = O.OCircuit(case["n"])
    _oracle_ops(c, case["ops"], regs, case["n"])
    nz = pershot_noise(case) or (0.0, 0.0, 0.0)
    shots = case["run"]["shots"] if shots is None else shots
    seed = case["run"]["seed"] if seed is None else seed
    idx, bits, _ = c.run_pershot(shots, make_prng(seed).state[0], nz[0], nz[1], nz[2], nb)
    return idx, bits, regs


def summarize(n, idx, bits, regs):
    shots = len(idx)
    probs = {}
    for i in idx.tolist():
        k = format(int(i), "b").zfill(n)[::-1]
        probs[k] = probs.get(k, 0) + 1
    probs = {k: v / shots for k, v in probs.items()}
    cregs = {name: [float(bits[:, f + j].sum()) / shots for j in range(s)] for name, (f, s) in regs.items()}
    return probs, cregs


def ket_pershot_circuit(case):
    from ket_b200 import Circuit

    def build(c, ops):
        for op in ops:
            if op[0] == "creg":
                c = c.creg(op[1], op[2])
            elif op[0] == "measure":
                c = c.measure(op[1], op[2], op[3])
            elif op[0] == "reset":
                c = c.reset(op[1], op[2])
            elif op[0] == "if":
                body = op[3]
                c = c.if_(op[1], op[2], lambda b, body=body: build(b, body))
            elif op[0] == "unitary":
                c = c.unitary(unitary_matrix(op[2]), *op[1])
            else:
                c = getattr(c, op[0])(*op[2], *op[1])
        return c

    return build(Circuit(case["n"]), case["ops"])


def check_pershot(case, probs, cregs, clean=None):
    """The assertions of the reference test a case restates."""
    def psum(keys):
        return sum(probs.get(k, 0.0) for k in keys)

    for chk in case["checks"]:
        kind = chk[0]
        if kind == "creg":
            assert abs(cregs[chk[1]][chk[2]] - chk[3]) < tol(chk[4]), (case["id"], chk, cregs)
        elif kind == "creg_near":
            assert abs(cregs[chk[1]][chk[2]] - chk[3]) <= chk[4], (case["id"], chk, cregs)
        elif kind == "creg_match":
            assert abs(cregs[chk[1]][0] - cregs[chk[2]][0]) < tol(chk[3]), (case["id"], chk, cregs)
        elif kind == "prob":
            assert abs(probs.get(chk[1], 0.0) - chk[2]) < tol(chk[3]), (case["id"], chk, probs)
        elif kind == "prob_near":
            assert abs(probs.get(chk[1], 0.0) - chk[2]) <= chk[3], (case["id"], chk, probs)
        elif kind == "sum_gt":
            assert psum(chk[1]) > chk[2], (case["id"], chk, probs)
        elif kind == "sum_lt":
            assert psum(chk[1]) < chk[2], (case["id"], chk, probs)
        elif kind == "keys_in":
            assert all(k in chk[1] for k in probs), (case["id"], probs)
        elif kind == "keys_char":
            assert all(k[chk[1]] == chk[2] for k in probs), (case["id"], probs)
        elif kind == "pos_close":
            s = sum(p for k, p in probs.items() if k[chk[1]] == chk[2])
            assert abs(s - chk[3]) < tol(chk[4]), (case["id"], chk, probs)
        elif kind == "pos_near":
            s = sum(p for k, p in probs.items() if k[chk[1]] == chk[2])
            assert abs(s - chk[3]) <= chk[4], (case["id"], chk, probs)
        elif kind == "total":
            assert abs(sum(probs.values()) - 1.0) < chk[1]
        elif kind == "shots":
            assert abs(sum(probs.values()) - 1.0) < 1e-12 and chk[1] == case["run"]["shots"]
        elif kind == "like_clean":
            assert clean is not None
            assert all(abs(v - clean.get(k, 0.0)) < chk[1] for k, v in probs.items()), (case["id"], probs, clean)
        else:
            raise AssertionError(f"unknown check {kind}")


def reference_draws(amps, draws_at=None, rng_seed=0):
    """Draws on and one ulp above the running sums, uniform draws, 0 and 1,
    and the reference's answer to each: the first kept entry whose running
    sum is >= r, the last kept entry's sum taken as 1.0."""
    p = amps.real * amps.real + amps.imag * amps.imag
    kept = np.nonzero(p > 1e-14)[0]
    ck = np.cumsum(p[kept])                # ascending index order, rounded each step
    ck[-1] = 1.0
    cum = np.cumsum(np.where(p > 1e-14, p, 0.0))
    idx = draws_at if draws_at is not None else np.arange(p.size)
    r = np.concatenate([cum[idx], np.nextafter(cum[idx], np.inf), [0.0, 1.0],
                        np.random.default_rng(rng_seed).random(4096)])
    r = r[r <= 1.0]
    return kept[np.searchsorted(ck, r, side="left")], r
