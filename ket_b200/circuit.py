"""Circuit and Distribution: the host-side mirror of the reference's Circuit API
(src/circuit.ts) over the B200 statevector engine.

A Circuit is an immutable op list built with the reference's builder-method
names; simulation is lazy.  The pure statevector path -- flattenOps,
svFromBitstring and simulatePure (circuit.ts:113-161) -- runs on the GPU
through the C ABI; the read-outs (run, exactProbs, statevector, amplitude,
probability, marginals, expectation) read the device-resident state.  The
final state of a circuit is cached per initial state, so asking for many
amplitudes costs one simulation, not one per call (the reference re-runs the
whole simulation inside every amplitude() call, circuit.ts:1491-1495).

There is no CPU fallback: without the CUDA library or a GPU every simulation
call raises.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from typing import Callable, Dict, Iterable, List, NamedTuple, Optional, Sequence, Tuple, Union

import numpy as np

from . import gates as G
from ._lib import (KET_C128, KET_C64, KetError, OP_BARRIER, OP_CNOT, OP_CONTROLLED, OP_CSRSWAP, OP_CSWAP, OP_IF, OP_MEASURE,
                   OP_RESET, OP_SINGLE, OP_SWAP, OP_TOFFOLI, OP_TWO, OP_UNITARY, RangeError, check, default_ctx,
                   exec_opts, ket_noise, ket_op, lib)

Number = Union[int, float]
Param = Union[int, float, str]

PRUNE = 1e-14  # statevector.ts:277 / complex.ts:24

# Published device noise profiles (DEVICES, circuit.ts:228-245): p1, p2, pMeas.
DEVICES = {
    "aria-1": {"qubits": 25, "nativeGates": ("gpi", "gpi2", "ms", "vz"), "noise": {"p1": 0.0003, "p2": 0.005, "pMeas": 0.004}},
    "forte-1": {"qubits": 36, "nativeGates": ("gpi", "gpi2", "ms", "vz", "zz"),
                "noise": {"p1": 0.0001, "p2": 0.002, "pMeas": 0.002}},
    "harmony": {"qubits": 11, "nativeGates": ("gpi", "gpi2", "ms", "vz"), "noise": {"p1": 0.001, "p2": 0.015, "pMeas": 0.01}},
    "ibm_sherbrooke": {"qubits": 127, "noise": {"p1": 2.4e-4, "p2": 7.4e-3, "pMeas": 1.35e-2}},
    "ibm_brisbane": {"qubits": 127, "noise": {"p1": 2.4e-4, "p2": 7.6e-3, "pMeas": 1.35e-2}},
    "ibm_torino": {"qubits": 133, "noise": {"p1": 2.0e-4, "p2": 3.0e-3, "pMeas": 1.0e-2}},
    "h1-1": {"qubits": 20, "noise": {"p1": 1.8e-5, "p2": 9.7e-4, "pMeas": 2.3e-3}},
    "h2-1": {"qubits": 56, "noise": {"p1": 1.9e-5, "p2": 1.1e-3, "pMeas": 1.0e-3}},
}


# Density-matrix noise profiles (DM_DEVICE_NOISE, density.ts:453-457): p1, p2.
DM_DEVICE_NOISE = {"aria-1": {"p1": 0.0003, "p2": 0.005}, "forte-1": {"p1": 0.0001, "p2": 0.002},
                   "harmony": {"p1": 0.001, "p2": 0.015}}


class DensityMatrix:
    """DensityMatrix (density.ts:274-372) over a device state of 2n qubits
    holding rho[row][col] at index (row << n) | col."""

    def __init__(self, qubits: int, state: "DeviceState"):
        self.qubits = qubits
        self._st = state

    def get(self, row: int, col: int) -> complex:
        """rho[row][col] (density.ts:283-286)."""
        return complex(self._st.amplitudes([(int(row) << self.qubits) | int(col)])[0])

    def probabilities(self) -> Dict[str, float]:
        """Diagonal probabilities, q0-leftmost keys, values > 1e-14 (density.ts:299-307)."""
        d = np.empty(1 << self.qubits, dtype=np.float64)
        check(lib().ket_dm_probs(self._st.h, d.ctypes.data_as(C.POINTER(C.c_double))))
        return {index_to_bitstring(r, self.qubits): float(v) for r, v in enumerate(d) if v > 1e-14}

    def purity(self) -> float:
        """Tr(rho^2) = sum of |rho[r][c]|^2 (density.ts:314-318)."""
        return self._st.norm2()

    def entropy(self) -> float:
        """Von Neumann entropy in bits (density.ts:328-346), from the eigenvalues of
        the dense Hermitian rho (host LAPACK)."""
        dim = 1 << self.qubits
        if dim > 4096:
            raise RangeError(f"entropy(): circuit too large (n={self.qubits}, dim={dim})")
        rho = self._st.amplitudes_dense().reshape(dim, dim)
        lam = np.linalg.eigvalsh(rho)
        return float(-sum(x * math.log2(x) for x in lam if x > 1e-14))

    def blochAngles(self, q: int) -> Dict[str, float]:
        """Bloch angles of qubit q (density.ts:356-372)."""
        out = np.empty(2, dtype=np.float64)
        check(lib().ket_dm_bloch(self._st.h, q, out.ctypes.data_as(C.POINTER(C.c_double))))
        return {"theta": float(out[0]), "phi": float(out[1])}

    def dense(self) -> np.ndarray:
        dim = 1 << self.qubits
        return self._st.amplitudes_dense().reshape(dim, dim)


def resolve_noise(noise):
    """run()'s noise option (circuit.ts:3411-3418): None, a device name, or a
    NoiseParams mapping {p1, p2, pMeas} -> (p1, p2, pMeas), or None."""
    if noise is None:
        return None
    if isinstance(noise, str):
        if noise not in DEVICES:
            raise TypeError(f"Unknown device profile '{noise}'. Known: {', '.join(DEVICES)}")
        noise = DEVICES[noise]["noise"]
    return (float(noise.get("p1") or 0), float(noise.get("p2") or 0), float(noise.get("pMeas") or 0))


class Op(NamedTuple):
    kind: str                 # single cnot swap two controlled toffoli cswap csrswap unitary barrier
    qubits: Tuple[int, ...]   # measure reset if subcircuit parametric
    gate: Optional[tuple] = None
    name: Optional[str] = None
    params: Tuple = ()
    extra: object = None      # creg info / if body / subcircuit body


_KIND_CODE = {"single": OP_SINGLE, "cnot": OP_CNOT, "swap": OP_SWAP, "two": OP_TWO, "controlled": OP_CONTROLLED,
              "toffoli": OP_TOFFOLI, "cswap": OP_CSWAP, "csrswap": OP_CSRSWAP, "unitary": OP_UNITARY,
              "barrier": OP_BARRIER}


def make_prng(seed: Optional[int] = None) -> Callable[[], float]:
    """makePrng (circuit.ts:813-819): xorshift32 (13, 17, 5) on uint32, seed 0 -> 1."""
    if seed is None:
        s = (int(time.time() * 1000) & 0xFFFFFFFF) or 1
    else:
        s = (int(seed) & 0xFFFFFFFF) or 1
    state = [s]

    def rng() -> float:
        x = state[0]
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        state[0] = x
        return x / 4294967296.0

    rng.state = state  # type: ignore[attr-defined]
    return rng


def prng_draws(seed: Optional[int], count: int) -> np.ndarray:
    """`count` successive makePrng(seed) draws, vectorised."""
    rng = make_prng(seed)
    s = rng.state[0]
    out = np.empty(count, dtype=np.float64)
    for i in range(count):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        out[i] = s
    return out / 4294967296.0


def bitstring_to_index(s: str, qubits: int, what: str = "initialState") -> int:
    """svFromBitstring (circuit.ts:136-140): q0 is the leftmost character."""
    if not isinstance(s, str) or len(s) != qubits or not s or any(ch not in "01" for ch in s):
        if what == "initialState":
            raise TypeError(f"initialState '{s}' must be a {qubits}-character binary string")
        raise TypeError(f"bitstring '{s}' must be a {qubits}-character binary string")
    return int(s[::-1], 2)


def index_to_bitstring(idx: int, qubits: int) -> str:
    """Distribution key (circuit.ts:911): idx.toString(2).padStart(n).reverse()."""
    return format(int(idx), "b").zfill(qubits)[::-1]


class Distribution:
    """Measurement result (circuit.ts:879-944)."""

    def __init__(self, qubits: int, shots: int, counts: Dict[int, int], cregs=None, truncated: bool = False):
        self.qubits = qubits
        self.shots = shots
        self.truncated = truncated
        probs, hist = {}, {}
        for idx, count in counts.items():
            prob = count / shots
            probs[index_to_bitstring(idx, qubits)] = prob
            hist[str(idx)] = prob
        self.probs = probs
        self.histogram = hist
        self.cregs = dict(cregs or {})

    @property
    def most(self) -> str:
        best, bp = "", -1.0
        for bs, p in self.probs.items():
            if p > bp:
                best, bp = bs, p
        return best

    @property
    def entropy(self) -> float:
        h = 0.0
        for p in self.probs.values():
            if p > 0:
                h -= p * math.log2(p)
        return h


class _Node:
    """Persistent op list: appending shares the prefix, so building an
    L-gate circuit costs O(L) instead of the reference's O(L^2) copies."""
    __slots__ = ("parent", "op", "length")

    def __init__(self, parent, op):
        self.parent = parent
        self.op = op
        self.length = (parent.length if parent else 0) + 1


def _ops_of(node) -> Tuple[Op, ...]:
    out = []
    while node is not None:
        out.append(node.op)
        node = node.parent
    return tuple(reversed(out))


def _to_complex_matrix(matrix) -> tuple:
    return tuple(tuple(complex(v["re"], v["im"]) if isinstance(v, dict) else complex(v) for v in row)
                 for row in matrix)


class Circuit:
    """Immutable circuit (circuit.ts:1090): every builder returns a new Circuit."""

    def __init__(self, qubits: int, ops: Iterable[Op] = (), cregs: Optional[dict] = None,
                 gates: Optional[dict] = None, _node=None):
        self.qubits = int(qubits)
        if _node is None:
            for op in ops:
                _node = _Node(_node, op)
        self._node = _node
        self._cregs = dict(cregs or {})
        self._gates = dict(gates or {})
        self._ops_cache = None
        self._sv_cache: Dict = {}

    # ------------------------------------------------------------------ op list
    @property
    def ops(self) -> Tuple[Op, ...]:
        if self._ops_cache is None:
            self._ops_cache = _ops_of(self._node)
        return self._ops_cache

    def __len__(self):
        return self._node.length if self._node else 0

    def _with(self, node, cregs=None, gates=None) -> "Circuit":
        return Circuit(self.qubits, cregs=self._cregs if cregs is None else cregs,
                       gates=self._gates if gates is None else gates, _node=node)

    def _add(self, op: Op) -> "Circuit":
        self._check_op(op)
        return self._with(_Node(self._node, op))

    def _check_op(self, op: Op) -> None:
        """#checkOp (circuit.ts:1113-1146)."""
        def q(i):
            if not isinstance(i, (int, np.integer)) or i < 0 or i >= self.qubits:
                raise RangeError(f"qubit index {i} is out of range for a {self.qubits}-qubit circuit")

        def diff(a, b):
            if a == b:
                raise TypeError(f"control and target qubits must differ (got {a})")

        k = op.kind
        if k in ("single", "measure", "reset"):
            q(op.qubits[0])
        elif k in ("cnot", "controlled"):
            q(op.qubits[0]); q(op.qubits[1]); diff(op.qubits[0], op.qubits[1])
        elif k in ("swap", "two"):
            q(op.qubits[0]); q(op.qubits[1])
        elif k in ("toffoli", "cswap", "csrswap"):
            for i in op.qubits:
                q(i)
        elif k in ("barrier", "parametric", "subcircuit"):
            for i in op.qubits:
                q(i)
        elif k == "unitary":
            if len(op.qubits) == 0:
                raise TypeError("unitary: qubits must be non-empty")
            exp = 1 << len(op.qubits)
            if len(op.gate) != exp or any(len(r) != exp for r in op.gate):
                raise TypeError(f"unitary: matrix must be {exp}x{exp} for {len(op.qubits)} qubit(s), got "
                                f"{len(op.gate)}x{len(op.gate[0]) if op.gate else 0}")
            for i in op.qubits:
                q(i)
        elif k == "if":
            for inner in op.extra[2]:
                self._check_op(inner)

    def _single(self, q, gate, name, params=()):
        return self._add(Op("single", (q,), gate, name, tuple(params)))

    def _ctrl(self, c, t, gate, name, params=()):
        return self._add(Op("controlled", (c, t), gate, name, tuple(params)))

    def _param(self, name, params, qubits):
        return self._add(Op("parametric", tuple(qubits), None, name, tuple(params)))

    # ------------------------------------------------------------------ gates (circuit.ts:1152-1421)
    def id(self, q): return self._single(q, G.Id, "id")
    def h(self, q): return self._single(q, G.H, "h")
    def x(self, q): return self._single(q, G.X, "x")
    def y(self, q): return self._single(q, G.Y, "y")
    def z(self, q): return self._single(q, G.Z, "z")
    def s(self, q): return self._single(q, G.S, "s")
    def si(self, q): return self._single(q, G.Si, "si")
    def sdg(self, q): return self._single(q, G.Si, "sdg")
    def t(self, q): return self._single(q, G.T, "t")
    def ti(self, q): return self._single(q, G.Ti, "ti")
    def tdg(self, q): return self._single(q, G.Ti, "tdg")
    def v(self, q): return self._single(q, G.V, "v")
    def vi(self, q): return self._single(q, G.Vi, "vi")
    def srn(self, q): return self._single(q, G.V, "srn")
    def srndg(self, q): return self._single(q, G.Vi, "srndg")
    def r2(self, q): return self._single(q, G.R2, "r2")
    def r4(self, q): return self._single(q, G.R4, "r4")
    def r8(self, q): return self._single(q, G.R8, "r8")

    def rx(self, theta: Param, q: int):
        if isinstance(theta, str): return self._param("rx", [theta], [q])
        return self._single(q, G.Rx(theta), "rx", [theta])

    def ry(self, theta: Param, q: int):
        if isinstance(theta, str): return self._param("ry", [theta], [q])
        return self._single(q, G.Ry(theta), "ry", [theta])

    def rz(self, theta: Param, q: int):
        if isinstance(theta, str): return self._param("rz", [theta], [q])
        return self._single(q, G.Rz(theta), "rz", [theta])

    def vz(self, theta: Param, q: int):
        if isinstance(theta, str): return self._param("vz", [theta], [q])
        return self._single(q, G.Rz(theta), "vz", [theta])

    def u1(self, lam: Param, q: int):
        if isinstance(lam, str): return self._param("u1", [lam], [q])
        return self._single(q, G.U1(lam), "u1", [lam])

    def p(self, lam: Param, q: int):
        if isinstance(lam, str): return self._param("p", [lam], [q])
        return self._single(q, G.U1(lam), "p", [lam])

    def u2(self, phi: Param, lam: Param, q: int):
        if isinstance(phi, str) or isinstance(lam, str): return self._param("u2", [phi, lam], [q])
        return self._single(q, G.U2(phi, lam), "u2", [phi, lam])

    def u3(self, theta: Param, phi: Param, lam: Param, q: int):
        if any(isinstance(v, str) for v in (theta, phi, lam)): return self._param("u3", [theta, phi, lam], [q])
        return self._single(q, G.U3(theta, phi, lam), "u3", [theta, phi, lam])

    def cnot(self, control: int, target: int):
        return self._add(Op("cnot", (control, target), None, "cnot"))

    def cx(self, control: int, target: int):
        return self.cnot(control, target)

    def swap(self, a: int, b: int):
        return self._add(Op("swap", (a, b), None, "swap"))

    def _two(self, a, b, gate, name, params=()):
        return self._add(Op("two", (a, b), gate, name, tuple(params)))

    def xx(self, theta: Param, a: int, b: int):
        if isinstance(theta, str): return self._param("xx", [theta], [a, b])
        return self._two(a, b, G.Xx(theta), "xx", [theta])

    def yy(self, theta: Param, a: int, b: int):
        if isinstance(theta, str): return self._param("yy", [theta], [a, b])
        return self._two(a, b, G.Yy(theta), "yy", [theta])

    def zz(self, theta: Param, a: int, b: int):
        if isinstance(theta, str): return self._param("zz", [theta], [a, b])
        return self._two(a, b, G.Zz(theta), "zz", [theta])

    def xy(self, theta: Param, a: int, b: int):
        if isinstance(theta, str): return self._param("xy", [theta], [a, b])
        return self._two(a, b, G.Xy(theta), "xy", [theta])

    def iswap(self, a, b): return self._two(a, b, G.ISwap, "iswap")
    def srswap(self, a, b): return self._two(a, b, G.SrSwap, "srswap")

    def ms(self, phi0: Param, phi1: Param, a: int, b: int):
        if isinstance(phi0, str) or isinstance(phi1, str): return self._param("ms", [phi0, phi1], [a, b])
        return self._two(a, b, G.Ms(phi0, phi1), "ms", [phi0, phi1])

    def cy(self, c, t): return self._ctrl(c, t, G.Y, "cy")
    def cz(self, c, t): return self._ctrl(c, t, G.Z, "cz")
    def ch(self, c, t): return self._ctrl(c, t, G.H, "ch")
    def cr2(self, c, t): return self._ctrl(c, t, G.R2, "cr2")
    def cr4(self, c, t): return self._ctrl(c, t, G.R4, "cr4")
    def cr8(self, c, t): return self._ctrl(c, t, G.R8, "cr8")
    def cs(self, c, t): return self._ctrl(c, t, G.S, "cs")
    def ct(self, c, t): return self._ctrl(c, t, G.T, "ct")
    def csdg(self, c, t): return self._ctrl(c, t, G.Si, "csdg")
    def ctdg(self, c, t): return self._ctrl(c, t, G.Ti, "ctdg")
    def csrn(self, c, t): return self._ctrl(c, t, G.V, "csrn")

    def crx(self, theta: Param, c: int, t: int):
        if isinstance(theta, str): return self._param("crx", [theta], [c, t])
        return self._ctrl(c, t, G.Rx(theta), "crx", [theta])

    def cry(self, theta: Param, c: int, t: int):
        if isinstance(theta, str): return self._param("cry", [theta], [c, t])
        return self._ctrl(c, t, G.Ry(theta), "cry", [theta])

    def crz(self, theta: Param, c: int, t: int):
        if isinstance(theta, str): return self._param("crz", [theta], [c, t])
        return self._ctrl(c, t, G.Rz(theta), "crz", [theta])

    def cu1(self, lam: Param, c: int, t: int):
        if isinstance(lam, str): return self._param("cu1", [lam], [c, t])
        return self._ctrl(c, t, G.U1(lam), "cu1", [lam])

    def cu2(self, phi: Param, lam: Param, c: int, t: int):
        if isinstance(phi, str) or isinstance(lam, str): return self._param("cu2", [phi, lam], [c, t])
        return self._ctrl(c, t, G.U2(phi, lam), "cu2", [phi, lam])

    def cu3(self, theta: Param, phi: Param, lam: Param, c: int, t: int):
        if any(isinstance(v, str) for v in (theta, phi, lam)): return self._param("cu3", [theta, phi, lam], [c, t])
        return self._ctrl(c, t, G.U3(theta, phi, lam), "cu3", [theta, phi, lam])

    def gpi(self, phi: Param, q: int):
        if isinstance(phi, str): return self._param("gpi", [phi], [q])
        return self._single(q, G.Gpi(phi), "gpi", [phi])

    def gpi2(self, phi: Param, q: int):
        if isinstance(phi, str): return self._param("gpi2", [phi], [q])
        return self._single(q, G.Gpi2(phi), "gpi2", [phi])

    def ccx(self, c1: int, c2: int, target: int):
        return self._add(Op("toffoli", (c1, c2, target), None, "ccx"))

    def cswap(self, control: int, a: int, b: int):
        return self._add(Op("cswap", (control, a, b), None, "cswap"))

    def csrswap(self, control: int, a: int, b: int):
        return self._add(Op("csrswap", (control, a, b), None, "csrswap"))

    def barrier(self, *qubits: int):
        qs = tuple(qubits) if qubits else tuple(range(self.qubits))
        return self._add(Op("barrier", qs, None, "barrier"))

    def unitary(self, matrix, *qubits: int):
        return self._add(Op("unitary", tuple(qubits), _to_complex_matrix(matrix), "unitary"))

    # ------------------------------------------------------------------ classical ops (recorded only)
    def creg(self, name: str, size: int):
        cr = dict(self._cregs)
        cr[name] = size
        return self._with(self._node, cregs=cr)

    def measure(self, q: int, creg: str, bit: int):
        # the reference's measure() does not check q (circuit.ts:1607-1615):
        # a qubit outside the state reads 0
        cr = dict(self._cregs)
        cr[creg] = max(cr.get(creg, 0), bit + 1)
        return self._with(_Node(self._node, Op("measure", (q,), None, "measure", (), (creg, bit))), cregs=cr)

    def reset(self, q: int, value: int = 0):
        r = self._add(Op("reset", (q,), None, "reset"))
        return r.x(q) if value == 1 else r

    def if_(self, creg: str, value: int, build: Callable[["Circuit"], "Circuit"]):
        inner = build(Circuit(self.qubits, gates=self._gates))
        return self._add(Op("if", (), None, "if", (), (creg, value, inner.ops)))

    # ------------------------------------------------------------------ named gates (circuit.ts:1659-1697)
    def defineGate(self, name: str, sub: "Circuit"):
        if any(op.kind in ("measure", "reset", "if") for op in sub.ops):
            raise TypeError(f"Gate '{name}' contains classical ops (measure/reset/if), which are not supported "
                            "inside named gates")
        gs = dict(self._gates)
        gs[name] = sub
        return self._with(self._node, gates=gs)

    def gate(self, name: str, *qubits: int):
        sub = self._gates.get(name)
        if sub is None:
            raise TypeError(f"Unknown gate '{name}'. Register it first with .defineGate(name, subcircuit).")
        if len(qubits) != sub.qubits:
            raise TypeError(f"Gate '{name}' expects {sub.qubits} qubit(s), got {len(qubits)}")
        return self._add(Op("subcircuit", tuple(qubits), None, name, (), sub.ops))

    def decompose(self):
        return Circuit(self.qubits, flatten_ops(self.ops), self._cregs, self._gates)

    def append(self, other: "Circuit"):
        if other.qubits != self.qubits:
            raise TypeError(f"append: qubit count mismatch ({self.qubits} vs {other.qubits})")
        node = self._node
        for op in other.ops:
            node = _Node(node, op)
        return self._with(node)

    # ------------------------------------------------------------------ parameters (circuit.ts:1730-1763)
    @property
    def params(self) -> List[str]:
        return sorted(_collect_params(self.ops))

    def bind(self, values: Dict[str, float]) -> "Circuit":
        def resolve(p):
            if not isinstance(p, str):
                return p
            if p in values:
                return values[p]
            raise TypeError(f"bind: unbound parameter '{p}'. Provide a value for it in the bind() call.")

        def rebuild(ops):
            out = []
            for op in ops:
                if op.kind == "parametric":
                    out.append(resolve_parametric(op.name, [resolve(p) for p in op.params], op.qubits))
                elif op.kind == "if":
                    out.append(op._replace(extra=(op.extra[0], op.extra[1], tuple(rebuild(op.extra[2])))))
                else:
                    out.append(op)
            return out

        return Circuit(self.qubits, rebuild(self.ops), self._cregs, self._gates)

    # ------------------------------------------------------------------ simulation
    def _require_pure(self, what: str):
        if any(op.kind in ("measure", "reset", "if") for op in self.ops):
            raise TypeError(f"{what} requires a pure circuit — remove measure/reset/if ops")

    def _state(self, initialState: Optional[str] = None, precision: int = KET_C128, fusion: int = -1,
               prune: bool = True) -> "DeviceState":
        key = (initialState, precision, fusion, prune)
        st = self._sv_cache.get(key)
        if st is None:
            init = bitstring_to_index(initialState, self.qubits) if initialState is not None else 0
            flat = flatten_ops(self.ops)  # throws on unbound parameters, like the reference
            st = DeviceState(self.qubits, precision)
            st.set_basis(init)
            st.apply(flat, fusion=fusion, prune=prune)
            self._sv_cache.clear()  # hold one device state per circuit
            self._sv_cache[key] = st
        return st

    def statevector(self, initialState: Optional[str] = None) -> Dict[int, complex]:
        """statevector() (circuit.ts:1431-1441): non-zero amplitudes keyed by index."""
        self._require_pure("statevector()")
        unbound = _collect_params(self.ops)
        if unbound:
            raise TypeError("statevector() requires bound parameters. Call bind({ "
                            + ", ".join(f"{p}: value" for p in unbound) + " }) first.")
        a = self._state(initialState).amplitudes_dense()
        nz = np.nonzero(a)[0]
        return {int(i): complex(a[i]) for i in nz}

    def compile_kernels(self, precision: int = KET_C128, prune: bool = True) -> int:
        """Compile, on all host cores and ahead of the first run, the pass
        kernels this circuit's plan uses (ket_jit_compile; no GPU needed), so
        that runs under the default policy use them at any qubit count.
        Returns the number of distinct kernels.  No counterpart in the
        reference."""
        self._require_pure("compile_kernels()")
        arr, m, k = ops_to_abi(flatten_ops(self.ops))
        mv = np.ascontiguousarray(m).view(np.float64)
        o = exec_opts(-1, prune)
        kernels = C.c_int64()
        log = C.create_string_buffer(1 << 14)
        rc = lib().ket_jit_compile(self.qubits, precision, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                                   C.byref(o), C.byref(kernels), log, len(log))
        if rc:
            raise KetError(log.value.decode(errors="replace") or lib().ket_last_error().decode(), rc)
        return int(kernels.value)

    def statevector_array(self, initialState: Optional[str] = None, precision: int = KET_C128) -> np.ndarray:
        """Dense complex128 array of all 2^n amplitudes (index bit q = qubit q)."""
        self._require_pure("statevector()")
        return self._state(initialState, precision).amplitudes_dense()

    def amplitude(self, bitstring: str) -> complex:
        """amplitude() (circuit.ts:1491-1495)."""
        idx = bitstring_to_index(bitstring, self.qubits, what="bitstring")
        self._require_pure("statevector()")
        return complex(self._state().amplitudes([idx])[0])

    def amplitudes(self, indices: Sequence[int], initialState: Optional[str] = None) -> np.ndarray:
        """Many amplitudes from one simulation (indices are integers, bit q = qubit q)."""
        self._require_pure("statevector()")
        return self._state(initialState).amplitudes(indices)

    def probability(self, bitstring: str) -> float:
        a = self.amplitude(bitstring)
        return a.real * a.real + a.imag * a.imag

    def marginals(self, initialState: Optional[str] = None) -> List[float]:
        """marginals() (circuit.ts:1508-1518): P(qubit q = 1) for each q."""
        self._require_pure("statevector()")
        return list(self._state(initialState).marginals())

    def dm(self, noise=None) -> DensityMatrix:
        """dm() (circuit.ts:4562-4579, runDM density.ts:475-588): the exact density
        matrix from |0..0>, with depolarizing noise {p1, p2} or a DM_DEVICE_NOISE name."""
        if any(op.kind in ("measure", "reset", "if") for op in self.ops):
            raise TypeError("dm() requires a pure circuit — remove measure/reset/if ops")
        if isinstance(noise, str):
            if noise not in DM_DEVICE_NOISE:
                raise TypeError(f"Unknown device profile '{noise}'. Known: {', '.join(DM_DEVICE_NOISE)}")
            noise = DM_DEVICE_NOISE[noise]
        p1 = float((noise or {}).get("p1") or 0)
        p2 = float((noise or {}).get("p2") or 0)
        arr, m, k = ops_to_abi(flatten_ops(self.ops))
        st = DeviceState(2 * self.qubits)
        mv = np.ascontiguousarray(m).view(np.float64)
        check(lib().ket_dm_run(st.h, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, p1, p2))
        return DensityMatrix(self.qubits, st)

    def blochAngles(self, q: int, initialState: Optional[str] = None) -> Dict[str, float]:
        """blochAngles(q) (circuit.ts:4102-4129): {theta, phi} of qubit q's
        reduced density matrix."""
        self._require_pure("blochAngles()")
        out = np.empty(6, dtype=np.float64)
        check(lib().ket_bloch(self._state(initialState).h, q, out.ctypes.data_as(C.POINTER(C.c_double))))
        return {"theta": float(out[4]), "phi": float(out[5])}

    def circuitMatrix(self) -> np.ndarray:
        """circuitMatrix() (circuit.ts:1462-1485): the 2^n x 2^n matrix,
        matrix[row][col], rows and columns with q0 as the most significant bit.
        TypeError for measure/reset/if, RangeError above 12 qubits."""
        if any(op.kind in ("measure", "reset", "if") for op in self.ops):
            raise TypeError("circuitMatrix() requires a pure circuit — remove measure/reset/if ops")
        n = self.qubits
        if n > 12:
            raise RangeError(f"circuitMatrix(): circuit too large ({n} qubits = {1 << n}×{1 << n} matrix)")
        arr, m, k = ops_to_abi(flatten_ops(self.ops))
        out = np.empty((1 << n, 1 << n), dtype=np.complex128)
        mv = np.ascontiguousarray(m).view(np.float64)
        check(lib().ket_circuit_matrix(default_ctx(), n, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                                       None, out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def marginal_dist(self, qubits: Sequence[int], initialState: Optional[str] = None) -> np.ndarray:
        """Joint distribution of `qubits` (bin bit k = qubits[k])."""
        self._require_pure("statevector()")
        return self._state(initialState).marginal_dist(qubits)

    def exactProbs(self, initialState: Optional[str] = None) -> Dict[str, float]:
        """exactProbs() (circuit.ts:3700-3711): q0-leftmost key -> p for p > 1e-14."""
        if any(op.kind in ("measure", "reset", "if") for op in self.ops):
            raise TypeError("exactProbs() requires a pure circuit — no measure, reset, or if ops")
        idx, p = self._state(initialState).probs_sparse()
        n = self.qubits
        return {index_to_bitstring(i, n): float(v) for i, v in zip(idx.tolist(), p.tolist())}

    def exactProbsArray(self, initialState: Optional[str] = None) -> np.ndarray:
        """exactProbs() as a dense array (p <= 1e-14 reported as 0) for states too
        large for a keyed record."""
        self._require_pure("exactProbs()")
        return self._state(initialState).probs_dense()

    def expectation(self, pauli: str) -> float:
        """expectation() (circuit.ts:3728-3753): pauli[q] acts on qubit q."""
        n = self.qubits
        pauli = pauli.upper()
        if len(pauli) != n:
            raise TypeError(f"pauli '{pauli}' length must equal qubits ({n})")
        if any(ch not in "IXYZ" for ch in pauli):
            raise TypeError("pauli must contain only I, X, Y, Z")
        if not any(ch in "XYZ" for ch in pauli):
            return 1.0
        self._require_pure("exactProbs()")
        return self._state().expect_pauli(pauli)

    def run(self, shots: int = 1024, seed: Optional[int] = None, noise=None,
            initialState: Optional[str] = None) -> Distribution:
        """run() pure fast path (circuit.ts:3406-3453): simulate once, sample shots
        by a lower-bound search of the ascending-index FP64 CDF."""
        nz = resolve_noise(noise)
        if initialState is not None:
            bitstring_to_index(initialState, self.qubits)
        if nz is not None or any(op.kind in ("measure", "reset", "if") for op in self.ops):
            return self._run_pershot(shots, seed, nz, initialState)
        rng_draws = prng_draws(seed, shots)
        idx = self._state(initialState).sample(rng_draws)
        counts: Dict[int, int] = {}
        for i in idx.tolist():
            counts[i] = counts.get(i, 0) + 1
        return Distribution(self.qubits, shots, counts, {name: [0.0] * size for name, size in self._cregs.items()})

    def run_shots(self, shots: int = 1024, seed: Optional[int] = None, noise=None,
                  initialState: Optional[str] = None):
        """The per-shot records behind run()'s per-shot path (circuit.ts:3455-3481):
        (sampled index per shot, classical bits [shots, bits], {register: (first
        bit, size)}, xorshift32 state after the last draw).  One device
        trajectory per shot through ket_run_shots; all shots draw one makePrng
        stream in the reference's order."""
        nz = resolve_noise(noise)
        init = bitstring_to_index(initialState, self.qubits) if initialState is not None else 0
        arr, m, k, ncbits, layout = shots_to_abi(self.ops, self._cregs)
        st = DeviceState(self.qubits)
        noise_s = ket_noise(*(nz if nz is not None else (0.0, 0.0, 0.0)))
        state = C.c_uint32(make_prng(seed).state[0])
        out_idx = np.zeros(max(shots, 1), dtype=np.uint64)
        out_bits = np.zeros(max(shots * ncbits, 1), dtype=np.uint8)
        mv = np.ascontiguousarray(m).view(np.float64)
        check(lib().ket_run_shots(st.h, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                                  C.byref(noise_s) if nz is not None else None, init, shots, C.byref(state), ncbits,
                                  out_idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                  out_bits.ctypes.data_as(C.POINTER(C.c_uint8))))
        bits = out_bits[: shots * ncbits].reshape(shots, ncbits)
        return out_idx[:shots], bits, layout, int(state.value)

    def _run_pershot(self, shots: int, seed: Optional[int], nz, initialState: Optional[str]) -> Distribution:
        idx, bits, layout, _ = self.run_shots(shots, seed, None if nz is None else
                                              {"p1": nz[0], "p2": nz[1], "pMeas": nz[2]}, initialState)
        counts: Dict[int, int] = {}
        for i in idx.tolist():
            counts[i] = counts.get(i, 0) + 1
        cregs = {name: [float(bits[:, off + j].sum()) / shots if shots else 0.0 for j in range(size)]
                 for name, (off, size) in layout.items()}
        return Distribution(self.qubits, shots, counts, cregs)

    # ------------------------------------------------------------------ JSON (circuit.ts:3768-3806)
    def toJSON(self) -> dict:
        """Circuit.toJSON: {ket: 1, qubits, cregs, gates, ops}, gates by meta."""
        from .circuit_json import to_json
        return to_json(self)

    @staticmethod
    def fromJSON(j) -> "Circuit":
        """Circuit.fromJSON: a CircuitJSON dict or its JSON text."""
        from .circuit_json import from_json
        return from_json(j)

    # ------------------------------------------------------------------ lowering to the C ABI
    def to_abi(self):
        return ops_to_abi(flatten_ops(self.ops))


def _collect_params(ops) -> set:
    names = set()
    for op in ops:
        if op.kind == "parametric":
            for p in op.params:
                if isinstance(p, str):
                    names.add(p)
        elif op.kind == "if":
            names |= _collect_params(op.extra[2])
    return names


def resolve_parametric(name: str, ps, qubits) -> Op:
    """resolveParametric (circuit.ts:1047-1073)."""
    q = tuple(qubits)
    single = {"rx": G.Rx, "ry": G.Ry, "rz": G.Rz, "vz": G.Rz, "u1": G.U1, "p": G.U1, "gpi": G.Gpi, "gpi2": G.Gpi2}
    if name in single:
        return Op("single", (q[0],), single[name](ps[0]), name, tuple(ps))
    if name == "u2":
        return Op("single", (q[0],), G.U2(ps[0], ps[1]), name, tuple(ps))
    if name == "u3":
        return Op("single", (q[0],), G.U3(ps[0], ps[1], ps[2]), name, tuple(ps))
    two = {"xx": G.Xx, "yy": G.Yy, "zz": G.Zz, "xy": G.Xy}
    if name in two:
        return Op("two", (q[0], q[1]), two[name](ps[0]), name, tuple(ps))
    if name == "ms":
        return Op("two", (q[0], q[1]), G.Ms(ps[0], ps[1]), name, tuple(ps))
    ctrl = {"crx": G.Rx, "cry": G.Ry, "crz": G.Rz, "cu1": G.U1}
    if name in ctrl:
        return Op("controlled", (q[0], q[1]), ctrl[name](ps[0]), name, tuple(ps))
    if name == "cu2":
        return Op("controlled", (q[0], q[1]), G.U2(ps[0], ps[1]), name, tuple(ps))
    if name == "cu3":
        return Op("controlled", (q[0], q[1]), G.U3(ps[0], ps[1], ps[2]), name, tuple(ps))
    raise TypeError(f"bind: unknown parametric gate '{name}'")


def flatten_ops(ops) -> Tuple[Op, ...]:
    """flattenOps (circuit.ts:113-133): throws on unbound parameters, inlines
    named sub-circuits with their qubits remapped."""
    has_sub = False
    for op in ops:
        if op.kind == "parametric":
            names = ", ".join(sorted(_collect_params(ops)))
            raise TypeError(f"Circuit has unbound parameters: [{names}]. Call bind({{ {names} }}) first.")
        if op.kind == "subcircuit":
            has_sub = True
    if not has_sub:
        return tuple(ops)
    out = []
    for op in ops:
        if op.kind == "subcircuit":
            qmap = op.qubits
            out.extend(flatten_ops([_remap(inner, qmap) for inner in op.extra]))
        else:
            out.append(op)
    return tuple(out)


def _remap(op: Op, qmap) -> Op:
    if op.kind in ("measure", "reset", "if", "parametric"):
        return op
    return op._replace(qubits=tuple(qmap[i] for i in op.qubits))


def _fill_gate(o, op: Op, mats: List[complex]):
    o.kind = _KIND_CODE[op.kind]
    qs = op.qubits
    if len(qs) > 10:
        if op.kind == "barrier":
            qs = qs[:1]
        else:
            raise TypeError("op with more than 10 qubits is not supported")
    o.nq = len(qs)
    for j, qq in enumerate(qs):
        o.q[j] = int(qq)
    if op.gate is not None:
        o.mat = len(mats)
        for row in op.gate:
            mats.extend(row)
    else:
        o.mat = -1


def ops_to_abi(ops):
    """Lower flat ops to (ket_op array, matrix buffer, count)."""
    arr = (ket_op * max(1, len(ops)))()
    mats: List[complex] = []
    k = 0
    for op in ops:
        if op.kind in ("measure", "reset", "if"):
            raise TypeError("pure path got a measure/reset/if op")
        _fill_gate(arr[k], op, mats)
        k += 1
    m = np.asarray(mats, dtype=np.complex128) if mats else np.zeros(1, dtype=np.complex128)
    return arr, m, k


def shots_to_abi(ops, cregs: Dict[str, int]):
    """Lower ops with measure / reset / if to ket_run_shots' encoding:
    (ket_op array, matrix buffer, count, classical bits, {register: (first
    bit, size)}).  Registers take consecutive bits in declaration order (the
    Map order of the reference's #cregs).  An if-body follows its if op;
    bodies are flattened as applyOps does when it runs them.  A measure into a
    register the circuit does not hold -- one declared only inside an if body,
    whose builder circuit the reference discards -- is not recorded."""
    layout, nb = {}, 0
    for name, size in cregs.items():
        layout[name] = (nb, int(size))
        nb += int(size)
    entries = []

    def lower(seq):
        for op in flatten_ops(seq):
            if op.kind == "measure":
                creg, bit = op.extra
                reg = layout.get(creg)
                cb = reg[0] + bit if reg is not None and 0 <= bit < reg[1] else -1
                entries.append((OP_MEASURE, (int(op.qubits[0]), cb)))
            elif op.kind == "reset":
                entries.append((OP_RESET, (int(op.qubits[0]),)))
            elif op.kind == "if":
                creg, value, body = op.extra
                first, size = layout.get(creg, (0, 0))
                if size > 31:
                    raise NotImplementedError("if() on a register of more than 31 bits")
                v = int(value) if float(value).is_integer() and -(1 << 31) <= value < (1 << 31) else -1
                pos = len(entries)
                entries.append(None)
                lower(body)
                entries[pos] = (OP_IF, (first, size, v, len(entries) - pos - 1))
            else:
                entries.append(op)

    lower(ops)
    arr = (ket_op * max(1, len(entries)))()
    mats: List[complex] = []
    for i, e in enumerate(entries):
        if isinstance(e, Op):
            _fill_gate(arr[i], e, mats)
        else:
            code, qs = e
            arr[i].kind = code
            arr[i].nq = len(qs)
            for j, v in enumerate(qs):
                arr[i].q[j] = v
            arr[i].mat = -1
    m = np.asarray(mats, dtype=np.complex128) if mats else np.zeros(1, dtype=np.complex128)
    return arr, m, len(entries), nb, layout


class DeviceState:
    """A device-resident dense state owned through the C ABI."""

    def __init__(self, n: int, precision: int = KET_C128):
        self.n = n
        self.precision = precision
        self.h = C.c_void_p()
        check(lib().ket_state_alloc(default_ctx(), n, precision, C.byref(self.h)))

    def __del__(self):
        try:
            if self.h:
                lib().ket_state_free(self.h)
        except Exception:
            pass

    def set_basis(self, idx: int):
        check(lib().ket_state_set_basis(self.h, int(idx)))

    def set_amplitudes(self, a: np.ndarray, offset: int = 0):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        check(lib().ket_state_set_amplitudes(self.h, offset, a.size, a.view(np.float64).ctypes.data_as(
            C.POINTER(C.c_double))))

    def apply(self, ops, fusion: int = -1, prune: bool = True, specialize: int = 0):
        arr, m, k = ops_to_abi(ops)
        mv = np.ascontiguousarray(m).view(np.float64)
        o = exec_opts(fusion, prune, specialize)
        check(lib().ket_apply_ops(self.h, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, C.byref(o)))

    def apply_abi(self, arr, m, k, fusion: int = -1, prune: bool = True, specialize: int = 0, reg_bits: int = 0,
                  stage: int = 0):
        """specialize: 0 automatic, 1 run-time compiled pass kernels (compiled
        first where missing), -1 the interpreter only.  reg_bits: register
        bits of the compiled kernels' programs (0 automatic, 4 or 5).  stage:
        the compiled kernels' tile loads (1 TMA-staged, -1 into registers, 0
        automatic)."""
        mv = np.ascontiguousarray(m).view(np.float64)
        o = exec_opts(fusion, prune, specialize, reg_bits, stage)
        check(lib().ket_apply_ops(self.h, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, C.byref(o)))

    def amplitudes_dense(self) -> np.ndarray:
        N = 1 << self.n
        out = np.empty(N, dtype=np.complex128)
        check(lib().ket_state_get_amplitudes(self.h, 0, N, out.view(np.float64).ctypes.data_as(
            C.POINTER(C.c_double))))
        return out

    def amplitudes(self, indices) -> np.ndarray:
        idx = np.ascontiguousarray(indices, dtype=np.uint64)
        out = np.empty(max(idx.size, 1), dtype=np.complex128)
        check(lib().ket_amplitudes(self.h, idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size,
                                   out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))))
        return out[: idx.size]

    def probs_dense(self, thr: float = PRUNE) -> np.ndarray:
        out = np.empty(1 << self.n, dtype=np.float64)
        check(lib().ket_probs_dense(self.h, thr, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def probs_sparse(self, thr: float = PRUNE):
        cnt = C.c_uint64()
        check(lib().ket_probs_sparse(self.h, thr, None, None, 0, C.byref(cnt)))
        n = cnt.value
        idx = np.empty(max(n, 1), dtype=np.uint64)
        p = np.empty(max(n, 1), dtype=np.float64)
        check(lib().ket_probs_sparse(self.h, thr, idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                     p.ctypes.data_as(C.POINTER(C.c_double)), n, C.byref(cnt)))
        return idx[:n], p[:n]

    def marginals(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(lib().ket_marginals(self.h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def marginal_dist(self, qubits) -> np.ndarray:
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        out = np.empty(1 << q.size, dtype=np.float64)
        check(lib().ket_marginal_dist(self.h, q.ctypes.data_as(C.POINTER(C.c_int)), q.size,
                                      out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def norm2(self) -> float:
        out = C.c_double()
        check(lib().ket_norm2(self.h, C.byref(out)))
        return out.value

    def compare(self, other: "DeviceState"):
        """(<self|other>, max_i |self_i - other_i|), accumulated in FP64 on the GPU."""
        ov = (C.c_double * 2)()
        mx = C.c_double()
        check(lib().ket_state_compare(self.h, other.h, ov, C.byref(mx)))
        return complex(ov[0], ov[1]), mx.value

    def sample(self, r: np.ndarray, thr: float = PRUNE) -> np.ndarray:
        r = np.ascontiguousarray(r, dtype=np.float64)
        out = np.empty(max(r.size, 1), dtype=np.uint64)
        check(lib().ket_sample(self.h, r.ctypes.data_as(C.POINTER(C.c_double)), r.size, thr,
                               out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out[: r.size]

    def expect_pauli(self, pauli: str) -> float:
        out = C.c_double()
        check(lib().ket_expect_pauli(self.h, pauli.encode(), C.byref(out)))
        return out.value

    def expect_pauli_sum(self, terms) -> float:
        coeffs = np.ascontiguousarray([t[0] for t in terms] or [0.0], dtype=np.float64)
        ops = "".join(t[1] for t in terms).encode()
        out = C.c_double()
        check(lib().ket_expect_pauli_sum(self.h, len(terms), coeffs.ctypes.data_as(C.POINTER(C.c_double)), ops,
                                         C.byref(out)))
        return out.value
