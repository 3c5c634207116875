"""ctypes wrapper for the CPU oracle (oracle/ket_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker for the GPU engine.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
The product package (ket_b200) never imports it and has no CPU fallback.

The oracle restates the reference TypeScript library (dmvjs/ket) file by file;
ket_oracle.cpp's header lists the file:line ranges it follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libket_oracle.so")

SPARSE = 0        # the reference's pruning sparse map
DENSE = 1         # dense FP64, no pruning
DENSE_PRUNE = 2   # dense FP64 with the reference's |a|^2 < 1e-14 flush

ANS_REAL_AMPLITUDES = 0
ANS_EFFICIENT_SU2 = 1
ANS_HEA_LADDER = 2

KIND_NAMES = ["single", "cnot", "swap", "two", "controlled", "toffoli", "cswap", "csrswap", "unitary", "barrier"]

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "ket_oracle.cpp"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = C.CDLL(_LIB_PATH)
    vp, i32, u32, u64, dbl = C.c_void_p, C.c_int, C.c_uint32, C.c_uint64, C.c_double
    P = C.POINTER
    sig = {
        "orc_last_error": (C.c_char_p, []),
        "orc_circuit_new": (vp, [i32]),
        "orc_circuit_free": (None, [vp]),
        "orc_circuit_copy": (vp, [vp]),
        "orc_circuit_nops": (i32, [vp]),
        "orc_circuit_qubits": (i32, [vp]),
        "orc_add": (i32, [vp, C.c_char_p, P(i32), i32, P(dbl), i32]),
        "orc_add_unitary": (i32, [vp, P(i32), i32, P(dbl)]),
        "orc_op_info": (i32, [vp, i32, P(i32), P(i32), P(i32), P(dbl), i32]),
        "orc_simulate": (vp, [vp, u64, i32]),
        "orc_state_free": (None, [vp]),
        "orc_state_nnz": (u64, [vp]),
        "orc_state_get": (None, [vp, u64, P(dbl)]),
        "orc_state_dense": (None, [vp, P(dbl)]),
        "orc_state_prune_stats": (None, [vp, P(u64), P(dbl)]),
        "orc_exact_probs": (u64, [vp, P(u64), P(dbl), u64]),
        "orc_run": (None, [vp, i32, u32, P(u64)]),
        "orc_marginals": (None, [vp, P(dbl)]),
        "orc_expectation": (dbl, [vp, C.c_char_p, u64, i32]),
        "orc_vqe": (dbl, [vp, i32, P(dbl), C.c_char_p, i32]),
        "orc_ansatz_params": (i32, [i32, i32, i32]),
        "orc_ansatz": (vp, [i32, i32, i32, P(dbl)]),
        "orc_gradient": (None, [i32, i32, i32, P(dbl), i32, P(dbl), C.c_char_p, i32, P(dbl)]),
        "orc_minimize": (i32, [i32, i32, i32, P(dbl), i32, P(dbl), C.c_char_p, dbl, i32, dbl, i32, P(dbl), P(i32)]),
        "orc_qft": (vp, [i32]),
        "orc_iqft": (vp, [i32]),
        "orc_qaoa": (vp, [i32, P(i32), i32, P(dbl), P(dbl), i32]),
        "orc_maxcut_hamiltonian": (i32, [i32, P(i32), i32, P(dbl), C.c_char_p]),
        "orc_brickwork": (vp, [i32, i32, u32, i32, P(u32)]),
        "orc_regular3": (i32, [i32, P(u32), P(i32)]),
        "orc_prng_next": (u32, [P(u32)]),
        "orc_time_ops": (u64, [vp, u64, i32, i32, i32, P(dbl)]),
        "orc_circuit_matrix": (None, [vp, P(dbl)]),
        "orc_dm_run": (vp, [vp, dbl, dbl]),
        "orc_dm_free": (None, [vp]),
        "orc_dm_nnz": (u64, [vp]),
        "orc_dm_dense": (None, [vp, i32, P(dbl)]),
        "orc_dm_purity": (dbl, [vp]),
        "orc_dm_entropy": (dbl, [vp, i32]),
        "orc_dm_bloch": (None, [vp, i32, i32, P(dbl)]),
        "orc_bloch": (None, [vp, i32, P(dbl)]),
        "orc_add_measure": (i32, [vp, i32, i32]),
        "orc_add_reset": (i32, [vp, i32]),
        "orc_add_if": (i32, [vp, i32, i32, i32, vp]),
        "orc_run_pershot": (u32, [vp, u64, i32, u32, dbl, dbl, dbl, i32, P(u64), P(C.c_uint8)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class OracleError(Exception):
    pass


class OracleRangeError(OracleError):
    """Mirrors the reference's RangeError (qubit out of range)."""


class OracleTypeError(OracleError):
    """Mirrors the reference's TypeError (control == target, bad shape, unknown gate)."""


class OCircuit:
    """Oracle circuit: an op list built by the reference's builder-method names."""

    def __init__(self, n: int = 0, handle=None):
        self._L = lib()
        self.h_ = handle if handle is not None else self._L.orc_circuit_new(n)

    def __del__(self):
        try:
            self._L.orc_circuit_free(self.h_)
        except Exception:
            pass

    @property
    def qubits(self) -> int:
        return self._L.orc_circuit_qubits(self.h_)

    def __len__(self):
        return self._L.orc_circuit_nops(self.h_)

    def copy(self) -> "OCircuit":
        return OCircuit(handle=self._L.orc_circuit_copy(self.h_))

    def add(self, name: str, qubits, params=()) -> "OCircuit":
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        p = np.ascontiguousarray(params, dtype=np.float64)
        if p.size == 0:
            p = np.zeros(1)
        rc = self._L.orc_add(self.h_, name.encode(), _ip(q), int(q.size), _dp(p), len(params))
        self._raise(rc)
        return self

    def unitary(self, matrix, qubits) -> "OCircuit":
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128)).view(np.float64)
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        rc = self._L.orc_add_unitary(self.h_, _ip(q), int(q.size), _dp(np.ascontiguousarray(m)))
        self._raise(rc)
        return self

    def _raise(self, rc):
        if rc == 1:
            raise OracleRangeError(self._L.orc_last_error().decode())
        if rc == 2:
            raise OracleTypeError(self._L.orc_last_error().decode())

    def op_info(self, i: int):
        kind = C.c_int()
        nq = C.c_int()
        qs = np.zeros(16, dtype=np.int32)
        mat = np.zeros(2 * 4096, dtype=np.float64)
        m = self._L.orc_op_info(self.h_, i, C.byref(kind), _ip(qs), C.byref(nq), _dp(mat), 4096)
        mm = mat[: 2 * m].view(np.complex128).copy()
        return KIND_NAMES[kind.value], [int(x) for x in qs[: nq.value]], mm

    # classical ops (circuit.ts:1598-1642); classical bits are numbered
    # consecutively over all registers by the caller
    def measure(self, q: int, cbit: int) -> "OCircuit":
        self._raise(self._L.orc_add_measure(self.h_, q, cbit))
        return self

    def reset(self, q: int) -> "OCircuit":
        self._raise(self._L.orc_add_reset(self.h_, q))
        return self

    def if_(self, reg0: int, regn: int, value: int, body: "OCircuit") -> "OCircuit":
        self._raise(self._L.orc_add_if(self.h_, reg0, regn, value, body.h_))
        return self

    def run_pershot(self, shots: int, seed_state: int, p1=0.0, p2=0.0, pmeas=0.0, ncbits=0, init: int = 0):
        """run() per-shot path (circuit.ts:3455-3481): (sampled index per shot,
        classical bits per shot [shots, ncbits], xorshift32 state after the
        last draw).  seed_state: the stream's state (makePrng: seed, 0 -> 1)."""
        idx = np.zeros(max(shots, 1), dtype=np.uint64)
        bits = np.zeros(max(shots * ncbits, 1), dtype=np.uint8)
        st = self._L.orc_run_pershot(self.h_, init, shots, seed_state, p1, p2, pmeas, ncbits,
                                     idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                     bits.ctypes.data_as(C.POINTER(C.c_uint8)))
        return idx[:shots], bits[: shots * ncbits].reshape(shots, ncbits), int(st)

    def dm(self, p1: float = 0.0, p2: float = 0.0) -> "ODM":
        """runDM (density.ts:475-588) with depolarizing noise p1, p2."""
        return ODM(self._L.orc_dm_run(self.h_, p1, p2), self.qubits)

    def circuit_matrix(self) -> np.ndarray:
        """circuitMatrix() (circuit.ts:1462-1485): one sparse simulation per column."""
        dim = 1 << self.qubits
        out = np.zeros((dim, dim), dtype=np.complex128)
        self._L.orc_circuit_matrix(self.h_, out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def simulate(self, init: int = 0, mode: int = SPARSE) -> "OState":
        return OState(self._L.orc_simulate(self.h_, init, mode), self.qubits)

    def time_ops(self, first: int, count: int, init: int = 0, mode: int = SPARSE):
        """(seconds, amplitude updates) for ops [first, first+count) after
        simulating ops [0, first) untimed."""
        sec = C.c_double()
        upd = self._L.orc_time_ops(self.h_, init, mode, first, count, C.byref(sec))
        return sec.value, int(upd)

    def expectation(self, pauli: str, init: int = 0, mode: int = SPARSE) -> float:
        return self._L.orc_expectation(self.h_, pauli.encode(), init, mode)

    def vqe(self, terms, mode: int = SPARSE) -> float:
        coeffs, ops = _terms(terms, self.qubits)
        return self._L.orc_vqe(self.h_, len(terms), _dp(coeffs), ops, mode)


def _terms(terms, n):
    coeffs = np.ascontiguousarray([t[0] for t in terms], dtype=np.float64)
    if coeffs.size == 0:
        coeffs = np.zeros(1)
    ops = "".join(t[1] for t in terms)
    assert all(len(t[1]) == n for t in terms)
    return coeffs, ops.encode()


class ODM:
    """The oracle's density matrix (density.ts DensityMatrix)."""

    def __init__(self, handle, n):
        self._L = lib()
        self.h_ = handle
        self.n = n

    def __del__(self):
        try:
            self._L.orc_dm_free(self.h_)
        except Exception:
            pass

    def dense(self) -> np.ndarray:
        dim = 1 << self.n
        out = np.zeros((dim, dim), dtype=np.complex128)
        self._L.orc_dm_dense(self.h_, self.n, out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def nnz(self) -> int:
        return int(self._L.orc_dm_nnz(self.h_))

    def purity(self) -> float:
        return self._L.orc_dm_purity(self.h_)

    def entropy(self) -> float:
        return self._L.orc_dm_entropy(self.h_, self.n)

    def bloch(self, q: int):
        out = np.zeros(2)
        self._L.orc_dm_bloch(self.h_, self.n, q, _dp(out))
        return out

    def probabilities(self) -> dict:
        """probabilities() (density.ts:299-307): q0-leftmost key -> Re rho[r][r] > 1e-14."""
        d = np.real(np.diag(self.dense()))
        return {format(r, "b").zfill(self.n)[::-1]: float(v) for r, v in enumerate(d) if v > 1e-14}


class OState:
    def __init__(self, handle, n):
        self._L = lib()
        self.h_ = handle
        self.n = n

    def __del__(self):
        try:
            self._L.orc_state_free(self.h_)
        except Exception:
            pass

    def nnz(self) -> int:
        return int(self._L.orc_state_nnz(self.h_))

    def amplitude(self, idx: int) -> complex:
        out = np.zeros(2)
        self._L.orc_state_get(self.h_, idx, _dp(out))
        return complex(out[0], out[1])

    def dense(self) -> np.ndarray:
        out = np.zeros(2 << self.n, dtype=np.float64)
        self._L.orc_state_dense(self.h_, _dp(out))
        return out.view(np.complex128)

    def prune_stats(self):
        ev = C.c_uint64()
        mx = C.c_double()
        self._L.orc_state_prune_stats(self.h_, C.byref(ev), C.byref(mx))
        return int(ev.value), float(mx.value)

    def exact_probs(self):
        """(indices, probabilities) with p > 1e-14, ascending index."""
        cnt = self._L.orc_exact_probs(self.h_, None, None, 0)
        idx = np.zeros(max(cnt, 1), dtype=np.uint64)
        p = np.zeros(max(cnt, 1), dtype=np.float64)
        self._L.orc_exact_probs(self.h_, idx.ctypes.data_as(C.POINTER(C.c_uint64)), _dp(p), cnt)
        return idx[:cnt], p[:cnt]

    def run(self, shots: int, seed: int) -> np.ndarray:
        out = np.zeros(max(shots, 1), dtype=np.uint64)
        self._L.orc_run(self.h_, shots, seed & 0xFFFFFFFF, out.ctypes.data_as(C.POINTER(C.c_uint64)))
        return out[:shots]

    def bloch(self, q: int):
        """blochAngles(q) (circuit.ts:4102-4129): (rho00, rho11, Re rho01, Im rho01, theta, phi)."""
        out = np.zeros(6)
        self._L.orc_bloch(self.h_, q, _dp(out))
        return out

    def marginals(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.float64)
        self._L.orc_marginals(self.h_, _dp(out))
        return out


def qft(n: int) -> OCircuit:
    return OCircuit(handle=lib().orc_qft(n))


def iqft(n: int) -> OCircuit:
    return OCircuit(handle=lib().orc_iqft(n))


def qaoa(n, edges, gamma, beta) -> OCircuit:
    e = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1))
    g = np.ascontiguousarray(gamma, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    return OCircuit(handle=lib().orc_qaoa(n, _ip(e), len(edges), _dp(g), _dp(b), len(gamma)))


def maxcut_hamiltonian(n, edges):
    e = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1))
    coeffs = np.zeros(len(edges) + 1)
    ops = C.create_string_buffer((len(edges) + 1) * n + 1)
    k = lib().orc_maxcut_hamiltonian(n, _ip(e), len(edges), _dp(coeffs), ops)
    raw = ops.raw.decode()
    return [(float(coeffs[t]), raw[t * n:(t + 1) * n]) for t in range(k)]


def ansatz_params(kind, n, reps) -> int:
    return lib().orc_ansatz_params(kind, n, reps)


def ansatz(kind, n, reps, params) -> OCircuit:
    p = np.ascontiguousarray(params, dtype=np.float64)
    return OCircuit(handle=lib().orc_ansatz(kind, n, reps, _dp(p)))


def gradient(kind, n, reps, params, terms, mode=SPARSE) -> np.ndarray:
    p = np.ascontiguousarray(params, dtype=np.float64)
    coeffs, ops = _terms(terms, n)
    g = np.zeros(p.size)
    lib().orc_gradient(kind, n, reps, _dp(p), len(terms), _dp(coeffs), ops, mode, _dp(g))
    return g


def minimize(kind, n, reps, params, terms, lr=0.1, steps=200, tol=1e-6, mode=SPARSE):
    p = np.array(params, dtype=np.float64)
    coeffs, ops = _terms(terms, n)
    e = C.c_double()
    conv = C.c_int()
    k = lib().orc_minimize(kind, n, reps, _dp(p), len(terms), _dp(coeffs), ops, lr, steps, tol, mode,
                           C.byref(e), C.byref(conv))
    return {"params": p, "energy": e.value, "steps": k, "converged": bool(conv.value)}


def brickwork(n, layers, seed, with_qft=False):
    st = C.c_uint32()
    c = OCircuit(handle=lib().orc_brickwork(n, layers, seed, 1 if with_qft else 0, C.byref(st)))
    return c, int(st.value)


def regular3(n, state):
    st = C.c_uint32(state)
    edges = np.zeros(3 * n, dtype=np.int32)
    k = lib().orc_regular3(n, C.byref(st), _ip(edges))
    return [(int(edges[2 * i]), int(edges[2 * i + 1])) for i in range(k)], int(st.value)


def prng_next(state):
    st = C.c_uint32(state)
    v = lib().orc_prng_next(C.byref(st))
    return int(v), int(st.value)
