"""ctypes binding of the engine's C ABI (include/ket_sv.h).

This is the Python twin of the Node N-API addon (napi/ket_addon.c): it maps
status codes to the exceptions the reference throws (RangeError / TypeError)
and owns the process-wide default context.  There is no fallback: if the
CUDA library is missing or no GPU is present, the calls raise.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("KET_SV_LIB") or os.path.join(_HERE, "libket_sv.so")

KET_OK, KET_ERR_RANGE, KET_ERR_TYPE, KET_ERR_OOM, KET_ERR_CUDA, KET_ERR_TIMEOUT, KET_ERR_UNSUPPORTED = range(7)
KET_C128, KET_C64 = 0, 1

OP_SINGLE, OP_CNOT, OP_SWAP, OP_TWO, OP_CONTROLLED, OP_TOFFOLI, OP_CSWAP, OP_CSRSWAP, OP_UNITARY, OP_BARRIER = range(10)
OP_MEASURE, OP_RESET, OP_IF = 10, 11, 12  # ket_run_shots only
MAX_OP_QUBITS = 10

PG = {"rx": 0, "ry": 1, "rz": 2, "vz": 2, "u1": 3, "p": 3, "gpi": 4, "gpi2": 5, "crx": 6, "cry": 7, "crz": 8,
      "cu1": 9, "xx": 10, "yy": 11, "zz": 12, "xy": 13}


class RangeError(ValueError):
    """The reference's RangeError (e.g. a qubit index out of range)."""


class KetError(RuntimeError):
    """An engine failure with no reference counterpart (device, memory, timeout);
    `code` is the ket_status value."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


class ket_op(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nq", C.c_int32), ("q", C.c_int32 * MAX_OP_QUBITS), ("mat", C.c_int64)]


class ket_noise(C.Structure):
    _fields_ = [("p1", C.c_double), ("p2", C.c_double), ("pmeas", C.c_double)]


class ket_exec_opts(C.Structure):
    _fields_ = [("fusion", C.c_int32), ("prune", C.c_int32), ("specialize", C.c_int32), ("reg_bits", C.c_int32),
                ("stage", C.c_int32), ("reserved", C.c_int32 * 3)]


class ket_batch_template(C.Structure):
    _fields_ = [("nqubits", C.c_int32), ("nops", C.c_int32), ("nbinds", C.c_int32), ("nterms", C.c_int32),
                ("op_first", C.c_int64), ("bind_first", C.c_int64), ("term_first", C.c_int64),
                ("pauli_first", C.c_int64)]


class ket_param_binding(C.Structure):
    _fields_ = [("op", C.c_int32), ("gate", C.c_int32), ("param", C.c_int32), ("reserved", C.c_int32),
                ("scale", C.c_double), ("shift", C.c_double)]


_lib = None
_lock = threading.Lock()


def lib():
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"ket_b200 CUDA library not built: {LIB_PATH} is missing (run ket_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        vp, i32, u64, dbl, sz = C.c_void_p, C.c_int, C.c_uint64, C.c_double, C.c_size_t
        P = C.POINTER
        sigs = {
            "ket_last_error": (C.c_char_p, []),
            "ket_abi_version": (i32, []),
            "ket_exec_opts_default": (None, [P(ket_exec_opts)]),
            "ket_debug_fail_alloc": (i32, [i32]),
            "ket_debug_batch_hook": (i32, [i32, C.c_uint32]),
            "ket_debug_adjoint_budget": (i32, [C.c_int64]),
            "ket_debug_stage_drop": (i32, [C.c_int64]),
            "ket_batch_config": (i32, [vp, i32, i32]),
            "ket_ctx_create": (i32, [i32, P(vp)]),
            "ket_ctx_destroy": (i32, [vp]),
            "ket_ctx_scratch_bytes": (i32, [vp, P(u64)]),
            "ket_ctx_profile": (i32, [vp, i32]),
            "ket_ctx_profile_read": (i32, [vp, P(i32), P(C.c_float), sz, P(sz)]),
            "ket_ctx_launch_count": (i32, [vp, P(u64)]),
            "ket_measure_fp64": (i32, [vp, P(dbl)]),
            "ket_ctx_stream": (i32, [vp, P(vp)]),
            "ket_marginals_noalloc": (i32, [vp, i32, i32, vp, vp]),
            "ket_state_compare": (i32, [vp, vp, P(dbl), P(dbl)]),
            "ket_ctx_io_bytes": (i32, [vp, P(u64), P(u64)]),
            "ket_state_alloc": (i32, [vp, i32, i32, P(vp)]),
            "ket_state_free": (i32, [vp]),
            "ket_state_qubits": (i32, [vp, P(i32), P(i32)]),
            "ket_state_set_basis": (i32, [vp, u64]),
            "ket_state_set_amplitudes": (i32, [vp, u64, u64, P(dbl)]),
            "ket_state_get_amplitudes": (i32, [vp, u64, u64, P(dbl)]),
            "ket_state_copy": (i32, [vp, vp]),
            "ket_apply_ops": (i32, [vp, P(ket_op), sz, P(dbl), sz, P(ket_exec_opts)]),
            "ket_plan_stats": (i32, [i32, i32, P(ket_op), sz, P(dbl), sz, P(ket_exec_opts), P(C.c_int64)]),
            "ket_jit_wait": (i32, []),
            "ket_jit_shutdown": (i32, []),
            "ket_jit_stats": (i32, [P(C.c_int64), P(dbl)]),
            "ket_jit_compile": (i32, [i32, i32, P(ket_op), sz, P(dbl), sz, P(ket_exec_opts), P(C.c_int64),
                                    C.c_char_p, sz]),
            "ket_plan_program_stats": (i32, [i32, i32, P(ket_op), sz, P(dbl), sz, P(ket_exec_opts),
                                             P(C.c_int64)]),
            "ket_amplitudes": (i32, [vp, P(u64), sz, P(dbl)]),
            "ket_probs_dense": (i32, [vp, dbl, P(dbl)]),
            "ket_probs_sparse": (i32, [vp, dbl, P(u64), P(dbl), u64, P(u64)]),
            "ket_marginals": (i32, [vp, P(dbl)]),
            "ket_marginal_dist": (i32, [vp, P(i32), i32, P(dbl)]),
            "ket_norm2": (i32, [vp, P(dbl)]),
            "ket_sample": (i32, [vp, P(dbl), sz, dbl, P(u64)]),
            "ket_run_shots": (i32, [vp, P(ket_op), sz, P(dbl), sz, P(ket_noise), u64, sz, P(C.c_uint32), i32,
                                    P(u64), P(C.c_uint8)]),
            "ket_debug_pershot_path": (i32, [i32]),
            "ket_circuit_matrix": (i32, [vp, i32, P(ket_op), sz, P(dbl), sz, P(ket_exec_opts), P(dbl)]),
            "ket_bloch": (i32, [vp, i32, P(dbl)]),
            "ket_dm_run": (i32, [vp, P(ket_op), sz, P(dbl), sz, dbl, dbl]),
            "ket_dm_probs": (i32, [vp, P(dbl)]),
            "ket_dm_bloch": (i32, [vp, i32, P(dbl)]),
            "ket_program_from_json": (i32, [C.c_char_p, sz, P(vp)]),
            "ket_program_free": (i32, [vp]),
            "ket_program_info": (i32, [vp, P(i32), P(sz), P(sz), P(i32), P(i32), P(i32)]),
            "ket_program_ops": (i32, [vp, P(ket_op), sz, P(dbl), sz]),
            "ket_program_creg": (i32, [vp, i32, C.c_char_p, sz, P(i32), P(i32)]),
            "ket_expect_pauli": (i32, [vp, C.c_char_p, P(dbl)]),
            "ket_expect_pauli_sum": (i32, [vp, i32, P(dbl), C.c_char_p, P(dbl)]),
            "ket_adjoint_gradient": (i32, [vp, i32, u64, P(ket_op), sz, P(dbl), sz, P(ket_param_binding), sz,
                                           P(dbl), i32, i32, i32, P(dbl), C.c_char_p, i32, P(dbl), P(dbl)]),
            "ket_shift_gradient": (i32, [vp, i32, u64, P(ket_op), sz, P(dbl), sz, P(ket_param_binding), sz,
                                         P(dbl), i32, i32, i32, P(dbl), C.c_char_p, i32, P(dbl), P(dbl)]),
            "ket_batch_vqe": (i32, [vp, i32, P(ket_batch_template), P(ket_op), P(dbl), sz, P(ket_param_binding),
                                    P(dbl), C.c_char_p, i32, P(i32), P(dbl), i32, i32, P(dbl)]),
            "ket_batch_qaoa": (i32, [vp, i32, P(i32), P(i32), P(C.c_int64), P(i32), i32, P(dbl), P(dbl), i32,
                                     P(dbl)]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        # no pass-kernel compile may still run when the process tears down NVRTC
        atexit.register(L.ket_jit_shutdown)
        _lib = L
        return L


def check(rc: int):
    if rc == KET_OK:
        return
    msg = lib().ket_last_error().decode(errors="replace")
    if rc == KET_ERR_RANGE:
        raise RangeError(msg)
    if rc == KET_ERR_TYPE:
        raise TypeError(msg)
    raise KetError(f"ket engine error {rc}: {msg}", rc)


_ctx = None
_ctx_lock = threading.Lock()


def default_ctx():
    """Process-wide engine context on CUDA device 0 (created on first use)."""
    global _ctx
    if _ctx is None:
        with _ctx_lock:
            if _ctx is None:
                h = C.c_void_p()
                dev = int(os.environ.get("KET_DEVICE", "0"))
                check(lib().ket_ctx_create(dev, C.byref(h)))
                _ctx = h
    return _ctx


def jit_stats() -> dict:
    """Compiled pass kernels in this process: shapes known, compiled, failed,
    launches, and the compile seconds summed over threads."""
    out, cs = (C.c_int64 * 4)(), C.c_double()
    check(lib().ket_jit_stats(out, C.byref(cs)))
    return {"kernels": out[0], "compiled": out[1], "failed": out[2], "launches": out[3], "compile_s": cs.value}


def exec_opts(fusion: int = -1, prune: bool = True, specialize: int = 0, reg_bits: int = 0,
              stage: int = 0) -> ket_exec_opts:
    o = ket_exec_opts()
    lib().ket_exec_opts_default(C.byref(o))
    o.fusion = fusion
    o.prune = 1 if prune else 0
    o.specialize = specialize
    o.reg_bits = reg_bits
    o.stage = stage
    return o
