"""Builds and loads the fused-program emulator (tests/cpp/emulate_program.cpp)
together with the engine's planner sources -- test infrastructure, CPU only."""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "ket_b200", "csrc")
OUT = os.path.join(HERE, "cpp", "_build", "libemu.so")
SRCS = [os.path.join(HERE, "cpp", "emulate_program.cpp"), os.path.join(CSRC, "planner.cpp"),
        os.path.join(CSRC, "program.cpp")]
_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    deps = SRCS + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(d) for d in deps):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                        "-o", OUT, *SRCS], check=True)
    L = C.CDLL(OUT)
    from ket_b200._lib import ket_op
    L.emu_apply_nreg.restype = C.c_int
    L.emu_apply_nreg.argtypes = [C.c_int, C.POINTER(ket_op), C.c_size_t, C.POINTER(C.c_double), C.c_size_t, C.c_int,
                                 C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int]
    L.emu_type_count.restype = C.c_int64
    L.emu_type_count.argtypes = [C.c_int]
    L.emu_set_deferred.restype = None
    L.emu_set_deferred.argtypes = [C.c_int]
    L.emu_sw_count.restype = C.c_int64
    L.emu_sw_count.argtypes = []
    L.emu_lane_defer_count.restype = C.c_int64
    L.emu_lane_defer_count.argtypes = []
    L.emu_adjoint_plan_digest.restype = C.c_int
    L.emu_adjoint_plan_digest.argtypes = [C.c_int, C.POINTER(ket_op), C.c_size_t, C.POINTER(C.c_double), C.c_size_t,
                                          C.c_int, C.POINTER(C.c_uint64)]
    L.emu_plan_digest.restype = C.c_int
    L.emu_plan_digest.argtypes = [C.c_int, C.c_int, C.POINTER(ket_op), C.c_size_t, C.POINTER(C.c_double), C.c_size_t,
                                  C.c_int, C.c_int, C.POINTER(C.c_uint64)]
    _lib = L
    return L


def sw_count():
    """Ops with deferred register swaps (FOF_SW) in the programs of the last emu_apply call."""
    return lib().emu_sw_count()


def lane_defer_count():
    """Deferred X gates on lane bits in the programs of the last emu_apply call."""
    return lib().emu_lane_defer_count()


def type_count(fop_type):
    """Ops of the given FOpType in the programs of the last emu_apply call."""
    return lib().emu_type_count(fop_type)


def emu_apply(n, ops, init_state, prune=True, fusion=-1, nreg=5, deferred=True):
    """nreg: register bits of the emulated layouts (5: ordinary passes, 4: adjoint passes).
    deferred: run the programs' deferred register swaps as the compiled kernels
    do (True) or carry every swap out at once as the interpreter does (False)."""
    from ket_b200.circuit import ops_to_abi
    lib().emu_set_deferred(1 if deferred else 0)
    arr, m, k = ops_to_abi(ops)
    st = np.ascontiguousarray(init_state, dtype=np.complex128).copy()
    passes = (C.c_int64 * 2)()
    mv = np.ascontiguousarray(m).view(np.float64)
    rc = lib().emu_apply_nreg(n, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, 1 if prune else 0, fusion,
                              st.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)), passes, nreg)
    return rc, st, list(passes)


def plan_digest(n, ops, precision, prune=True, nreg=4):
    """(FNV-1a digest of every tiled pass's layouts and program bytes, tiled
    passes, program ops) for ops planned as a run on an n-qubit state would."""
    from ket_b200.circuit import ops_to_abi
    arr, m, k = ops_to_abi(ops)
    mv = np.ascontiguousarray(m).view(np.float64)
    out = (C.c_uint64 * 3)()
    rc = lib().emu_plan_digest(n, precision, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                               1 if prune else 0, nreg, out)
    assert rc == 0, rc
    return out[0], out[1], out[2]


def adjoint_plan_digest(n, ops, nreg=4):
    """plan_digest for an adjoint-style reverse plan of ops on n + 1 qubits
    (ancilla n, a probe after every one-qubit matrix or diagonal gate)."""
    from ket_b200.circuit import ops_to_abi
    arr, m, k = ops_to_abi(ops)
    mv = np.ascontiguousarray(m).view(np.float64)
    out = (C.c_uint64 * 3)()
    rc = lib().emu_adjoint_plan_digest(n, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, nreg, out)
    assert rc == 0, rc
    return out[0], out[1], out[2]
