"""Circuits loaded from ket's JSON run on the engine exactly as the circuits
they were written from (circuit.test.ts:4524-4532, :4568-4574)."""
import ctypes as C

import numpy as np
import pytest

import ket_b200 as K
from ket_b200 import _lib, workloads as W
from ket_b200.circuit import DeviceState, ops_to_abi, flatten_ops
from ket_b200.circuit_json import js_stringify, program_from_json

pytestmark = pytest.mark.gpu


def test_loaded_program_simulates_identically():
    c, _ = W.brickwork_qft(14, 12, 42)
    p = program_from_json(js_stringify(c.toJSON()))
    a = DeviceState(14)
    a.set_basis(0)
    a.apply_abi(p["ops"], p["mats"], p["count"])
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    b = DeviceState(14)
    b.set_basis(0)
    b.apply_abi(arr, m, k)
    assert np.array_equal(a.amplitudes_dense(), b.amplitudes_dense())
    # and the mirror's round trip gives the same distribution (circuit.test.ts:4568-4574)
    r1 = c.run(shots=1000, seed=7)
    r2 = K.Circuit.fromJSON(js_stringify(c.toJSON())).run(shots=1000, seed=7)
    assert r1.probs == r2.probs


def test_classical_round_trip_runs_identically():
    """circuit.test.ts:4524-4532, and the loader's packing through ket_run_shots."""
    orig = K.Circuit(2).creg("c", 1).h(0).measure(0, "c", 0).if_("c", 1, lambda c: c.x(1)).reset(0)
    loaded = K.Circuit.fromJSON(orig.toJSON())
    r1 = orig.run(shots=200, seed=99)
    r2 = loaded.run(shots=200, seed=99)
    assert r1.probs == r2.probs and r1.cregs == r2.cregs
    p = program_from_json(js_stringify(orig.toJSON()))
    st = DeviceState(2)
    state = C.c_uint32(99)
    idx = np.zeros(200, dtype=np.uint64)
    bits = np.zeros(200 * p["ncbits"], dtype=np.uint8)
    mv = p["mats"].view(np.float64)
    _lib.check(_lib.lib().ket_run_shots(st.h, p["ops"], p["count"], mv.ctypes.data_as(C.POINTER(C.c_double)),
                                        p["mats"].size, None, 0, 200, C.byref(state), p["ncbits"],
                                        idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                        bits.ctypes.data_as(C.POINTER(C.c_uint8))))
    i2, b2, _, _ = orig.run_shots(200, seed=99)
    assert np.array_equal(idx, i2) and np.array_equal(bits.reshape(200, -1), b2)
