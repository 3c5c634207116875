"""ket's circuit JSON: the Python mirror's Circuit.toJSON / fromJSON and the
C ABI's loader (ket_program_from_json), against the reference's
toJSON / fromJSON tests (circuit.test.ts:4386-4605) restated, JSON text
written by hand from opsToJSON's field order (circuit.ts:583-600), and each
other: both loaders must give the same op list and the same matrices, bit for
bit."""
import ctypes as C
import math

import numpy as np
import pytest

import ket_b200 as K
from ket_b200 import _lib
from ket_b200.circuit import flatten_ops, ops_to_abi, shots_to_abi
from ket_b200.circuit_json import js_stringify, program_from_json

PI = math.pi


def rt(c):
    return K.Circuit.fromJSON(c.toJSON())


def abi_list(arr, m, k):
    out = []
    for i in range(k):
        o = arr[i]
        mat = None
        if o.kind in (_lib.OP_SINGLE, _lib.OP_CONTROLLED, _lib.OP_TWO, _lib.OP_UNITARY) and o.mat >= 0:
            d = 1 << (o.nq if o.kind == _lib.OP_UNITARY else (2 if o.kind == _lib.OP_TWO else 1))
            mat = np.asarray(m[o.mat:o.mat + d * d]).view(np.float64).tobytes()
        out.append((o.kind, tuple(o.q[j] for j in range(o.nq)), mat))
    return out


def same_ops(a, b):
    return abi_list(*ops_to_abi(flatten_ops(a.ops))) == abi_list(*ops_to_abi(flatten_ops(b.ops)))


def loader_ops(c):
    p = program_from_json(js_stringify(c.toJSON()))
    assert p["qubits"] == c.qubits
    return abi_list(p["ops"], p["mats"], p["count"])


def builders():
    t = PI / 7
    return {
        "h": lambda c: c.h(0), "x": lambda c: c.x(0), "y": lambda c: c.y(0), "z": lambda c: c.z(0),
        "s": lambda c: c.s(0), "si": lambda c: c.si(0), "sdg": lambda c: c.sdg(0), "t": lambda c: c.t(0),
        "ti": lambda c: c.ti(0), "tdg": lambda c: c.tdg(0), "v": lambda c: c.v(0), "vi": lambda c: c.vi(0),
        "srn": lambda c: c.srn(0), "srndg": lambda c: c.srndg(0), "id": lambda c: c.id(0),
        "rx": lambda c: c.rx(t, 0), "ry": lambda c: c.ry(t, 0), "rz": lambda c: c.rz(t, 0), "vz": lambda c: c.vz(t, 0),
        "u1": lambda c: c.u1(t, 0), "p": lambda c: c.p(t, 0), "u2": lambda c: c.u2(t, t, 0),
        "u3": lambda c: c.u3(t, t, t, 0), "gpi": lambda c: c.gpi(t, 0), "gpi2": lambda c: c.gpi2(t, 0),
        "r248": lambda c: c.r2(0).r4(0).r8(0),
        "cnot": lambda c: c.h(0).cnot(0, 1), "swap": lambda c: c.x(0).swap(0, 1),
        "xx": lambda c: c.xx(t, 0, 1), "yy": lambda c: c.yy(t, 0, 1), "zz": lambda c: c.zz(t, 0, 1),
        "xy": lambda c: c.xy(t, 0, 1), "iswap": lambda c: c.iswap(0, 1), "srswap": lambda c: c.srswap(0, 1),
        "ms": lambda c: c.ms(t, t, 0, 1),
        "cy": lambda c: c.h(0).cy(0, 1), "cz": lambda c: c.h(0).cz(0, 1), "ch": lambda c: c.h(0).ch(0, 1),
        "crx": lambda c: c.h(0).crx(t, 0, 1), "cry": lambda c: c.h(0).cry(t, 0, 1),
        "crz": lambda c: c.h(0).crz(t, 0, 1), "cu1": lambda c: c.h(0).cu1(t, 0, 1),
        "cu2": lambda c: c.h(0).cu2(t, t, 0, 1), "cu3": lambda c: c.h(0).cu3(t, t, t, 0, 1),
        "cs": lambda c: c.h(0).cs(0, 1), "ct": lambda c: c.h(0).ct(0, 1), "csdg": lambda c: c.h(0).csdg(0, 1),
        "ctdg": lambda c: c.h(0).ctdg(0, 1), "cr2": lambda c: c.h(0).cr2(0, 1), "cr4": lambda c: c.h(0).cr4(0, 1),
        "cr8": lambda c: c.h(0).cr8(0, 1), "csrn": lambda c: c.h(0).csrn(0, 1),
        "ccx": lambda c: c.x(0).x(1).ccx(0, 1, 2), "cswap": lambda c: c.x(0).x(1).cswap(0, 1, 2),
        "csrswap": lambda c: c.x(0).csrswap(0, 1, 2),
        "unitary": lambda c: c.unitary([[0, 1], [1, 0]], 2).unitary(
            [[complex(0.6, 0), complex(0, 0.8)], [complex(0, 0.8), complex(0.6, 0)]], 1),
        "barrier": lambda c: c.h(0).barrier().h(1),
    }


def test_schema_version_and_qubits():
    """circuit.test.ts:4401-4407, :4594-4599"""
    assert K.Circuit(1).h(0).toJSON()["ket"] == 1
    assert rt(K.Circuit(3)).qubits == 3
    j = K.Circuit(1).rx(PI / 3, 0).toJSON()
    assert "gate" not in j["ops"][0] and j["ops"][0]["meta"]["name"] == "rx"


@pytest.mark.parametrize("name", list(builders()))
def test_round_trip_every_gate(name):
    """circuit.test.ts:4415-4509: every gate survives the round trip; here the
    op lists and matrices must be identical, and the C loader must produce
    the same op list as the Python mirror."""
    c = builders()[name](K.Circuit(3))
    assert same_ops(c, rt(c))
    assert loader_ops(c) == abi_list(*ops_to_abi(flatten_ops(c.ops)))


def test_json_text():
    """JSON.stringify(c.toJSON()) for circuits whose text follows from
    opsToJSON's field order and Number::toString."""
    cases = [
        (K.Circuit(2).h(0).cnot(0, 1),
         '{"ket":1,"qubits":2,"cregs":{},"gates":{},"ops":[{"kind":"single","q":0,"meta":{"name":"h"}},'
         '{"kind":"cnot","control":0,"target":1}]}'),
        (K.Circuit(1).rx(0.5, 0).u3(1, 1e-7, 2.5e21, 0),
         '{"ket":1,"qubits":1,"cregs":{},"gates":{},"ops":[{"kind":"single","q":0,"meta":{"name":"rx","params":[0.5]}},'
         '{"kind":"single","q":0,"meta":{"name":"u3","params":[1,1e-7,2.5e+21]}}]}'),
        (K.Circuit(2).creg("c", 1).h(0).measure(0, "c", 0).if_("c", 1, lambda c: c.x(1)).reset(0),
         '{"ket":1,"qubits":2,"cregs":{"c":1},"gates":{},"ops":[{"kind":"single","q":0,"meta":{"name":"h"}},'
         '{"kind":"measure","q":0,"creg":"c","bit":0},{"kind":"if","creg":"c","value":1,"ops":'
         '[{"kind":"single","q":1,"meta":{"name":"x"}}]},{"kind":"reset","q":0}]}'),
        (K.Circuit(3).xx(0.25, 0, 2).crz(-0.125, 2, 1).ccx(0, 1, 2).csrswap(2, 0, 1).barrier(0, 1),
         '{"ket":1,"qubits":3,"cregs":{},"gates":{},"ops":[{"kind":"two","a":0,"b":2,"meta":{"name":"xx","params":[0.25]}},'
         '{"kind":"controlled","control":2,"target":1,"meta":{"name":"crz","params":[-0.125]}},'
         '{"kind":"toffoli","c1":0,"c2":1,"target":2},{"kind":"csrswap","control":2,"a":0,"b":1},'
         '{"kind":"barrier","qubits":[0,1]}]}'),
        (K.Circuit(2).defineGate("bell", K.Circuit(2).h(0).cnot(0, 1)).gate("bell", 1, 0),
         '{"ket":1,"qubits":2,"cregs":{},"gates":{"bell":{"qubits":2,"ops":[{"kind":"single","q":0,"meta":'
         '{"name":"h"}},{"kind":"cnot","control":0,"target":1}]}},"ops":[{"kind":"subcircuit","name":"bell",'
         '"qubits":[1,0],"def":[{"kind":"single","q":0,"meta":{"name":"h"}},{"kind":"cnot","control":0,"target":1}]}]}'),
        (K.Circuit(1).unitary([[0, 1], [1, 0]], 0),
         '{"ket":1,"qubits":1,"cregs":{},"gates":{},"ops":[{"kind":"unitary","qubits":[0],'
         '"matrix":[[[0,0],[1,0]],[[1,0],[0,0]]]}]}'),
    ]
    for c, text in cases:
        assert js_stringify(c.toJSON()) == text
        assert js_stringify(K.Circuit.fromJSON(text).toJSON()) == text


def test_classical_registers_and_ops():
    """circuit.test.ts:4511-4532: registers survive; measure / reset / if round
    trip; the C loader packs them as ket_run_shots expects."""
    j = K.Circuit(2).creg("c", 2).toJSON()
    assert j["cregs"]["c"] == 2
    K.Circuit.fromJSON(j).measure(0, "c", 0)
    c = (K.Circuit(3).creg("c", 1).creg("d", 2).h(0).measure(0, "c", 0).if_("c", 1, lambda b: b.x(1))
         .measure(1, "d", 1).if_("d", 2, lambda b: b.if_("c", 1, lambda bb: bb.h(2))).reset(0))
    loaded = rt(c)
    a1, m1, k1, n1, l1 = shots_to_abi(c.ops, c._cregs)
    a2, m2, k2, n2, l2 = shots_to_abi(loaded.ops, loaded._cregs)
    assert abi_list(a1, m1, k1) == abi_list(a2, m2, k2) and (n1, l1) == (n2, l2)
    p = program_from_json(js_stringify(c.toJSON()))
    assert p["classical"] and p["ncbits"] == n1 and p["registers"] == l1
    assert abi_list(p["ops"], p["mats"], p["count"]) == abi_list(a1, m1, k1)


def test_named_gates():
    """circuit.test.ts:4534-4546"""
    bell = K.Circuit(2).h(0).cnot(0, 1)
    orig = K.Circuit(4).defineGate("bell", bell).gate("bell", 0, 1).gate("bell", 2, 3)
    loaded = rt(orig)
    assert same_ops(orig, loaded) and "bell" in loaded.toJSON()["gates"]
    inner = K.Circuit(1).h(0).z(0)
    outer = K.Circuit(2).defineGate("inner", inner).gate("inner", 0).gate("inner", 1)
    assert same_ops(outer, rt(outer))
    assert loader_ops(orig) == abi_list(*ops_to_abi(flatten_ops(orig.ops)))
    assert loader_ops(outer) == abi_list(*ops_to_abi(flatten_ops(outer.ops)))


def test_from_json_string_and_ghz():
    """circuit.test.ts:4548-4552, :4601-4605"""
    orig = K.Circuit(1).h(0)
    assert same_ops(orig, K.Circuit.fromJSON(js_stringify(orig.toJSON())))
    c = K.Circuit(5).h(0)
    for i in range(4):
        c = c.cnot(i, i + 1)
    assert same_ops(c, rt(c))


def test_errors():
    """circuit.test.ts:4578-4592: TypeErrors in the mirror, KET_ERR_TYPE in the loader."""
    bad = [{"ket": 2, "qubits": 1, "cregs": {}, "gates": {}, "ops": []},
           {"ket": 1, "qubits": 1, "cregs": {}, "gates": {}, "ops": [{"kind": "teleport", "q": 0}]},
           {"ket": 1, "qubits": 1, "cregs": {}, "gates": {}, "ops": [{"kind": "single", "q": 0, "meta": {"name": "banana"}}]}]
    for j in bad:
        with pytest.raises(TypeError):
            K.Circuit.fromJSON(j)
        with pytest.raises(TypeError):
            program_from_json(js_stringify(j))
    # unbound parameters load in the mirror (bind() later) but not into an op list
    c = K.Circuit(1).rx("theta", 0)
    K.Circuit.fromJSON(c.toJSON())
    with pytest.raises(TypeError, match="unbound"):
        program_from_json(js_stringify(c.toJSON()))


def test_parser_robustness():
    L = _lib.lib()
    h = C.c_void_p()
    ok = ('  {"ket" : 1 , "qubits":2,"cregs":{"r\\u00e9g\\n\\"x\\"":1,"\\ud83d\\ude00":2},"gates":{},'
          '"ops":[{"kind":"single","q":0,"meta":{"name":"rx","params":[-1.5E-3]}},{"kind":"measure","q":1,'
          '"creg":"\\ud83d\\ude00","bit":1}]}  ')
    p = program_from_json(ok)
    assert list(p["registers"]) == ['rég\n"x"', "\U0001F600"]
    assert p["registers"]["\U0001F600"] == (1, 2) and p["ops"][1].q[1] == 2
    assert p["mats"][0] == complex(math.cos(-1.5e-3 / 2), 0)
    for text in ["", "{", '{"ket":1', '{"ket":1,"qubits":1,"cregs":{},"gates":{},"ops":[]} x', "[" * 1000 + "]" * 1000,
                 '{"ket":1,"qubits":1,"cregs":{},"gates":{},"ops":[{"kind":"single","q":0,"meta":{"name":"h"}},]}',
                 '{"ket":1,"qubits":1,"cregs":{},"gates":{},"ops":[{"kind":"single","q":01}]}',
                 '{"ket":1,"qubits":1,"cregs":{},"gates":{},"ops":[{"kind":"single","q":"\\x"}]}',
                 '{"ket":1,"qubits":41,"cregs":{},"gates":{},"ops":[]}']:
        raw = text.encode()
        assert L.ket_program_from_json(raw, len(raw), C.byref(h)) == _lib.KET_ERR_TYPE, text[:40]
