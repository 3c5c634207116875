"""ket's circuit JSON (schema "ket": 1): Circuit.toJSON / Circuit.fromJSON
(circuit.ts:3768-3806, opsToJSON / opsFromJSON :532-600) for the Python
mirror, JSON.stringify's text (so that a file written here is byte-for-byte
the one the reference writes), and the C ABI's loader (ket_program_from_json),
which lowers the same text straight to the engine's op list for hosts without
Node or Python."""
from __future__ import annotations

import ctypes as C
import json
import math
from typing import Dict, List, Optional, Union

import numpy as np

from . import gates as G
from ._lib import check, ket_op, lib

# ---------------------------------------------------------------- gate matrices from meta (circuit.ts:467-529)
_SINGLE_FIXED = {"h": G.H, "x": G.X, "y": G.Y, "z": G.Z, "s": G.S, "si": G.Si, "sdg": G.Si, "t": G.T, "ti": G.Ti,
                 "tdg": G.Ti, "v": G.V, "vi": G.Vi, "srn": G.V, "srndg": G.Vi, "sx": G.V, "sxdg": G.Vi, "id": G.Id,
                 "r2": G.R2, "r4": G.R4, "r8": G.R8}
_CTRL_FIXED = {"cx": G.X, "cy": G.Y, "cz": G.Z, "ch": G.H, "cs": G.S, "ct": G.T, "csdg": G.Si, "ctdg": G.Ti,
               "cr2": G.R2, "cr4": G.R4, "cr8": G.R8, "csrn": G.V}


def _p(ps, i):
    return ps[i] if i < len(ps) else float("nan")


def _single(name, ps):
    if name in _SINGLE_FIXED:
        return _SINGLE_FIXED[name]
    one = {"rx": G.Rx, "ry": G.Ry, "rz": G.Rz, "vz": G.Rz, "u1": G.U1, "p": G.U1, "gpi": G.Gpi, "gpi2": G.Gpi2}
    if name in one:
        return one[name](_p(ps, 0))
    if name == "u2":
        return G.U2(_p(ps, 0), _p(ps, 1))
    if name == "u3":
        return G.U3(_p(ps, 0), _p(ps, 1), _p(ps, 2))
    raise TypeError(f"fromJSON: unknown single-qubit gate '{name}'")


def _two(name, ps):
    one = {"xx": G.Xx, "yy": G.Yy, "zz": G.Zz, "xy": G.Xy}
    if name in one:
        return one[name](_p(ps, 0))
    if name == "iswap":
        return G.ISwap
    if name == "srswap":
        return G.SrSwap
    if name == "ms":
        return G.Ms(_p(ps, 0), _p(ps, 1))
    raise TypeError(f"fromJSON: unknown two-qubit gate '{name}'")


def _ctrl(name, ps):
    if name in _CTRL_FIXED:
        return _CTRL_FIXED[name]
    one = {"crx": G.Rx, "cry": G.Ry, "crz": G.Rz, "cu1": G.U1}
    if name in one:
        return one[name](_p(ps, 0))
    if name == "cu2":
        return G.U2(_p(ps, 0), _p(ps, 1))
    if name == "cu3":
        return G.U3(_p(ps, 0), _p(ps, 1), _p(ps, 2))
    raise TypeError(f"fromJSON: unknown controlled gate '{name}'")


# ---------------------------------------------------------------- opsToJSON / opsFromJSON
def _meta(op) -> dict:
    m = {"name": op.name}
    if op.params:
        m["params"] = [float(p) if not isinstance(p, str) else p for p in op.params]
    return m


def ops_to_json(ops) -> list:
    """opsToJSON (circuit.ts:583-600): gate ops carry their meta, not matrices."""
    out = []
    for op in ops:
        k, q = op.kind, op.qubits
        if k == "single":
            out.append({"kind": "single", "q": q[0], "meta": _meta(op)})
        elif k == "cnot":
            out.append({"kind": "cnot", "control": q[0], "target": q[1]})
        elif k == "swap":
            out.append({"kind": "swap", "a": q[0], "b": q[1]})
        elif k == "two":
            out.append({"kind": "two", "a": q[0], "b": q[1], "meta": _meta(op)})
        elif k == "controlled":
            out.append({"kind": "controlled", "control": q[0], "target": q[1], "meta": _meta(op)})
        elif k == "toffoli":
            out.append({"kind": "toffoli", "c1": q[0], "c2": q[1], "target": q[2]})
        elif k in ("cswap", "csrswap"):
            out.append({"kind": k, "control": q[0], "a": q[1], "b": q[2]})
        elif k == "measure":
            out.append({"kind": "measure", "q": q[0], "creg": op.extra[0], "bit": op.extra[1]})
        elif k == "reset":
            out.append({"kind": "reset", "q": q[0]})
        elif k == "if":
            out.append({"kind": "if", "creg": op.extra[0], "value": op.extra[1], "ops": ops_to_json(op.extra[2])})
        elif k == "subcircuit":
            out.append({"kind": "subcircuit", "name": op.name, "qubits": list(q), "def": ops_to_json(op.extra)})
        elif k == "barrier":
            out.append({"kind": "barrier", "qubits": list(q)})
        elif k == "unitary":
            out.append({"kind": "unitary", "qubits": list(q),
                        "matrix": [[[z.real, z.imag] for z in row] for row in op.gate]})
        elif k == "parametric":
            out.append({"kind": "parametric", "name": op.name, "params": list(op.params), "qubits": list(q)})
        else:
            raise TypeError(f"toJSON: unknown op kind '{k}'")
    return out


def ops_from_json(raw) -> list:
    """opsFromJSON (circuit.ts:532-580)."""
    from .circuit import Op
    out = []
    for o in raw:
        k = o.get("kind") if isinstance(o, dict) else None
        if k in ("single", "two", "controlled"):
            meta = o.get("meta")
            if not isinstance(meta, dict) or "name" not in meta:
                raise TypeError(f"fromJSON: {k} op without meta")
            name, ps = meta["name"], tuple(meta.get("params") or ())
            if k == "single":
                out.append(Op("single", (o["q"],), _single(name, ps), name, ps))
            elif k == "two":
                out.append(Op("two", (o["a"], o["b"]), _two(name, ps), name, ps))
            else:
                out.append(Op("controlled", (o["control"], o["target"]), _ctrl(name, ps), name, ps))
        elif k == "cnot":
            out.append(Op("cnot", (o["control"], o["target"]), None, "cnot"))
        elif k == "swap":
            out.append(Op("swap", (o["a"], o["b"]), None, "swap"))
        elif k == "toffoli":
            out.append(Op("toffoli", (o["c1"], o["c2"], o["target"]), None, "ccx"))
        elif k in ("cswap", "csrswap"):
            out.append(Op(k, (o["control"], o["a"], o["b"]), None, k))
        elif k == "measure":
            out.append(Op("measure", (o["q"],), None, "measure", (), (o["creg"], o["bit"])))
        elif k == "reset":
            out.append(Op("reset", (o["q"],), None, "reset"))
        elif k == "if":
            out.append(Op("if", (), None, "if", (), (o["creg"], o["value"], tuple(ops_from_json(o["ops"])))))
        elif k == "subcircuit":
            out.append(Op("subcircuit", tuple(o["qubits"]), None, o["name"], (), tuple(ops_from_json(o["def"]))))
        elif k == "barrier":
            out.append(Op("barrier", tuple(o["qubits"]), None, "barrier"))
        elif k == "parametric":
            out.append(Op("parametric", tuple(o["qubits"]), None, o["name"], tuple(o["params"])))
        elif k == "unitary":
            m = tuple(tuple(complex(z[0], z[1]) for z in row) for row in o["matrix"])
            out.append(Op("unitary", tuple(o["qubits"]), m, "unitary"))
        else:
            raise TypeError(f"fromJSON: unknown op kind '{k}'")
    return out


def to_json(circ) -> dict:
    """Circuit.toJSON (circuit.ts:3768-3778)."""
    gates = {name: {"qubits": sub.qubits, "ops": ops_to_json(sub.ops)} for name, sub in circ._gates.items()}
    return {"ket": 1, "qubits": circ.qubits, "cregs": dict(circ._cregs), "gates": gates,
            "ops": ops_to_json(circ.ops)}


def from_json(j: Union[dict, str]):
    """Circuit.fromJSON (circuit.ts:3794-3806): a dict or JSON text."""
    from .circuit import Circuit
    if isinstance(j, (str, bytes)):
        j = json.loads(j)
    if j.get("ket") != 1:
        raise TypeError(f"fromJSON: unsupported schema version {j.get('ket')}")
    gates = {name: Circuit(d["qubits"], ops_from_json(d["ops"])) for name, d in j.get("gates", {}).items()}
    return Circuit(j["qubits"], ops_from_json(j["ops"]), dict(j.get("cregs", {})), gates)


# ---------------------------------------------------------------- JSON.stringify's text
def js_number(x) -> str:
    """Number.prototype.toString (ECMA-262 Number::toString) as JSON.stringify
    writes it: shortest round-trip digits, exponent form below 1e-6 and from
    1e21 on; NaN and infinities become null."""
    if isinstance(x, bool):
        return "true" if x else "false"
    if isinstance(x, int):
        x = float(x) if abs(x) >= 2 ** 53 else x
        if isinstance(x, int):
            return str(x)
    if math.isnan(x) or math.isinf(x):
        return "null"
    if x == 0:
        return "0"
    sign = "-" if x < 0 else ""
    # repr gives the shortest round-trip digits; write them as D x 10^q
    mant, _, exp = repr(abs(x)).partition("e")
    ip, _, fp = mant.partition(".")
    digits = (ip + fp).lstrip("0")
    q = (int(exp) if exp else 0) - len(fp)
    stripped = digits.rstrip("0")
    q += len(digits) - len(stripped)
    digits = stripped
    k = len(digits)
    n = k + q  # the value is 0.digits x 10^n
    if k <= n <= 21:
        s = digits + "0" * (n - k)
    elif 0 < n <= 21:
        s = digits[:n] + "." + digits[n:]
    elif -6 < n <= 0:
        s = "0." + "0" * (-n) + digits
    else:
        e = n - 1
        s = digits[0] + ("." + digits[1:] if k > 1 else "") + "e" + ("+" if e >= 0 else "-") + str(abs(e))
    return sign + s


def js_stringify(v) -> str:
    """JSON.stringify(v) with no indentation, for the values toJSON builds."""
    if v is None:
        return "null"
    if isinstance(v, (bool, int, float, np.floating, np.integer)):
        return js_number(v.item() if isinstance(v, (np.floating, np.integer)) else v)
    if isinstance(v, str):
        return json.dumps(v, ensure_ascii=False)
    if isinstance(v, dict):
        return "{" + ",".join(json.dumps(str(k), ensure_ascii=False) + ":" + js_stringify(x) for k, x in v.items()) + "}"
    if isinstance(v, (list, tuple)):
        return "[" + ",".join(js_stringify(x) for x in v) + "]"
    raise TypeError(f"js_stringify: {type(v).__name__}")


# ---------------------------------------------------------------- the C ABI's loader
def program_from_json(text: Union[str, bytes]) -> dict:
    """Load JSON text with ket_program_from_json: {qubits, ops (ket_op array),
    mats (complex), count, ncbits, registers {name: (first, size)}, classical}."""
    raw = text.encode() if isinstance(text, str) else bytes(text)
    L = lib()
    h = C.c_void_p()
    check(L.ket_program_from_json(raw, len(raw), C.byref(h)))
    try:
        nq, nops, nmat = C.c_int(), C.c_size_t(), C.c_size_t()
        ncb, nregs, cl = C.c_int(), C.c_int(), C.c_int()
        check(L.ket_program_info(h, C.byref(nq), C.byref(nops), C.byref(nmat), C.byref(ncb), C.byref(nregs),
                                 C.byref(cl)))
        arr = (ket_op * max(1, nops.value))()
        mats = np.zeros(max(1, nmat.value), dtype=np.complex128)
        check(L.ket_program_ops(h, arr, nops.value, mats.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                mats.size))
        regs: Dict[str, tuple] = {}
        buf = C.create_string_buffer(256)
        for i in range(nregs.value):
            f, s = C.c_int(), C.c_int()
            check(L.ket_program_creg(h, i, buf, 256, C.byref(f), C.byref(s)))
            regs[buf.value.decode()] = (f.value, s.value)
        return {"qubits": nq.value, "ops": arr, "mats": mats, "count": nops.value, "ncbits": ncb.value,
                "registers": regs, "classical": bool(cl.value)}
    finally:
        L.ket_program_free(h)
