"""ket_b200: a B200-native dense statevector engine behind ket's Circuit API.

The engine is a C-ABI shared library (include/ket_sv.h, built from
ket_b200/csrc for sm_100a); this package is its host-side mirror of the
reference's TypeScript interface (src/circuit.ts, src/algorithms.ts).
"""
from ._lib import KET_C128, KET_C64, KetError, RangeError
from .circuit import Circuit, DeviceState, Distribution, flatten_ops, make_prng
from .algorithms import (AnsatzFn, MinimizeResult, PauliTerm, efficientSU2, gradient, gradient_shift, iqft,
                         maxCutHamiltonian, minimize, qaoa, qft, realAmplitudes, vqe)
from . import gates
from .batch import batch_qaoa

__all__ = ["Circuit", "Distribution", "DeviceState", "flatten_ops", "make_prng", "KET_C128", "KET_C64", "KetError",
           "RangeError", "AnsatzFn", "MinimizeResult", "PauliTerm", "efficientSU2", "gradient", "gradient_shift",
           "iqft", "maxCutHamiltonian", "minimize", "qaoa", "qft", "realAmplitudes", "vqe", "gates"]
