"""The pass kernels compiled per program (jit.cpp) build for sm_100a without a
GPU: the program generator's output for circuits that use every op kind is
turned into kernel source and compiled with NVRTC, in both precisions, with
and without the reference's pruning."""
import ctypes as C

import numpy as np
import pytest

from test_gpu_parity import random_gates


def _compile(n, gates, precision, prune):
    import ket_b200 as K
    from ket_b200 import _lib
    from ket_b200.circuit import flatten_ops, ops_to_abi
    c = K.Circuit(n)
    for name, qs, ps in gates:
        c = c.unitary(ps, *qs) if name == "unitary" else getattr(c, name)(*ps, *qs)
    arr, m, k = ops_to_abi(flatten_ops(c.ops))
    mv = np.ascontiguousarray(m).view(np.float64)
    o = _lib.exec_opts(prune=prune)
    kernels = C.c_int64()
    log = C.create_string_buffer(1 << 14)
    rc = _lib.lib().ket_jit_compile(n, precision, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size,
                                    C.byref(o), C.byref(kernels), log, len(log))
    return rc, kernels.value, log.value.decode(errors="replace")


@pytest.mark.parametrize("precision,prune", [(0, True), (1, False)])
def test_generated_kernels_compile(precision, prune):
    rc, kernels, log = _compile(13, random_gates(13, 70, 5), precision, prune)
    assert rc == 0, log
    assert kernels >= 1


def test_generated_kernels_compile_four_register_bits():
    """States of 26 qubits and more use programs with 4 register bits."""
    rc, kernels, log = _compile(26, random_gates(26, 60, 9), 0, True)
    assert rc == 0, log
    assert kernels >= 1


def test_plan_without_tiled_passes_compiles_nothing():
    rc, kernels, _ = _compile(8, random_gates(8, 20, 1), 0, True)
    assert rc == 0 and kernels == 0


EXIT_SCRIPT = r"""
import sys, threading, time, ctypes as C
sys.path.insert(0, sys.argv[1])
import numpy as np
from ket_b200 import _lib
from ket_b200.workloads import brickwork_qft
from ket_b200.circuit import ops_to_abi, flatten_ops
L = _lib.lib()
c, _ = brickwork_qft(22, 30, 5)
arr, m, k = ops_to_abi(flatten_ops(c.ops))
mv = np.ascontiguousarray(m).view(np.float64)
o = _lib.exec_opts()
def run():
    kern, log = C.c_int64(), C.create_string_buffer(256)
    L.ket_jit_compile(22, 0, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, C.byref(o),
                      C.byref(kern), log, 256)
threading.Thread(target=run, daemon=True).start()
time.sleep(2.0)
"""


def test_exit_while_compiling_is_clean():
    """A process that exits while kernels are still compiling exits cleanly:
    the binding's exit hook (ket_jit_shutdown) drops the queued compiles and
    waits for the running ones before the process tears NVRTC down."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", EXIT_SCRIPT, root], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]


TORCH_FIRST_SCRIPT = r"""
import sys, ctypes as C
sys.path.insert(0, sys.argv[1])
import torch  # noqa: F401  (brings its own libnvrtc.so.12 into the process)
import numpy as np
from ket_b200 import _lib
from ket_b200.workloads import brickwork_qft
from ket_b200.circuit import ops_to_abi, flatten_ops
c, _ = brickwork_qft(14, 2, 3)
arr, m, k = ops_to_abi(flatten_ops(c.ops))
mv = np.ascontiguousarray(m).view(np.float64)
o = _lib.exec_opts()
kern, log = C.c_int64(), C.create_string_buffer(1 << 14)
rc = _lib.lib().ket_jit_compile(14, 0, arr, k, mv.ctypes.data_as(C.POINTER(C.c_double)), m.size, C.byref(o),
                                C.byref(kern), log, len(log))
assert rc == 0 and kern.value >= 1, log.value.decode(errors="replace")[:2000]
"""


def test_compiles_after_torch_is_imported():
    """torch links its own, older NVRTC under the same soname; the kernels
    still compile when torch was imported first."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", TORCH_FIRST_SCRIPT, root], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]


def test_circuit_compile_kernels_ahead_of_a_run():
    """Circuit.compile_kernels fills the process's kernel cache (no GPU)."""
    import ket_b200 as K
    from ket_b200 import _lib
    from ket_b200.workloads import brickwork_qft
    c, _ = brickwork_qft(13, 3, 8)
    before = _lib.jit_stats()
    n = c.compile_kernels()
    after = _lib.jit_stats()
    assert n >= 1 and after["kernels"] >= before["kernels"] and after["failed"] == before["failed"]
    assert c.compile_kernels() == n  # cached: nothing new to compile
    assert _lib.jit_stats()["compiled"] == after["compiled"]
    with pytest.raises(TypeError):
        K.Circuit(1).creg("c", 1).measure(0, "c", 0).compile_kernels()
