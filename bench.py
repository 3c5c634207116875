#!/usr/bin/env python3
"""Benchmark of the B200 statevector engine on its headline workload.

Workload (one step): the 30-qubit dense complex128 state (16 GiB in HBM) is
reset to |0...0>, then the seeded 40-layer brickwork circuit followed by
qft(30) -- 2260 gates -- is applied, and the outputs are read back: 1024
amplitudes at seeded basis indices and the joint distribution of q0..q9.
Inputs are synthetic (xorshift32 seed 42, see ket_b200/workloads.py); the
16 GiB state exceeds the 126 MB L2, so no flush is needed between steps.

  value   gates/s over K steps timed by CUDA events on the engine's stream
          (barrier + synchronize on both sides; max over ranks); the state
          is resident, the step includes planning and every launch
  e2e     gates/s by wall clock through the public API from host buffers
          (op list + matrices in, amplitudes and marginals out)

The roofline entry is for the dominant kernel, the register-tiled fused pass:
algorithmic bytes per launch = 2 * 16 * 2^30 (one read and one write of the
state), divided by its mean event-timed duration.

--impl reference times the reference algorithm on the host cores instead:
the sparse-map restatement of src/statevector.ts (oracle/, the reference
itself is TypeScript and no JavaScript runtime exists on these machines) on
bounded samples of the same circuit family at 20 qubits, all host cores
running copies in parallel, converted to the same unit.

Multi-GPU (torchrun): the engine runs on one GPU; each rank runs an
independent replica of the workload (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ket", choices=["ket", "reference"])
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--layers", type=int, default=40)
    ap.add_argument("--prune", type=int, default=1, help="1: reference pruning semantics (default), 0: plain dense")
    ap.add_argument("--specialize", type=int, default=1,
                    help="register-tiled passes: 1 kernels compiled per pass program (compiled during warm-up), "
                         "-1 the interpreter k_fused2, 0 automatic")
    ap.add_argument("--stage", type=int, default=0,
                    help="compiled kernels' tile loads: 1 TMA-staged, -1 into registers, 0 automatic")
    ap.add_argument("--reg-bits", type=int, default=0, help="register bits of compiled programs (0 automatic, 4, 5)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the VQE-gradient, QAOA-batch and complex64 measurements")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Dist:
    """torch.distributed plumbing for replicas: barrier and max over ranks.
    backend "nccl" (one GPU per rank) or "gloo" (host tensors, used by the CPU
    tests of this plumbing)."""

    def __init__(self, world, rank, local, backend="nccl", timeout_s=600):
        self.world, self.rank, self.local = world, rank, local
        self.pg = None
        self.device = "cpu"
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(local)
                kw["device_id"] = torch.device("cuda", local)
                self.device = "cuda"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist
            self.torch = torch
            self.pg = True

    def barrier(self):
        if self.pg:
            self.dist.barrier()

    def max(self, v):
        if not self.pg:
            return v
        t = self.torch.tensor([float(v)], device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        busy = [s for s, p in zip(sm, power) if p > 200] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def ncu_traffic(n):
    """DRAM bytes per fused-pass launch from the committed ncu summary, scaled
    from the profiled state size to 2^n amplitudes."""
    try:
        with open(os.path.join(ROOT, "profiles", "fused_pass_traffic.json")) as f:
            d = json.load(f)
        return d["dram_bytes_per_launch"] * 2.0 ** (n - d["qubits"])
    except Exception:
        return None


# ---------------------------------------------------------------- CPU baseline
SAMPLE_N, SAMPLE_FIRST, SAMPLE_OPS = 20, 70, 12


def cpu_sample(_=None):
    """Time the reference algorithm (sparse map with pruning, 1 thread) on
    ops [SAMPLE_FIRST, SAMPLE_FIRST + SAMPLE_OPS) = [70, 82) of the 20-qubit
    brickwork(40)+qft(20) circuit (seed 42), after simulating ops [0, 70)
    untimed.  Returns (seconds, amplitude updates)."""
    from oracle import oracle as O
    c, _ = O.brickwork(SAMPLE_N, 40, 42, with_qft=True)
    return c.time_ops(SAMPLE_FIRST, SAMPLE_OPS, mode=O.SPARSE)


def cpu_rate(nproc):
    """30-qubit-equivalent gates/s of nproc parallel copies of the sample."""
    if nproc <= 1:
        sec, upd = cpu_sample()
        return upd / sec / 2.0 ** 30, sec
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(nproc) as pool:
        res = pool.map(cpu_sample, range(nproc))
    wall = time.time() - t0
    upd = sum(r[1] for r in res)
    slowest = max(r[0] for r in res)
    return upd / slowest / 2.0 ** 30, wall


def sample_desc(cores):
    return (f"reference algorithm (sparse Map + 1e-14 pruning, restated in C++: oracle/ket_oracle.cpp) on ops "
            f"[{SAMPLE_FIRST},{SAMPLE_FIRST + SAMPLE_OPS}) of the {SAMPLE_N}-qubit brickwork(40)+qft({SAMPLE_N}) "
            f"circuit, seed 42, {cores} process(es); rate = amplitude updates/s / 2^30")


def run_reference(args):
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_rate(cores)
    vals = []
    t0 = time.time()
    for _ in range(args.steps):
        v, _w = cpu_rate(cores)
        vals.append(v)
    wall = time.time() - t0
    value = statistics.mean(vals)
    line = {
        "impl": "reference",
        "metric": "30q gates/s",
        "value": value,
        "unit": "gates/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "30-qubit brickwork(40 layers)+qft(30), seed 42, complex128; reference sampled at "
                               f"{SAMPLE_N} qubits", "qubits": args.qubits},
        "cpu_baseline": {"value": value, "unit": "gates/s", "cores": cores, "kind": "port",
                         "sample": sample_desc(cores)},
        "e2e": {"value": value, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm
def run_ket(args):
    world, rank, local = dist_env()
    os.environ["KET_DEVICE"] = str(local)
    dist = Dist(world, rank, local)
    import ctypes as C

    import numpy as np

    from ket_b200 import _lib, workloads as W
    from ket_b200.circuit import DeviceState, flatten_ops, ops_to_abi

    n = args.qubits
    circ, idx = W.brickwork_qft(n, args.layers, 42)
    arr, mats, k = ops_to_abi(flatten_ops(circ.ops))
    L = _lib.lib()
    ctx = _lib.default_ctx()
    st = DeviceState(n)
    prune = bool(args.prune)
    marg_q = list(range(10))
    idx_arr = np.array(idx, dtype=np.uint64)

    def step():
        st.set_basis(0)
        st.apply_abi(arr, mats, k, prune=prune, specialize=args.specialize, reg_bits=args.reg_bits,
                     stage=args.stage)
        a = st.amplitudes(idx_arr)
        md = st.marginal_dist(marg_q)
        return a, md

    # cold call: the first run of this circuit shape in the process, through
    # the default policy (ready compiled kernels, interpreter otherwise, missing
    # kernels compiled in the background) -- what a user's first run() sees
    cold = None
    if not args.no_extras:
        torch_sync = __import__("torch").cuda.synchronize
        torch_sync()
        t = time.perf_counter()
        st.set_basis(0)
        st.apply_abi(arr, mats, k, prune=prune, specialize=0, reg_bits=args.reg_bits, stage=args.stage)
        st.amplitudes(idx_arr)
        st.marginal_dist(marg_q)
        torch_sync()
        cold = time.perf_counter() - t
    tw = time.perf_counter()
    jit_note = None
    for w in range(args.warmup):
        try:
            step()
        except Exception as e:  # no runtime compiler on this host: the interpreter runs every pass
            if args.specialize != 1 or w:
                raise
            jit_note = f"compiled pass kernels unavailable ({e}); interpreter"
            print(jit_note, file=sys.stderr)
            args.specialize = -1
            step()
    warm_s = time.perf_counter() - tw
    jst, jcs = (C.c_int64 * 4)(), C.c_double()
    _lib.check(L.ket_jit_stats(jst, C.byref(jcs)))
    jit0 = list(jst)

    def counters():
        lc = C.c_uint64()
        h2d, d2h = C.c_uint64(), C.c_uint64()
        L.ket_ctx_launch_count(ctx, C.byref(lc))
        L.ket_ctx_io_bytes(ctx, C.byref(h2d), C.byref(d2h))
        return lc.value, h2d.value, d2h.value

    import torch
    sp = C.c_void_p()
    _lib.check(L.ket_ctx_stream(ctx, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value, device=torch.device("cuda", local))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    L.ket_ctx_profile(ctx, 1)
    clocks = ClockSampler(local)
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    c0 = counters()
    t0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    dist.barrier()
    c1 = counters()
    clk = clocks.stop()
    cnt = C.c_size_t()
    cap = 1 << 20
    kinds = (C.c_int * cap)()
    ms = (C.c_float * cap)()
    _lib.check(L.ket_ctx_profile_read(ctx, kinds, ms, cap, C.byref(cnt)))
    kinds_all, ms_all = list(kinds[: cnt.value]), list(ms[: cnt.value])
    L.ket_ctx_profile(ctx, 0)

    _lib.check(L.ket_jit_stats(jst, C.byref(jcs)))
    jit_launches = jst[3] - jit0[3]
    dev_s = ev0.elapsed_time(ev1) / 1e3
    dev_max = dist.max(dev_s)
    wall_max = dist.max(wall)
    busy_s = sum(ms_all) / 1e3
    gates_total = k * args.steps * world
    value = gates_total / dev_max
    e2e = gates_total / wall_max
    fused = [t for kd, t in zip(kinds_all, ms_all) if kd == 0]
    peak, peak_kind = hbm_peak()
    bytes_per_launch = 2 * 16 * 2.0 ** n
    achieved = bytes_per_launch / (statistics.mean(fused) / 1e3) / 1e9 if fused else None
    passes_per_step = len(fused) / args.steps if fused else 0
    line = {
        "metric": "30q gates/s",
        "value": value,
        "unit": "gates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_max / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c128 (f64)",
        "data": "synthetic",
        "config": {"workload": f"{n}-qubit brickwork({args.layers} layers)+qft({n}), seed 42, complex128, "
                               "outputs 1024 amplitudes + q0-q9 marginals",
                   "qubits": n, "gates_per_step": k, "fused_passes_per_step": passes_per_step,
                   "pruning": "reference (|a|^2<1e-14 flushed per gate)" if prune else "off (plain dense)",
                   "l2_flush": "not needed: 16 GiB state > 126 MB L2",
                   "parallelism": f"replicas x{world}",
                   "kernel_busy_ms_per_step": busy_s / args.steps * 1e3,
                   "pass_kernels": (f"compiled per pass program at run time ({jit_launches} of {len(fused)} "
                                    f"timed passes; {jst[1]} kernels compiled during warm-up in {warm_s:.1f} s "
                                    f"wall, cached by program shape, matrices read at run time)")
                   if jit_launches else (jit_note or "interpreter (k_fused2)")},
        "e2e": {"value": e2e, "unit": "gates/s", "h2d_bytes_per_step": (c1[1] - c0[1]) // args.steps,
                "d2h_bytes_per_step": (c1[2] - c0[2]) // args.steps},
        "gpu_launches": c1[0] - c0[0],
        "cold_call": ({"seconds": cold, "gates_per_s": k / cold,
                       "policy": "first run of the shape: default policy (interpreter where no compiled kernel is "
                                 "ready, compiles queued in the background)"} if cold else None),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                     "traffic": ncu_traffic(n),
                     "kernel": "ket_pass (register-tiled fused pass compiled per program)" if jit_launches
                     else "k_fused2 (register-tiled fused pass)",
                     "bytes_per_launch": bytes_per_launch},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, _ = cpu_rate(1)
        line["cpu_baseline"] = {"value": v, "unit": "gates/s", "cores": 1, "kind": "port", "sample": sample_desc(1)}
    if world == 1 and not args.no_extras and n == 30:
        del st
        line.update(extras())
    dist.close()
    if rank == 0:
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- other workloads of the metric
def extras():
    """The other measurements the headline metric names, each on its own
    synthetic workload, each with the roofline that bounds it:
      config1_16q  the reference's own size: exactProbs + 4096 shots of the
                   16-qubit brickwork(20) through the Circuit API, end to end,
                   beside the reference algorithm on one core and the dense
                   CPU oracle on every core
      vqe24        adjoint gradients of the 24-qubit TFIM VQE (8 layers of Ry,
                   Rz and a CNOT ladder, 384 parameters), 64 parameter vectors,
                   against the reference's parameter-shift rule on the same engine
      qaoa_batch   4096 QAOA MaxCut instances (3-regular graphs, n in 10..22
                   even, p = 4) in one persistent launch
      vqe_batch    1024 vqe() energies of hardware-efficient ansatze on 8..13
                   qubits (4 layers, TFIM) in one persistent launch
      precision    complex64 against complex128 at 31 qubits (brickwork, 30
                   layers) and the complex64 33-qubit run of the same family
      cpu_dense    the dense FP64 CPU oracle (OpenMP, every host core) on the
                   16q and 20q members of the workload family
      pershot      run()'s per-shot path: 65536 noisy shots (aria-1) of a
                   12-qubit brickwork with a mid-circuit measure and reset
      json         loading the 30-qubit workload's circuit JSON
      dm           density matrices with aria-1 noise (8 and 12 qubits)
    Device times come from CUDA events the context records around each of its
    kernels (ket_ctx_profile); wall-clock figures are through the public API."""
    out = {}
    fp64 = measured_fp64()
    out["fp64_fma_per_s"] = fp64
    for name, fn in (("config1_16q", config1_measure), ("vqe24", vqe24_measure),
                     ("qaoa_batch", lambda: qaoa_measure(fp64)), ("vqe_batch", lambda: vqe_batch_measure(fp64)),
                     ("precision", precision_measure), ("cpu_dense", cpu_dense_measure),
                     ("pershot", pershot_measure), ("json", json_measure), ("dm", dm_measure)):
        try:
            out[name] = fn()
        except Exception as e:  # one failed extra does not drop the headline line
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def measured_fp64():
    import ctypes as C
    from ket_b200 import _lib
    r = C.c_double()
    _lib.check(_lib.lib().ket_measure_fp64(_lib.default_ctx(), C.byref(r)))
    return r.value


class Profiled:
    """Per-kernel CUDA-event times (kind, ms) of the context's launches inside
    the block."""

    def __enter__(self):
        from ket_b200 import _lib
        self.L, self.ctx = _lib.lib(), _lib.default_ctx()
        self._read()  # drop earlier records
        self.L.ket_ctx_profile(self.ctx, 1)
        return self

    def _read(self):
        import ctypes as C
        cnt = C.c_size_t()
        cap = 1 << 20
        kinds = (C.c_int * cap)()
        ms = (C.c_float * cap)()
        self.L.ket_ctx_profile_read(self.ctx, kinds, ms, cap, C.byref(cnt))
        return list(kinds[: cnt.value]), list(ms[: cnt.value])

    def __exit__(self, *exc):
        self.kinds, self.ms = self._read()
        self.L.ket_ctx_profile(self.ctx, 0)
        return False

    def busy_ms(self, kinds=None):
        return sum(t for k, t in zip(self.kinds, self.ms) if kinds is None or k in kinds)

    def launches(self, kinds=None):
        return sum(1 for k in self.kinds if kinds is None or k in kinds)


def config1_measure():
    """exactProbs + 4096 shots of brickwork(16, 20), seed 42 (the reference's
    own size), end to end through the Circuit API on a fresh circuit object
    each repeat; beside the reference algorithm (sparse oracle) on one core
    and the dense oracle on every core, and the reference's published
    qft(16) statevector() time on a 2-core CI runner (161 ms)."""
    from ket_b200 import workloads as W
    reps = 10
    c, _ = W.brickwork_circuit(16, 20, 42)
    c.exactProbs()
    c.run(shots=4096, seed=42)
    circs = [W.brickwork_circuit(16, 20, 42)[0] for _ in range(reps)]  # built untimed, as the oracle's is
    t = time.perf_counter()
    for c in circs:
        probs = c.exactProbs()
        c.run(shots=4096, seed=42)
    t_gpu = (time.perf_counter() - t) / reps
    with Profiled() as pf:
        c.exactProbs()
        c.run(shots=4096, seed=42)
    res = {"gates": len(c.ops), "keys": len(probs), "engine_ms": t_gpu * 1e3,
           "engine_kernel_ms": pf.busy_ms(), "engine_launches": pf.launches(),
           "reference_published_qft16_ms": 161.0,
           "unit": "ms per exactProbs() + run(4096 shots) (wall clock)",
           "roofline": "latency / launch bound: the 1 MiB state lives in L2"}
    try:
        from oracle import oracle as O
        oc, _ = O.brickwork(16, 20, 42)
        t = time.perf_counter()
        st = oc.simulate(mode=O.SPARSE)
        st.exact_probs()
        st.run(4096, 42)
        res["oracle_sparse_1core_ms"] = (time.perf_counter() - t) * 1e3
        t = time.perf_counter()
        st = oc.simulate(mode=O.DENSE)
        res["oracle_dense_allcores_simulate_ms"] = (time.perf_counter() - t) * 1e3
        res["host_cores"] = os.cpu_count()
    except Exception as e:
        res["oracle"] = f"unavailable: {e}"
    return res


def vqe24_measure():
    import numpy as np
    from ket_b200 import workloads as W
    from ket_b200.adjoint import adjoint_gradient, shift_gradient
    ans, H, P = W.tfim_vqe(24, 8, 64)
    P = np.array(P)
    adjoint_gradient(ans, H, P[:8])  # a batch of 8 compiles the pass kernels the timed batch reuses
    with Profiled() as pf:
        t = time.perf_counter()
        e, g = adjoint_gradient(ans, H, P)
        ta = time.perf_counter() - t
    t = time.perf_counter()
    e2, g2 = shift_gradient(ans, H, P[:1])
    ts = time.perf_counter() - t
    B = len(P)
    busy = pf.busy_ms()
    peak, _ = hbm_peak()
    # one read and one write of the 2^25-amplitude psi|lambda state
    pass_bytes = 2 * 16 * 2.0 ** 25
    return {"adjoint_grads_per_s": B / ta, "shift_grads_per_s": 1.0 / ts, "speedup": ts / (ta / B),
            "max_abs_grad_diff": float(np.max(np.abs(g2[0] - g[0]))), "params": int(P.shape[1]), "batch": B,
            "adjoint_ms_per_gradient_wall": ta / B * 1e3, "adjoint_kernel_ms_per_gradient": busy / B,
            "adjoint_launches_per_gradient": pf.launches() / B,
            "pass_equivalents_per_gradient_at_peak": (busy / B * 1e-3) * peak * 1e9 / pass_bytes,
            "unit": "gradients/s (wall clock); kernel ms from CUDA events"}


def qaoa_flops_bytes(n, p, tile=12):
    """FP64 flops and HBM bytes of one batch QAOA instance as k_batch_qaoa runs
    it: per layer the cost phase (a complex multiply, 6 flops per amplitude)
    and Rx on every qubit (6 flops per amplitude each), then the <C>
    reduction (3 flops per amplitude).  Instances of up to `tile` qubits live
    in shared memory (no HBM bytes); wider ones run 2p passes over HBM, the
    first writing and the last reading the state once, the others both."""
    N = 2.0 ** n
    flops = p * N * (6 + 6 * n) + 3 * N
    hbm = 0.0 if n <= tile else (2 * p - 1) * 2 * 16 * N
    return flops, hbm


def qaoa_measure(fp64):
    import numpy as np
    from ket_b200 import workloads as W
    from ket_b200.batch import batch_qaoa
    inst = W.qaoa_batch(4096, 4, 42)
    batch_qaoa(inst[:64])
    batch_qaoa(inst)
    t = time.perf_counter()
    res = batch_qaoa(inst)
    tq = time.perf_counter() - t
    with Profiled() as pf:
        batch_qaoa(inst)
    kern_s = pf.busy_ms() * 1e-3
    peak, _ = hbm_peak()
    fl = [qaoa_flops_bytes(n, len(g)) for n, _, g, _ in inst]
    sum_of_max = sum(max(f / (2 * fp64), b / (peak * 1e9)) for f, b in fl)
    max_of_sums = max(sum(f for f, _ in fl) / (2 * fp64), sum(b for _, b in fl) / (peak * 1e9))
    return {"instances": len(inst), "seconds": tq, "instances_per_s": len(inst) / tq,
            "kernel_seconds": kern_s, "mean_expected_cut": float(np.mean(res)),
            "roofline": {"bound": "fp64 (n <= 12, shared memory) / hbm (n > 12)",
                         "bound_seconds_sum_of_max": sum_of_max, "bound_seconds_max_of_sums": max_of_sums,
                         "frac": sum_of_max / kern_s, "fp64_flops": sum(f for f, _ in fl),
                         "hbm_bytes": sum(b for _, b in fl), "fp64_peak_flops": 2 * fp64, "hbm_peak_gbs": peak},
            "unit": "instances/s (wall clock); kernel seconds from CUDA events"}


def vqe_batch_measure(fp64):
    """1024 vqe() energies of hea_ladder(n, 4) + TFIM(n), n in 8..13, in one
    launch.  Roofline: FP64 flops of the gates (a 2x2 complex matrix on a pair
    is 28 flops, 14 per amplitude) and of the Pauli sums (about 12 per
    amplitude per term) at the measured FP64 rate; every state lives in shared
    memory, so HBM is not touched beyond the op lists."""
    from ket_b200 import workloads as W
    from ket_b200.batch import batch_vqe
    templates, inst = W.vqe_batch(1024)
    batch_vqe(templates, inst[:32])
    batch_vqe(templates, inst)
    t = time.perf_counter()
    e = batch_vqe(templates, inst)
    tw = time.perf_counter() - t
    with Profiled() as pf:
        batch_vqe(templates, inst)
    kern_s = pf.busy_ms() * 1e-3
    sizes = (8, 9, 10, 11, 12, 13)
    flops = 0.0
    for t_, _ in inst:
        n = sizes[t_]
        N = 2.0 ** n
        layers = 4
        flops += layers * 2 * n * 14 * N + len(templates[t_][1]) * 12 * N
    bound = flops / (2 * fp64)
    try:
        from oracle import oracle as O
        checked = []
        for i in range(0, len(inst), 128):
            t_, p = inst[i]
            oc = O.ansatz(O.ANS_HEA_LADDER, sizes[t_], 4, p)
            checked.append(abs(oc.vqe([(x.coeff, x.ops) for x in templates[t_][1]]) - e[i]))
        err = max(checked)
    except Exception as ex:
        err = f"oracle unavailable: {ex}"
    return {"instances": len(inst), "seconds": tw, "energies_per_s": len(inst) / tw, "kernel_seconds": kern_s,
            "max_abs_err_vs_oracle_sample": err,
            "roofline": {"bound": "fp64", "bound_seconds": bound, "frac": bound / kern_s, "fp64_flops": flops,
                         "fp64_peak_flops": 2 * fp64},
            "unit": "energies/s (wall clock); kernel seconds from CUDA events"}


def precision_measure():
    from ket_b200 import KET_C64, workloads as W
    from ket_b200.circuit import DeviceState, flatten_ops, ops_to_abi
    c31, _ = W.brickwork_circuit(31, 30, 42)
    arr, m, k = ops_to_abi(flatten_ops(c31.ops))
    a = DeviceState(31)
    a.set_basis(0)
    a.apply_abi(arr, m, k, specialize=1)
    b = DeviceState(31, KET_C64)
    b.set_basis(0)
    b.apply_abi(arr, m, k, specialize=1)
    ov, mx = a.compare(b)
    na, nb = a.norm2(), b.norm2()
    del a, b
    c33, _ = W.brickwork_circuit(33, 30, 42)
    arr, m, k = ops_to_abi(flatten_ops(c33.ops))
    s33 = DeviceState(33, KET_C64)
    s33.set_basis(0)
    t = time.perf_counter()
    s33.apply_abi(arr, m, k, specialize=-1)
    t33 = time.perf_counter() - t
    n33 = s33.norm2()
    s33.set_basis(0)
    s33.apply_abi(arr, m, k, specialize=1)  # compiles the pass kernels, untimed
    s33.set_basis(0)
    with Profiled() as pf:
        t = time.perf_counter()
        s33.apply_abi(arr, m, k, specialize=1)
        t33c = time.perf_counter() - t
    del s33
    passes = [x for kd, x in zip(pf.kinds, pf.ms) if kd == 0]
    peak, _ = hbm_peak()
    pass_bytes = 2 * 8 * 2.0 ** 33
    gbs = pass_bytes / (sum(passes) / len(passes) * 1e-3) / 1e9 if passes else None
    return {"fidelity_31q": abs(ov) ** 2 / (na * nb), "max_abs_amp_err_31q": mx,
            "norm_c128_31q": na, "norm_c64_31q": nb, "c64_33q_seconds_interpreter": t33,
            "c64_33q_norm": n33, "c64_33q_seconds_compiled": t33c, "c64_33q_gates_per_s_compiled": k / t33c,
            "c64_33q_passes": len(passes),
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                         "frac": gbs / peak if gbs else None, "bytes_per_pass": pass_bytes}}


def cpu_dense_measure():
    """The dense FP64 CPU oracle (OpenMP on every host core) on the 16- and
    20-qubit members of the workload family: the all-core CPU baseline."""
    from oracle import oracle as O
    res = {"host_cores": os.cpu_count(), "unit": "gates/s (wall clock)"}
    for n, layers, qft in ((16, 20, False), (20, 40, True)):
        oc, _ = O.brickwork(n, layers, 42, with_qft=qft)
        t = time.perf_counter()
        oc.simulate(mode=O.DENSE)
        dt = time.perf_counter() - t
        key = f"{n}q_brickwork{layers}" + (f"_qft{n}" if qft else "")
        res[key] = {"gates": len(oc), "seconds": dt, "gates_per_s": len(oc) / dt}
    return res


def dm_measure():
    """dm() with the aria-1 noise profile: brickwork(8, 10) on the engine and
    on the oracle's restatement of runDM (the CPU checker), with the largest
    entry difference, and brickwork(12, 10) on the engine alone."""
    import numpy as np
    from ket_b200 import workloads as W
    from ket_b200.circuit import flatten_ops
    res = {"noise": "aria-1", "unit": "seconds per dm() (wall clock)"}
    for n in (8, 12):
        c, _ = W.brickwork_circuit(n, 10, 42)
        c.dm(noise="aria-1")
        t = time.perf_counter()
        d = c.dm(noise="aria-1")
        res[f"engine_{n}q_s"] = time.perf_counter() - t
        res[f"purity_{n}q"] = d.purity()
        if n == 8:
            try:
                from oracle import oracle as O
            except Exception as e:
                res["oracle"] = f"unavailable: {e}"
                continue
            oc = O.OCircuit(n)
            for op in flatten_ops(c.ops):
                oc.add(op.name, list(op.qubits), list(op.params))
            t = time.perf_counter()
            o = oc.dm(0.0003, 0.005)
            res["oracle_8q_s"] = time.perf_counter() - t
            res["max_entry_diff_8q"] = float(np.max(np.abs(d.dense() - o.dense())))
    return res

def json_measure(reps: int = 20):
    """Loading ket's circuit JSON for the 30-qubit workload (2260 gates):
    the C ABI's loader against the Python mirror's Circuit.fromJSON."""
    import ket_b200 as K
    from ket_b200 import workloads as W
    from ket_b200.circuit_json import js_stringify, program_from_json
    c, _ = W.brickwork_qft(30, 40, 42)
    text = js_stringify(c.toJSON())
    p = program_from_json(text)
    t = time.perf_counter()
    for _ in range(reps):
        p = program_from_json(text)
    tc = (time.perf_counter() - t) / reps
    t = time.perf_counter()
    K.Circuit.fromJSON(text)
    tp = time.perf_counter() - t
    return {"ops": p["count"], "bytes": len(text), "loader_ms": tc * 1e3, "loader_MB_per_s": len(text) / tc / 1e6,
            "python_mirror_ms": tp * 1e3, "unit": "ms per load (wall clock, host)"}


def pershot_measure(shots: int = 65536, sample: int = 32):
    """Shots/s of run()'s per-shot path through the public API, and the
    oracle's per-shot run (the CPU checker) on the first `sample` shots."""
    from ket_b200 import workloads as W
    from ket_b200.circuit import DEVICES, flatten_ops, make_prng
    c = W.midcircuit_brickwork(12, 10, 42)
    c.run(shots=1024, seed=1, noise="aria-1")
    t = time.perf_counter()
    dist = c.run(shots=shots, seed=7, noise="aria-1")
    tp = time.perf_counter() - t
    res = {"qubits": 12, "ops": len(c.ops), "shots": shots, "noise": "aria-1", "seconds": tp,
           "shots_per_s": shots / tp, "distinct_outcomes": len(dist.probs), "unit": "shots/s (wall clock)"}
    idx, bits, layout, _ = c.run_shots(sample, seed=7, noise="aria-1")
    try:
        from oracle import oracle as O
    except Exception as e:  # the oracle library could not be built here
        res["oracle"] = f"unavailable: {e}"
        return res
    oc = O.OCircuit(12)
    for op in flatten_ops(c.ops):
        if op.kind == "measure":
            oc.measure(op.qubits[0], layout[op.extra[0]][0] + op.extra[1])
        elif op.kind == "reset":
            oc.reset(op.qubits[0])
        else:
            oc.add(op.name, list(op.qubits), list(op.params))
    nz = DEVICES["aria-1"]["noise"]
    t = time.perf_counter()
    oidx, obits, _ = oc.run_pershot(sample, make_prng(7).state[0], nz["p1"], nz["p2"], nz["pMeas"], bits.shape[1])
    to = time.perf_counter() - t
    res["oracle_shots_per_s"] = sample / to
    res["oracle_sample_shots"] = sample
    res["sample_matches_oracle"] = bool((idx == oidx).all() and (bits == obits).all())
    return res


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ket(args)


if __name__ == "__main__":
    sys.exit(main())
