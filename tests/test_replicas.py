"""Replica plumbing of bench.py on the CPU: two gloo ranks take the barrier and
the max over ranks that the multi-GPU bench uses for its timings (the engine
itself runs one state per GPU, so replicas exchange nothing else)."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_ranks_take_max_over_ranks():
    code = textwrap.dedent(f"""
        import os, sys
        sys.path.insert(0, {ROOT!r})
        import bench
        world, rank, local = bench.dist_env()
        d = bench.Dist(world, rank, local, backend="gloo", timeout_s=60)
        d.barrier()
        m = d.max(1.5 + rank)          # rank 1 is the slow one
        d.barrier()
        d.close()
        print("MAX", rank, m)
    """)
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        out, _ = p.communicate(timeout=120)
        assert p.returncode == 0, out
        outs.append(out)
    for r, out in enumerate(outs):
        assert f"MAX {r} 2.5" in out, out


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(1, 0, 0)
    d.barrier()
    assert d.max(3.25) == 3.25
    d.close()
