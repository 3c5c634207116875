"""Autotuner for the batched QAOA launch (ket_batch_qaoa).

The persistent batch kernel has two shape parameters: threads per CTA
(128, 256, 512) and the tile width in qubits (11 or 12).  The tile width
decides which instances run whole in shared memory and how wider ones are
split into tiled passes, and with the CTA size it sets how many CTAs share an
SM.  Which shape is fastest depends on the mix of instance sizes, so the tuner
times every candidate on the caller's own batch (graph-replayed launches,
wall clock around synchronous calls, best of `repeats`) and keeps the winner
in a small JSON cache keyed by the batch's shape: the histogram of qubit
counts, the layer count and the instance count rounded to a power of two.

Cache file: $KET_B200_CACHE/autotune.json, default ~/.cache/ket_b200/.
"""
from __future__ import annotations

import json
import os
import time
from collections import Counter
from typing import Dict, List, Optional, Sequence, Tuple

from ._lib import check, default_ctx, lib

CANDIDATES: List[Tuple[int, int]] = [(256, 12), (128, 12), (512, 12), (256, 11), (128, 11), (512, 11)]


def _cache_path() -> str:
    d = os.environ.get("KET_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "ket_b200")
    return os.path.join(d, "autotune.json")


def _load() -> Dict[str, dict]:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(cache: Dict[str, dict]) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only costs a re-tune next time


def batch_signature(instances: Sequence) -> str:
    sizes = Counter(int(inst[0]) for inst in instances)
    p = len(instances[0][2]) if instances else 0
    bucket = 1 << max(0, (len(instances) - 1).bit_length())
    hist = ",".join(f"{n}:{sizes[n] / len(instances):.2f}" for n in sorted(sizes))
    return f"qaoa|p={p}|N~{bucket}|{hist}"


def set_batch_config(block_threads: int, tile_bits: int) -> None:
    check(lib().ket_batch_config(default_ctx(), block_threads, tile_bits))


def tune_batch_qaoa(instances: Sequence, repeats: int = 2, candidates=None) -> dict:
    """Time every candidate shape on `instances`; returns and caches
    {"block_threads", "tile_bits", "seconds", "timings"}."""
    from .batch import _run
    cands = list(candidates or CANDIDATES)
    wide = max(int(inst[0]) for inst in instances)
    cands = [(nt, tb) for nt, tb in cands if wide <= 2 * tb]
    timings = {}
    for nt, tb in cands:
        set_batch_config(nt, tb)
        _run(instances, True)  # warm: allocation, capture
        best = float("inf")
        for _ in range(repeats):
            t = time.perf_counter()
            _run(instances, True)
            best = min(best, time.perf_counter() - t)
        timings[f"{nt}x{tb}"] = best
    nt, tb = min(cands, key=lambda c: timings[f"{c[0]}x{c[1]}"])
    set_batch_config(nt, tb)
    res = {"block_threads": nt, "tile_bits": tb, "seconds": timings[f"{nt}x{tb}"], "timings": timings}
    cache = _load()
    cache[batch_signature(instances)] = res
    _store(cache)
    return res


def cached_batch_config(instances: Sequence) -> Optional[dict]:
    return _load().get(batch_signature(instances))
