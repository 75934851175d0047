"""Autotuner of the blind-rotation launch shape.

For a key set and a batch size it times the candidate shapes (ciphertexts
per CTA, L1 prefetch of key words, persistent CTAs) with CUDA events on a
representative batch, applies the fastest to the keys and records it in a
JSON cache keyed by GPU name, parameter set and batch bucket, so later
processes apply it without timing.  Shapes change speed only, never results.
"""
from __future__ import annotations

import json
import os
import tempfile

import numpy as np
import torch

from .engine import Keys

CACHE_PATH = os.environ.get("TFHE_B200_TUNE_CACHE",
                            os.path.join(os.path.expanduser("~"), ".cache", "tfhe_b200", "tuning.json"))


def bucket(batch: int) -> int:
    """Power-of-4 batch bucket (1, 4, 16, ..., 65536 and above)."""
    b = 1
    while b * 4 <= max(1, batch) and b < 65536:
        b *= 4
    return b


def _key(keys: Keys, batch: int) -> str:
    name = torch.cuda.get_device_name(torch.cuda.current_device())
    return f"{name}|{keys.params.name}|{bucket(batch)}"


def load_cache(path: str = CACHE_PATH) -> dict:
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path: str = CACHE_PATH) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path), suffix=".tmp")
    with os.fdopen(fd, "w") as fh:
        json.dump(cache, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def candidates(keys: Keys, batch: int):
    """Shapes worth timing: the automatic shape (K = 0), the automatic K
    requested explicitly and half of it, each with prefetch auto/off/on and
    persistent on/off."""
    kmax, _, _ = keys.launch_shape(batch)
    ks = [0] + sorted({kmax, max(1, kmax // 2)}, reverse=True)
    out = []
    for k in ks:
        for pf in (-1, 0, 1):
            for pers in (1, 0):
                out.append((k, pf, pers))
    return out


def time_shape(keys: Keys, shape, a, b, lut, reps: int = 2) -> float:
    keys.set_tuning(*shape)
    keys.cuboot_merge(a, b, lut)                      # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        keys.cuboot_merge(a, b, lut)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(keys: Keys, batch: int, path: str = CACHE_PATH, use_cache: bool = True, tune_batch: int = None,
             reps: int = 2, seed: int = 0):
    """Pick, apply and cache the fastest launch shape for `batch`; returns
    (shape, {shape: ms}) where shape = (ciphertexts_per_cta, prefetch,
    persistent)."""
    cache = load_cache(path) if use_cache else {}
    key = _key(keys, batch)
    if use_cache and key in cache:
        shape = tuple(cache[key]["shape"])
        keys.set_tuning(*shape)
        return shape, {}
    p = keys.params
    tb = tune_batch or min(batch, 4096)
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", torch.cuda.current_device())
    rnd = lambda shape: torch.from_numpy(rng.integers(0, 2 ** 32, size=shape, dtype=np.uint64)
                                         .astype(np.uint32).view(np.int32)).to(dev)
    a, b, lut = rnd((tb, p.n)), rnd((tb,)), rnd((1, 2, p.N))
    times = {}
    for shape in candidates(keys, tb):
        times[shape] = time_shape(keys, shape, a, b, lut, reps)
    best = min(times, key=times.get)
    keys.set_tuning(*best)
    if use_cache:
        cache[key] = {"shape": list(best), "ms": times[best], "tune_batch": tb}
        save_cache(cache, path)
    return best, times
