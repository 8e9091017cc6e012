"""Autotuner of the launch configuration: robots per CTA (bin count),
threads and springs per thread, and the shared-memory-vs-streamed cutover.

For a population, every compiled shape that can hold its largest robot is
tried with a few bin counts (whole waves of the GPU) and, as the streamed
alternative, one robot per CTA; when robots are too large for one CTA,
also every split over a thread-block cluster (2, 4 or 8 parts, each part
shape); each candidate runs a short burst of steps
timed with CUDA events on the context's stream.  The simulator's state and
clock are restored afterwards, the fastest candidate is applied, and the
choice is cached per population signature (robot sizes, mode, stress
tracking, time step) in a JSON file.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os

import numpy as np

from . import _lib

CACHE = os.environ.get("MB_AUTOTUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "mercury_b200", "autotune.json"))


def kernel_shapes() -> list[dict]:
    n = _lib.LIB.mb_kernel_shapes(None, 0)
    arr = (_lib.LaunchConfig * n)()
    _lib.LIB.mb_kernel_shapes(arr, n)
    return [{f: getattr(c, f) for f, _ in c._fields_} for c in arr]


def signature(batch, mode: int, track: bool, dt: float) -> str:
    h = hashlib.sha1()
    h.update(np.diff(batch.mass_offsets).astype(np.int64).tobytes())
    h.update(np.diff(batch.spring_offsets).astype(np.int64).tobytes())
    h.update(np.int64(batch.active_springs()).tobytes())
    h.update(f"{mode}/{int(track)}/{dt!r}".encode())
    return h.hexdigest()


def _load_cache() -> dict:
    try:
        with open(CACHE) as f:
            return json.load(f)
    except Exception:
        return {}


def _store_cache(d: dict) -> None:
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        tmp = CACHE + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f)
        os.replace(tmp, CACHE)
    except Exception:
        pass


def _time(sim, steps: int, track: bool) -> float:
    import torch
    st = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.run_steps(steps, track)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def tune(sim, batch, track: bool = False, steps: int = 300, use_cache: bool = True,
         sms: int | None = None, verbose: bool = False, upload=None, key: str | None = None) -> dict:
    """Picks and applies the fastest launch configuration for `batch` on
    `sim` (a Simulator whose mode, materials and time step are set).  Returns
    {"config": ..., "rate": spring-updates/s, "candidates": [...]}.
    `upload` (default: sim.set_batch(batch)) re-uploads the population after
    each configuration change -- e.g. Simulator.set_voxel_population for a
    population built on the device -- and `key` replaces the cache key."""
    import torch

    mode = ctypes.c_int()
    _lib.check(_lib.LIB.mb_get_mode(sim._ctx, ctypes.byref(mode)), sim._ctx)
    dt = sim.getDeltaT()
    upload = upload or (lambda: sim.set_batch(batch))
    key = key or signature(batch, mode.value, track, dt)
    cache = _load_cache() if use_cache else {}
    if key in cache:
        cfg = cache[key]["config"]
        sim.set_launch_config(**cfg)
        upload()
        return cache[key]

    if sms is None:
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    active = batch.active_springs()
    t0 = sim.getTotalTime()
    cands = []
    configs = []
    for shape in kernel_shapes():
        bin_options = [0] if shape["streamed"] else [0, sms, 2 * sms, 3 * sms]
        for bins in bin_options:
            configs.append(dict(threads=shape["threads"], springs_per_thread=shape["springs_per_thread"],
                                masses_per_thread=shape["masses_per_thread"], bins=bins, chunk=1000,
                                use_graph=1, streamed=shape["streamed"], cluster=0))
    from .simulator import plan
    if plan(batch, num_sms=sms)["cluster"]:
        # robots too large for one CTA: every cluster size and part shape
        for cluster in (2, 4, 8):
            for spt in (8, 10, 12):
                configs.append(dict(threads=1024, springs_per_thread=spt, masses_per_thread=2, bins=0,
                                    chunk=1000, use_graph=1, streamed=0, cluster=cluster))
    for cfg in configs:
        try:
            sim.set_launch_config(**cfg)
            upload()
        except _lib.MercuryError:
            continue
        got = sim.launch_config()
        if any(c["config"] == got for c in cands):
            continue
        sim.run_steps(min(50, steps), track)  # warm-up: module load, graph
        el = _time(sim, steps, track)
        rate = active * steps / el
        cands.append({"config": got, "rate": rate})
        if verbose:
            print(f"  {got} -> {rate:.3e} spring-updates/s", flush=True)
    if not cands:
        raise _lib.MercuryError(3, "no launch configuration holds this population")
    best = max(cands, key=lambda c: c["rate"])
    cfg = dict(best["config"])
    sim.set_launch_config(**cfg)
    upload()  # fresh state: tuning runs advanced the old one
    _lib.check(_lib.LIB.mb_set_total_time(sim._ctx, t0), sim._ctx)
    res = {"config": cfg, "rate": best["rate"], "candidates": cands}
    if use_cache:
        cache[key] = {"config": cfg, "rate": best["rate"]}
        _store_cache(cache)
    return res
