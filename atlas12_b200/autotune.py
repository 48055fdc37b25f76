"""Launch-shape autotuner for the batched ATLAS12 runtime.

The batched LINOP1 and RT kernels take their grid from two knobs
(atlasgpu_batch_set_shape): LINOP1 CTAs per SM over the batch, and the
number of resident waves the RT pass's frequency groups are sized for (more
waves: shorter groups, better balance of the per-frequency cost spread, more
partial sums to reduce).  tune_batch() times each knob's candidates on the
models actually loaded (CUDA events around each kernel, one timed iteration
per candidate after a warm-up one), keeps the fastest and caches the choice
as JSON per GPU and workload, so later batches of the same shape skip the
search.  Results do not depend on the shape beyond the grouping of the
frequency sums.
"""
import json
import os

from . import _lib

LINOP_CANDIDATES = (16, 32, 64)
RT_CANDIDATES = (32, 64, 128, 256)


def cache_path():
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "atlas12_b200", "batch_shapes.json")


def _key(batch, device_name):
    return f"{device_name}|numnu={batch.waveset.size}|nlines={batch.nlines}|nrhox={batch.nrhox}|slots={batch.nslots}"


def _device_name(device):
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return f"cuda:{device}"


def _time_kernels(batch, load):
    """(LINOP1 ms, RT ms) of one iteration with every slot running."""
    ctx = batch.ctx
    load()
    batch.step(1)  # first iteration (KAPCONT) and warm-up
    ctx.enable_timing(True)
    try:
        batch.step(1)
        return ctx.kernel_ms("batch_linop"), ctx.kernel_ms("batch_rt")
    finally:
        ctx.enable_timing(False)
        batch.run(poll_every=4)


def cached_shape(batch):
    """The cached launch shape for `batch`'s GPU and workload, or None."""
    path = cache_path()
    try:
        with open(path) as f:
            entry = json.load(f).get(_key(batch, _device_name(batch.ctx.device)))
    except (OSError, ValueError):
        return None
    return tuple(entry["shape"]) if entry else None


def tune_batch(batch, params, starts, use_cache=True):
    """Choose and set the fastest launch shape for `batch` on these models
    (params [n, 4], starts: n dicts; the first nslots are loaded).  Returns
    (linop_ctas_per_sm, rt_waves, timings)."""
    key = _key(batch, _device_name(batch.ctx.device))
    path = cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        lc, rw = cache[key]["shape"]
        batch.set_shape(lc, rw)
        return lc, rw, cache[key]

    def load():
        for s in range(batch.nslots):
            teff, logg, mh, vt = params[s % len(params)]
            batch.load(s, teff, logg, vt, mh, starts[s % len(params)], max_iter=3, tol_percent=0.0)

    base_lc, base_rw = batch.shape()
    linop, rt = {}, {}
    for lc in LINOP_CANDIDATES:
        batch.set_shape(lc, base_rw)
        linop[lc] = _time_kernels(batch, load)[0]
    best_lc = min(linop, key=linop.get)
    for rw in RT_CANDIDATES:
        batch.set_shape(best_lc, rw)
        rt[rw] = _time_kernels(batch, load)[1]
    best_rw = min(rt, key=rt.get)
    batch.set_shape(best_lc, best_rw)
    entry = {"shape": [best_lc, best_rw], "linop_ms": {str(k): v for k, v in linop.items()},
             "rt_ms": {str(k): v for k, v in rt.items()}}
    if use_cache:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            cache[key] = entry
            with open(path, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
    return best_lc, best_rw, entry
