"""Launch-shape autotuner of the batched column step (lica_gpu_column_batch_steps_ex_device).

The step kernel runs one CTA per column, persistent over all the steps of a launch.  A
launch shape has two axes:
  * the CTA width -- 32, 64, 128 or 256 threads -- which also fixes how many columns share an
    SM (the 32- and 64-thread forms are bounded for 8 and 5 CTAs per SM, the wider ones run one
    or two; a one-warp CTA runs TEMP_EXTP's two phases one after the other);
  * the shared-memory cap of the Thomas arrays: as long a column as the CTAs per SM leave room
    for (the default), or none (every column's arrays in the L2-resident scratch).  Results
    are identical either way; the speed is not.
Which shape is fastest depends on the batch: many short columns favour narrow CTAs and more
columns per SM, a few long ones wide CTAs that finish each column sooner.

``tune(batch)`` times one warm-up step and ``trial_steps`` steps of each shape on a copy of
the batch's device state (the batch itself does not advance), keeps the fastest, and
caches the choice per GPU and batch shape: in memory, and in a JSON file
(``$LICA_TUNE_CACHE``, default ``~/.cache/lica_b200/column_tune.json``) so a later process
on the same GPU model skips the trial.  ``ColumnBatch.steps(threads=0)`` calls it.
"""
import json
import os
import threading

# (threads, tri_cap): tri_cap -1 = the largest the CTAs per SM allow, 0 = no shared arrays
SHAPES = ((32, -1), (64, -1), (128, -1), (256, -1), (32, 0), (64, 0), (128, 0), (256, 0))


def _name(shape):
    return f"{shape[0]}/{'smem' if shape[1] < 0 else 'scratch'}"


def _shape(entry):
    """A cache entry's shape, or None if it is not one of SHAPES."""
    try:
        sh = (int(entry["threads"]), int(entry.get("tri_cap", -1)))
    except (KeyError, TypeError, ValueError):
        return None
    return sh if sh in SHAPES else None
_lock = threading.Lock()
_memo = {}


def _cache_path():
    return os.environ.get("LICA_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "lica_b200", "column_tune.json"))


def _gpu_name(device):
    import torch
    return torch.cuda.get_device_name(device)


def batch_key(batch):
    """Shape of a batch for the cache: column count, total and longest column, and the
    column-length quartiles (the work per CTA and its spread)."""
    import numpy as np
    n = np.asarray(batch.n)
    q = np.percentile(n, [25, 50, 75]).astype(int).tolist()
    return f"ncol={batch.ncol},cells={int(n.sum())},nmax={int(n.max())},q={q[0]}/{q[1]}/{q[2]}"


def _load():
    try:
        with open(_cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(entries):
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as fh:
            json.dump(entries, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass   # a read-only home: the in-memory cache still holds the choice


def tune(batch, trial_steps=2, force=False):
    """The fastest launch shape for this batch on its GPU: ((threads, tri_cap), {shape name:
    ms per step} of the trial, or None when the choice came from the cache)."""
    import torch
    dev = batch.arrays["w"].device
    key = f"{_gpu_name(dev)}|{batch_key(batch)}"
    with _lock:
        if not force:
            if key in _memo:
                return _memo[key], None
            disk = _load()
            sh = _shape(disk[key]) if key in disk else None
            if sh is not None:
                _memo[key] = sh
                return sh, None
    times = {}
    for th, cap in SHAPES:
        trial = batch.to(dev)
        trial.steps(1, threads=th, tri_cap=cap)
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        trial.steps(trial_steps, threads=th, tri_cap=cap)
        b.record()
        torch.cuda.synchronize(dev)
        times[(th, cap)] = a.elapsed_time(b) / trial_steps
        del trial
    best = min(times, key=times.get)
    named = {_name(k): v for k, v in times.items()}
    with _lock:
        _memo[key] = best
        disk = _load()
        disk[key] = {"threads": best[0], "tri_cap": best[1], "ms_per_step": named}
        _store(disk)
    return best, named
