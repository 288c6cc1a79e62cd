"""Autotuner of the step's launch shapes, with a JSON cache keyed by GPU, kernel and length.

Every choice gives identical results; only the time changes.  The tuned shapes are:

* the deposit tile of the cell-ordered deposits and gathers: particles per lane (4 or 8);
* the grid size (CTAs per SM) of the per-particle deposit and gather and of the run kernels;
* the lines per CTA of the y transforms of each doubled length ("lines_nl_div:<prec>:L<n>":
  the widest tile that fits, or half of it), and the rows per CTA of the x transforms
  ("r2c_nl_div", "c2r_nl_div");
* the transform engine of the z pass at doubled length 512 (the radix-8-8-8 warp engine, or
  one exchange per transform with a 16 x 32 split);
* the line-pair tile of the Green build's even/odd transforms of each doubled length
  ("sym_nl_div", tuned where the spectra are rebuilt: the refit case and the batch).

``tune`` times each candidate on the caller's own workload (the FP32 step through the C ABI,
per-kernel CUDA-event times from the context profile), keeps the fastest in the context and
writes it to the cache; ``apply`` loads the cache into a new context.  The cache file is
``$OSC_TUNE_CACHE`` or ``~/.cache/openspacecharge_b200/autotune.json``:
``{"<GPU name>": {"<key>": {"value": v, "ms": t, "tuned_on": "<workload>"}}}``.
"""
from __future__ import annotations

import json
import os
import tempfile

from .native import OPT_PARTICLE_ORDER, OPT_PROFILE, ORDER_ANY, PREC_FP32

# candidate values per key family (0 = the built-in default)
CTAS = [0, 8, 32, 128]
RUNS = [4, 8]


def cache_path(path: str | None = None) -> str:
    if path:
        return path
    env = os.environ.get("OSC_TUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "openspacecharge_b200", "autotune.json")


def load_cache(path: str | None = None) -> dict:
    try:
        with open(cache_path(path)) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(data: dict, path: str | None = None) -> str:
    """Writes the cache atomically (temporary file, then rename)."""
    p = cache_path(path)
    os.makedirs(os.path.dirname(os.path.abspath(p)), exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(os.path.abspath(p)), prefix=".autotune", suffix=".json")
    with os.fdopen(fd, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, p)
    return p


def gpu_name(device: int = 0) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def apply(ctx, device: int = 0, path: str | None = None, gpu: str | None = None) -> dict:
    """Sets every cached choice of this GPU on the context; returns {key: value}."""
    entries = load_cache(path).get(gpu or gpu_name(device), {})
    applied = {}
    for key, ent in entries.items():
        v = int(ent["value"]) if isinstance(ent, dict) else int(ent)
        ctx.set_tuning(key, v)
        applied[key] = v
    return applied


def keys_for(grid, order: int, precision: int = PREC_FP32) -> dict:
    """Tuning keys that matter for a step on this grid in this particle order, each with the
    profile labels of the kernels it changes and its candidates."""
    ny = 2 * int(grid[1])
    prec = "f32" if precision == PREC_FP32 else "f64"
    nx = 2 * int(grid[0])
    ks = {f"lines_nl_div:{prec}:L{ny}": (("fft_y_fwd", "fft_y_inv"), [1, 2]),
          f"r2c_nl_div:{prec}:L{nx}": (("fft_x_r2c",), [1, 2]),
          f"c2r_nl_div:{prec}:L{nx}": (("fft_x_c2r",), [1, 2])}
    nz2 = 2 * int(grid[2])
    ks[f"zconv_engine:{prec}:L{nz2}"] = (("fft_z_conv",), [0, 1, 2] if precision == PREC_FP32 and nz2 == 512
                                         else [0, 2])
    if order == ORDER_ANY:
        ks["deposit_ctas_per_sm"] = (("deposit_f32",), CTAS)
        ks["gather_ctas_per_sm"] = (("interp_f32",), CTAS)
    else:
        ks["deposit_run"] = (("deposit_f32_runs",), RUNS)
        ks["gather_run"] = (("interp_f32_runs",), RUNS)
        ks["deposit_runs_ctas_per_sm"] = (("deposit_f32_runs",), [0, 8, 32])
        ks["gather_runs_ctas_per_sm"] = (("interp_f32_runs",), [0, 8, 32])
    return ks


def choose(times: dict) -> int:
    """The fastest candidate; ties go to the earlier (default-first) one."""
    best = None
    for v, t in times.items():
        if best is None or t < times[best]:
            best = v
    return best


def tune(ctx, step, grid, order: int = ORDER_ANY, precision: int = PREC_FP32, device: int = 0,
         path: str | None = None, reps: int = 3, workload: str = "", save: bool = True) -> dict:
    """Times each candidate of every key (`step()` runs one step on the context), keeps the
    fastest on the context and, with `save`, in the cache.  Returns {key: (value, {cand: ms})}."""
    ctx.set_option(OPT_PARTICLE_ORDER, order)
    result = {}
    for key, (labels, cands) in keys_for(grid, order, precision).items():
        times = {}
        for v in cands:
            ctx.set_tuning(key, v)
            step()  # warm-up with this shape
            ctx.synchronize()
            ctx.set_option(OPT_PROFILE, 1)
            ctx.profile_reset()
            for _ in range(reps):
                step()
            prof = ctx.profile()
            ctx.set_option(OPT_PROFILE, 0)
            times[v] = sum(prof[l][1] for l in labels if l in prof) / reps
        best = choose(times)
        ctx.set_tuning(key, best)
        result[key] = (best, times)
    if save:
        data = load_cache(path)
        g = data.setdefault(gpu_name(device), {})
        for key, (best, times) in result.items():
            g[key] = {"value": int(best), "ms": float(times[best]), "tuned_on": workload,
                      "candidates_ms": {str(k): float(t) for k, t in times.items()}}
        save_cache(data, path)
    return result


def _tune_key_set(ctx, step, keys, labels, cands, reps):
    result = {}
    for key in keys:
        times = {}
        for v in cands:
            ctx.set_tuning(key, v)
            step()
            ctx.synchronize()
            ctx.set_option(OPT_PROFILE, 1)
            ctx.profile_reset()
            for _ in range(reps):
                step()
            prof = ctx.profile()
            ctx.set_option(OPT_PROFILE, 0)
            times[v] = sum(prof[l][1] for l in labels if l in prof) / reps
        best = choose(times)
        ctx.set_tuning(key, best)
        result[key] = (best, times)
    return result


def _save(result, device, path, workload):
    data = load_cache(path)
    g = data.setdefault(gpu_name(device), {})
    for key, (best, times) in result.items():
        g[key] = {"value": int(best), "ms": float(times[best]), "tuned_on": workload,
                  "candidates_ms": {str(k): float(t) for k, t in times.items()}}
    save_cache(data, path)


def tune_lengths(ctx, step, lengths, precision: int = PREC_FP32, device: int = 0, path: str | None = None,
                 reps: int = 2, workload: str = "", save: bool = True, green: bool = False) -> dict:
    """The y-transform tile and the z-pass engine of every doubled length in `lengths` (a
    batched step touches several), each timed over the whole step's y or z passes (the other
    lengths' passes are the same in every trial); with `green`, also the line-pair tile of the Green build's
    even/odd transforms of each length (the step must rebuild its Green spectra)."""
    prec = "f32" if precision == PREC_FP32 else "f64"
    ls = sorted(set(int(v) for v in lengths))
    result = _tune_key_set(ctx, step, [f"lines_nl_div:{prec}:L{n2}" for n2 in ls], ("fft_y_fwd", "fft_y_inv"),
                           (1, 2), reps)
    result.update(_tune_key_set(ctx, step, [f"zconv_engine:{prec}:L{n2}" for n2 in ls], ("fft_z_conv",), (0, 2),
                                reps))
    if green:
        result.update(_tune_key_set(ctx, step, [f"sym_nl_div:{prec}:L{n2}" for n2 in ls], ("green_sym_lines",),
                                    (1, 2, 4), reps))
    if save:
        _save(result, device, path, workload)
    return result


def tune_green(ctx, step, grid, precision: int = PREC_FP32, device: int = 0, path: str | None = None,
               reps: int = 2, workload: str = "", save: bool = True) -> dict:
    """The line-pair tile of the Green build's even/odd transforms of each doubled length of
    `grid`, timed with the Green cache off so that every step rebuilds the spectra (the
    refit case); the cache budget is restored afterwards."""
    from .native import OPT_GREEN_CACHE_MB
    budget = ctx.get_option(OPT_GREEN_CACHE_MB)
    ctx.set_option(OPT_GREEN_CACHE_MB, 0)
    try:
        prec = "f32" if precision == PREC_FP32 else "f64"
        ls = sorted({2 * int(v) for v in grid})
        result = _tune_key_set(ctx, step, [f"sym_nl_div:{prec}:L{n2}" for n2 in ls], ("green_sym_lines",),
                               (1, 2, 4), reps)
    finally:
        ctx.set_option(OPT_GREEN_CACHE_MB, budget)
    if save:
        _save(result, device, path, workload)
    return result
