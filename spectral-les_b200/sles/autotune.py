"""Autotuner for the fused passes' kernel variants.

The passes are compiled in several tile geometries (``sles_plan_variant_count``
in include/sles.h): the x pass in four (tile width, tile ring or direct
loads, shared stash), the y passes in two tile widths (8 or 16 columns) and
the z pass with one or two z lines per work item (the last two on the float32
3D grids 128, 256 and 512).  All variants compute the same arithmetic
(identical results up to the compiler's floating-point contraction) and differ
only in speed, which depends on the grid size, precision, closure and scheme.
``tune(domain)`` times whole steps of the domain's own scheme with each
variant of each pass on scratch copies of the state (the domain's state is
not advanced), one pass at a time with the others at their current best
(x, then y, then z), keeps the fastest, and records the choices in a JSON
cache keyed by device, dimension, grid, precision, closure and scheme.  New
domains with a cached key pick the recorded variants up at construction
(``apply_cached``).

    from sles import autotune
    times = autotune.tune(domain)      # {pass: {variant: ms per step}}; domain now uses the fastest

The cache file is ``$SLES_TUNE_CACHE`` if set, else
``~/.cache/sles_b200/autotune.json``.
"""
from __future__ import annotations

import json
import os

import torch

from . import _native as nat

__all__ = ["tune", "apply_cached", "cache_path", "plan_key"]


def cache_path():
    return os.environ.get("SLES_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "sles_b200",
                                                             "autotune.json")


def plan_key(plan, scheme):
    """Cache key of a plan: device name, dim, n, precision, closure, scheme, parity."""
    d = plan.desc
    dev = torch.cuda.get_device_name(plan.device)
    return "%s|dim%d|n%d|%s|les%d|%s|parity%d" % (dev, d.dim, d.n, "f64" if d.dtype == nat.SLES_F64 else "f32",
                                                   d.les_model, scheme, d.parity)


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(table):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp%d" % os.getpid()
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home: the choice still applies to this plan


def apply_cached(plan, scheme):
    """Set the plan's variants from the cache; returns True if an entry existed."""
    ent = _load().get(plan_key(plan, scheme))
    if not ent:
        return False
    for p, v in ent.get("variants", {}).items():
        if 0 <= int(v) < plan.variant_count(int(p)):
            plan.set_variant(int(v), int(p))
    return True


def _step_fn(domain):
    """One step of the domain's scheme on scratch buffers (same kernels and
    launch sequence as the stepper; the domain's state is only read)."""
    plan, dt, dim = domain._plan, float(domain.dt), domain.dim
    A = domain._s_uhat.clone()
    B = torch.zeros_like(A)
    Cacc = torch.zeros_like(A)
    method = domain.method
    if method == "ETD2":
        F0, F1 = torch.zeros_like(A), torch.zeros_like(A)

        def step(primed):
            plan.stage(0, dt, A, None, F1, A, F0, None, None, nat.STAGE_PRIMED if primed else 0)
    elif method == "RK3":
        def step(primed):
            for rk in range(3):
                f = nat.STAGE_PRIMED if (primed or rk > 0) else 0
                plan.stage(rk, dt, A if rk == 0 else B, A, None, B, None, None, None, f)
            A.copy_(B)
    else:
        def step(primed):
            Cacc.copy_(A)
            for rk in range(4):
                f = nat.STAGE_RK4 | (nat.STAGE_PRIMED if (primed or rk > 0) else 0)
                plan.stage(rk, dt, A if rk == 0 else B, A, Cacc, B, None, None, None, f)
            A.copy_(B)
    return step


def tune(domain, steps=4, repeats=3, save=True, passes=nat.PASSES):
    """Time ``steps`` steps per variant (best of ``repeats``) of each pass with
    more than one variant, set the fastest on the domain's plan and record the
    choices.  Returns {pass: {variant: ms/step}} for the passes tuned."""
    plan = domain._plan
    todo = [p for p in passes if plan.variant_count(p) > 1]
    if not todo:
        return {}
    step = _step_fn(domain)
    st = torch.cuda.current_stream(plan.device)

    def time_it():
        step(False)  # first launch of this combination (attributes, occupancy query)
        best = None
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(steps):
                step(True)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            best = ms if best is None else min(best, ms)
        return best

    report = {}
    for p in todo:
        times = {}
        for v in range(plan.variant_count(p)):
            plan.set_variant(v, p)
            times[v] = time_it()
        win = min(times, key=times.get)
        plan.set_variant(win, p)
        report[p] = times
    domain._primed = None  # the workspace holds the scratch run's transforms
    if save:
        table = _load()
        table[plan_key(plan, domain.method)] = {
            "variants": {str(p): plan.get_variant(p) for p in passes if plan.variant_count(p) >= 1},
            "ms_per_step": {str(p): {str(k): round(t, 4) for k, t in tt.items()} for p, tt in report.items()}}
        _save(table)
    return report
