"""Autotuner for the element loop: threads per block (the element tile: 8
Gauss-point lanes per element, so block/8 elements per tile), the
scatter-add (FP64 atomics or colour blocks) and the element kernel (one
tile per block, or persistent blocks with the next tile's gather in
flight), picked by timing each
candidate on the caller's own mesh with the device phase timers
(sma_set_timing) and cached per (precision, scheme, size bucket).

The size bucket is the element count rounded to a power of two, so a cached
choice carries over to meshes of similar size (ensemble members, refinements).
"""
from __future__ import annotations

import json
import math
import os

CANDIDATES = ((32, "atomic", "plain"), (64, "atomic", "plain"), (128, "atomic", "plain"),
              (256, "atomic", "plain"), (128, "atomic", "pipe"), (256, "atomic", "pipe"),
              (64, "color", "plain"), (256, "color", "pipe"))


def cache_path() -> str:
    root = os.environ.get("ALYA_SMA_CACHE") or os.path.join(
        os.environ.get("XDG_CACHE_HOME", os.path.expanduser("~/.cache")), "alya_sma_b200")
    return os.path.join(root, "tuning.json")


def bucket(nelem: int) -> int:
    return 1 << max(0, int(round(math.log2(max(1, nelem)))))


def _key(precision, scheme, nelem):
    return f"{precision}/{scheme}/{bucket(nelem)}"


def load_cache(path=None) -> dict:
    try:
        with open(path or cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def save_cache(d, path=None):
    path = path or cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(d, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune(prob, precision="fp32", scheme="cd", candidates=CANDIDATES, steps=20, warmup=3,
         device=0, displ=None, use_cache=True, path=None, verbose=False):
    """Return {'block': b, 'scatter': s, 'step_ms': t, 'trials': {...}} for prob.

    Each candidate runs warmup + steps explicit steps from the same initial
    state (displ, if given) with per-phase device timing; the fastest whole
    step wins."""
    from . import ExplicitSolid
    key = _key(precision, scheme, prob.nelem)
    cache = load_cache(path) if use_cache else {}
    if use_cache and key in cache:
        return cache[key]
    trials = {}
    for block, scatter, variant in candidates:
        s = ExplicitSolid(prob, precision=precision, scatter=scatter, block=block, device=device,
                          scheme=scheme, variant=variant)
        if displ is not None:
            s.set("displ", displ)
        s.step(warmup)
        s.set_timing(True)
        s.step(steps)
        t = s.timers()
        s.close()
        name = f"{block}/{scatter}/{variant}"
        trials[name] = {"step_ms": t["step"][0] / steps, "element_ms": t["element"][0] / steps}
        if verbose:
            print(f"tune {key}: {name} step {trials[name]['step_ms']:.4f} ms")
    best = min(trials, key=lambda k: trials[k]["step_ms"])
    b, sc, va = best.split("/")
    res = {"block": int(b), "scatter": sc, "variant": va, "step_ms": trials[best]["step_ms"],
           "trials": trials}
    if use_cache:
        cache = load_cache(path)
        cache[key] = res
        save_cache(cache, path)
    return res


def autotuned(prob, precision="fp32", scheme="cd", device=0, **kw):
    """An ExplicitSolid built with the tuned block size and scatter."""
    from . import ExplicitSolid
    r = tune(prob, precision=precision, scheme=scheme, device=device, **kw)
    return ExplicitSolid(prob, precision=precision, scatter=r["scatter"], block=r["block"],
                         device=device, scheme=scheme, variant=r["variant"])


def tune_buckets(prob, precision="fp32", candidates=(32, 64, 128, 256), steps=10, warmup=3, device=0,
                 displ=None, rounds=1, verbose=False):
    """Per-size-bucket element blocks for an ensemble built with
    by_size=True: coordinate descent over the buckets (problem.size_buckets),
    each bucket's candidates timed with the others at their current pick,
    the whole step timed by the device phase timers (sma_set_timing) from
    the same start.  Adjacent buckets with the same pick are merged into one
    range (each range is one launch per step), and the plan is kept only if
    it beats the library's single launch at its default block, both timed
    again from the same start (best of three).  Returns {'plan': [(bucket,
    end, block)] or [] (the single default launch), 'step_ms',
    'default_step_ms', 'trials'}."""
    from . import ExplicitSolid
    from . import problem as P
    buckets = P.size_buckets(prob)
    ends = [e for _, e in buckets]
    s = ExplicitSolid(prob, precision=precision, device=device)
    if displ is not None:
        s.set("displ", displ)
    s.step(warmup)
    ckpt_state = (s.get("displ"), s.get("veloc"), s.get("accel"), s.state, s.time)

    def timed(plan_ends, blocks):
        d, v, a, st, tm = ckpt_state
        s.set("displ", d)
        s.set("veloc", v)
        s.set("accel", a)
        s.state = st
        s.time = tm
        s.set_launch_plan(plan_ends, blocks)
        s.step(1)                                   # graphs and caches of this plan
        s.set_timing(True)
        s.step(steps)
        t = s.timers()
        s.set_timing(False)
        return t["step"][0] / steps

    default_block = 128 if len(prob.props) > 1 else 32
    pick = [default_block] * len(ends)
    trials = {}
    for _ in range(rounds):
        for r in range(len(ends)):
            best_b, best_t = pick[r], None
            for b in candidates:
                trial = list(pick)
                trial[r] = b
                ms = timed(ends, trial)
                trials[f"{buckets[r][0]}:{b}"] = ms
                if verbose:
                    print(f"bucket {buckets[r][0]} block {b}: {ms:.4f} ms/step")
                if best_t is None or ms < best_t:
                    best_b, best_t = b, ms
            pick[r] = best_b
    # merge adjacent buckets with the same block: one launch per range
    plan = []
    for r in range(len(ends)):
        if plan and plan[-1][2] == pick[r]:
            plan[-1] = (plan[-1][0], ends[r], pick[r])
        else:
            plan.append((buckets[r][0], ends[r], pick[r]))
    p_ends, p_blocks = [e for _, e, _ in plan], [b for _, _, b in plan]
    final = min(timed(p_ends, p_blocks) for _ in range(3))
    base = min(timed([], []) for _ in range(3))
    s.set_launch_plan([], [])
    s.close()
    if len(plan) == 1 and plan[0][2] == default_block or not final < base:
        plan, final = [], base
    return {"plan": plan, "step_ms": final, "default_step_ms": base, "default_block": default_block,
            "trials": trials}
