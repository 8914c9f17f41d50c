"""Autotuner for launch shapes: times candidate configurations on the device and caches the
fastest per problem signature.

Tunables (the C ABI's `vp_plan_set_config` / `vp_batch_set_config`):

* single instance: the cluster-resident path (cluster size) for grids whose state fits one
  cluster, the persistent loop's band height (persist_rows), otherwise the staged step's tile
  (stage_rows x stage_threads) and the per-column
  kernel's rows per CTA;
* ensembles: rows per tile, columns per tile, threads per CTA and persistent CTAs per SM.

A candidate is scored by the device time (CUDA events, best of `repeats`) of a short forward
and adjoint run (`steps` steps, every state kept) on the problem's own mesh and equilibrium with
a seeded perturbation. Results are cached in a JSON file keyed by device name, SM count, ABI
version, dtype and problem shape, so the search runs once per machine and shape. The cache file
is `$VP_AUTOTUNE_CACHE`, else `~/.cache/warp_vp_solver_b200/autotune.json`.
"""

from __future__ import annotations

import hashlib
import json
import os
import threading
from typing import Callable, Iterable

import numpy as np

_LOCK = threading.Lock()


def default_cache_path() -> str:
    env = os.environ.get("VP_AUTOTUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "warp_vp_solver_b200", "autotune.json")


class TuneCache:
    """JSON cache {key: {"config": {...}, "ms": float, "tried": [[config, ms], ...]}}."""

    def __init__(self, path: str | None = None):
        self.path = path or default_cache_path()

    def load(self) -> dict:
        try:
            with open(self.path) as f:
                data = json.load(f)
            return data if isinstance(data, dict) else {}
        except (OSError, ValueError):
            return {}

    def get(self, key: str):
        return self.load().get(key)

    def put(self, key: str, entry: dict) -> None:
        with _LOCK:
            data = self.load()
            data[key] = entry
            d = os.path.dirname(self.path)
            if d:
                os.makedirs(d, exist_ok=True)
            tmp = f"{self.path}.{os.getpid()}.tmp"
            with open(tmp, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)


def signature(kind: str, **fields) -> str:
    """Stable cache key: kind plus sorted fields (arrays hashed)."""
    parts = [kind]
    for k in sorted(fields):
        v = fields[k]
        if isinstance(v, np.ndarray):
            v = hashlib.sha1(np.ascontiguousarray(v).tobytes()).hexdigest()[:16]
        parts.append(f"{k}={v}")
    return "|".join(parts)


def search(candidates: Iterable[dict], apply: Callable[[dict], bool], measure: Callable[[], float],
           repeats: int = 3):
    """Try each candidate: `apply` returns False when the candidate is not usable; `measure`
    returns a time in ms. Returns (best config, best ms, [(config, ms), ...])."""
    tried = []
    best, best_ms = None, float("inf")
    for cand in candidates:
        if not apply(cand):
            continue
        ms = min(measure() for _ in range(repeats))
        tried.append((dict(cand), float(ms)))
        if ms < best_ms:
            best, best_ms = dict(cand), float(ms)
    return best, best_ms, tried


def _device_fields():
    import torch

    from . import _capi
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return {"device": p.name, "sms": p.multi_processor_count, "abi": _capi.ABI_VERSION}


def _timer(fn, flush):
    import torch

    def run() -> float:
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b)
    return run


def plan_candidates(cfg: dict) -> list[dict]:
    """Candidate single-instance configurations around a plan's current one."""
    cands = []
    if cfg["cluster_size"] > 0:
        cands += [{"cluster_size": cn, "persist_rows": 0, "strip_rows": 0} for cn in (16, 8, 4, 2)]
    cands += [{"cluster_size": 0, "persist_rows": r, "strip_rows": 0} for r in (16, 8, 4)]
    cands += [{"cluster_size": 0, "persist_rows": 0, "strip_rows": r} for r in (4, 8, 16)]
    cands += [{"cluster_size": 0, "persist_rows": 0, "strip_rows": 0, "stage_rows": r, "stage_threads": c}
              for c in (256, 128) for r in (32, 16, 8, 4)]
    cands += [{"cluster_size": 0, "persist_rows": 0, "strip_rows": 0, "stage_rows": 0, "rows_per_cta": r}
              for r in (16, 8, 4)]
    return cands


def tune_plan(plan, steps: int = 8, repeats: int = 3, cache: TuneCache | None = None,
              force: bool = False) -> dict:
    """Pick the fastest launch shape for `plan` (a `plan.Plan`), apply it, and return
    {"config": ..., "ms": ..., "cached": bool}."""
    import torch

    cache = cache or TuneCache()
    key = signature("plan", nx=plan.nx, nv=plan.nv, dtype=str(plan.dtype), steps=steps,
                    **_device_fields())
    hit = None if force else cache.get(key)
    if hit is not None:
        plan.set_config(**hit["config"])
        return {"config": hit["config"], "ms": hit["ms"], "cached": True}
    dev = plan.device
    rng = np.random.default_rng(0)
    f_iv = torch.as_tensor(np.asarray(plan_feq(plan)) * (1.0 + 1e-3 * rng.standard_normal((plan.nx, plan.nv))),
                           dtype=torch.float64, device=dev)
    H = torch.as_tensor(1e-2 * rng.standard_normal(plan.nx), dtype=plan.dtype, device=dev)
    g_ee = torch.full((steps,), 1.0, dtype=plan.dtype, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    start = plan.get_config()

    def apply(c) -> bool:
        try:
            plan.set_config(**c)
            return True
        except (ValueError, NotImplementedError):
            return False

    def step():
        out = plan.forward(f_iv, H, steps, record_history=False, want_tape=True, checkpoint_every=1,
                           want_f_final=False)
        plan.backward(H, steps, out["tape"], out["every"], g_ee_hist=g_ee)

    best, ms, tried = search(plan_candidates(start), apply, _timer(step, flush), repeats)
    if best is None:
        plan.set_config(**{k: start[k] for k in ("rows_per_cta", "threads", "n_chunks", "cluster_size",
                                                   "stage_rows", "stage_threads", "persist_rows",
                                                   "strip_rows")})
        return {"config": None, "ms": None, "cached": False}
    plan.set_config(**best)
    cache.put(key, {"config": best, "ms": ms, "tried": tried})
    return {"config": best, "ms": ms, "cached": False, "tried": tried}


def plan_feq(plan) -> np.ndarray:
    """The plan's f_eq as given at construction (kept by the Python Plan)."""
    return plan.f_eq


def ensemble_candidates(cfg: dict) -> list[dict]:
    """The strip kernels first (where the ensemble qualifies for them), then tile shapes."""
    cands = []
    if cfg.get("strip", 0):
        cands.append({"strip": 1})
    for r in (8, 4, 2, 1):
        for chunk in (128, 256, 64):
            for th in (128, 256, 64):
                if th > chunk * 2:
                    continue
                cands.append({"rows_per_tile": r, "chunk_cols": chunk, "threads": th, "ctas_per_sm": 0, "strip": 0})
    return cands


def tune_ensemble(ens, steps: int = 6, repeats: int = 2, cache: TuneCache | None = None,
                  force: bool = False, max_candidates: int | None = None) -> dict:
    """Pick the fastest tile shape for an `ensemble.Ensemble`, apply it, return the choice."""
    import torch

    cache = cache or TuneCache()
    shapes = np.asarray(sorted(ens.shapes), dtype=np.int64)
    key = signature("ensemble", shapes=shapes, n=ens.n, dtype=str(ens.dtype), steps=steps,
                    **_device_fields())
    hit = None if force else cache.get(key)
    if hit is not None:
        ens.set_config(**hit["config"])
        return {"config": hit["config"], "ms": hit["ms"], "cached": True}
    dev = ens.device
    f_iv = torch.zeros(ens.total_cells, dtype=torch.float64, device=dev)
    rng = np.random.default_rng(0)
    H = torch.as_tensor(1e-2 * rng.standard_normal(ens.total_rows), dtype=ens.dtype, device=dev)
    g_ee = torch.ones(ens.n * steps, dtype=ens.dtype, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    state = {}

    def apply(c) -> bool:
        try:
            ens.set_config(**c)
            return True
        except (ValueError, NotImplementedError):
            return False

    def step():
        if "out" not in state or state.get("cfg") != ens.get_config():
            state["out"] = ens.alloc_outputs(steps, want_tape=True, want_f_final=False)
            state["cfg"] = ens.get_config()
            state["g"] = (torch.empty(ens.total_cells, dtype=ens.dtype, device=dev),
                          torch.empty(ens.total_rows, dtype=ens.dtype, device=dev))
        ens.forward_into(f_iv, H, steps, state["out"])
        ens.backward_into(H, steps, state["out"]["tape"], None, None, g_ee, *state["g"])

    cands = ensemble_candidates(ens.get_config())
    if max_candidates is not None:
        cands = cands[:max_candidates]
    best, ms, tried = search(cands, apply, _timer(step, flush), repeats)
    if best is None:
        return {"config": None, "ms": None, "cached": False}
    ens.set_config(**best)
    cache.put(key, {"config": best, "ms": ms, "tried": tried})
    return {"config": best, "ms": ms, "cached": False, "tried": tried}
