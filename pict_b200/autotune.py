"""Autotuner of the persistent Krylov launch shapes.

Tunables: the work-tile size of the Krylov kernels (cells per tile, 512..2048), the upper bound of
co-resident CTAs of a persistent launch (0 = every CTA the occupancy allows, or one CTA per SM) and
the CG recurrence (0: the reference's two-reduction order, 1: single reduction).  Each candidate is
timed on the real PISO step of the domain (CUDA events, after warm-up steps, from the same saved
state), and the fastest is applied.  Results are cached in a JSON file keyed by a signature of the
workload (dimensions, dtype, block sizes, solver settings, device), so later runs reuse them.
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os
from typing import Dict, Iterable, List, Optional

import torch

DEFAULT_TILES = (512, 1024, 2048)
DEFAULT_CAPS = (0, 1)          # 1: one CTA per SM (resolved to the SM count at tuning time)
DEFAULT_VARIANTS = (0, 1)


def workload_signature(domain, stepper_kwargs: Dict, device_name: str) -> str:
    """Stable key of a (batched) domain and its step settings."""
    sizes = sorted(tuple(int(s) for s in b.velocity.shape) for b in domain.getBlocks())
    desc = {
        "dims": domain.getSpatialDims(),
        "dtype": str(domain.getDtype()),
        "blocks": sizes,
        "settings": {k: stepper_kwargs[k] for k in sorted(stepper_kwargs)},
        "device": device_name,
    }
    return hashlib.sha1(json.dumps(desc, sort_keys=True, default=str).encode()).hexdigest()[:16]


def load_cache(path: Optional[str]) -> Dict:
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def save_cache(path: Optional[str], cache: Dict):
    if not path:
        return
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def candidates(tiles: Iterable[int] = DEFAULT_TILES, caps: Iterable[int] = DEFAULT_CAPS,
               variants: Iterable[int] = DEFAULT_VARIANTS) -> List[Dict]:
    return [dict(tile_cells=t, cap=c, cg_variant=v) for t, c, v in itertools.product(tiles, caps, variants)]


def _set_tiles(domain, tile_cells):
    domain.set_tile_cells(tile_cells)


def _time_steps(st, steps):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        st.step()
    e1.record()
    torch.cuda.synchronize()
    st.check()
    return e0.elapsed_time(e1) / steps


def autotune(domain, stepper_kwargs: Dict, cands: Optional[List[Dict]] = None, warmup: int = 2, steps: int = 3,
             cache_path: Optional[str] = None, verbose: bool = False):
    """Pick the fastest launch shape for stepping `domain` with PISOStepper(domain, **stepper_kwargs).

    Returns (best, table): the chosen candidate (already applied to the domain's tile table; pass
    ``best["p_group_size"]``, ``best["adv_group_size"]`` and ``best["cg_variant"]`` to the stepper) and
    the measured ms per step of every candidate.  The domain's block state is restored afterwards.
    """
    from .engine import PISOStepper
    dev = domain.getDevice()
    props = torch.cuda.get_device_properties(dev)
    key = workload_signature(domain, stepper_kwargs, props.name)
    cache = load_cache(cache_path)
    if key in cache:
        best = cache[key]["best"]
        _set_tiles(domain, best["tile_cells"])
        return best, cache[key]["table"]
    sms = props.multi_processor_count
    blocks = domain.getBlocks()
    saved = [(b.velocity.clone(), b.pressure.clone()) for b in blocks]
    saved_p = domain.pressureResult.clone()
    table = []
    for c in (cands or candidates()):
        for b, (v, p) in zip(blocks, saved):
            b.velocity.copy_(v)
            b.pressure.copy_(p)
        domain.pressureResult.copy_(saved_p)
        _set_tiles(domain, c["tile_cells"])
        gs = sms if c["cap"] == 1 else 0
        kw = dict(stepper_kwargs)
        kw.update(p_group_size=gs, adv_group_size=gs, cg_variant=c["cg_variant"])
        try:
            st = PISOStepper(domain, **kw)
            for _ in range(warmup):
                st.step()
            ms = _time_steps(st, steps)
        except Exception as e:  # a shape that cannot be launched (e.g. too many tiles for co-residency)
            ms = float("inf")
            if verbose:
                print("autotune: candidate %s failed: %s" % (c, e))
        row = dict(c, p_group_size=gs, adv_group_size=gs, ms_per_step=ms)
        table.append(row)
        if verbose:
            print("autotune:", row)
    for b, (v, p) in zip(blocks, saved):
        b.velocity.copy_(v)
        b.pressure.copy_(p)
    domain.pressureResult.copy_(saved_p)
    best = min(table, key=lambda r: r["ms_per_step"])
    _set_tiles(domain, best["tile_cells"])
    cache[key] = {"best": best, "table": table}
    save_cache(cache_path, cache)
    return best, table
