"""Autotuner of the fluid kernel's tile shape and register budget.

The fluid pass (Scheme_U_ + sources + the Euler update) is the step's largest
kernel; its best tile (cells along k, j, i per 256-thread CTA) and resident
CTAs per SM depend on the GPU, the precision and the blocks' extents (lanes
idle at block edges that are not multiples of the tile, face fluxes per
tile, register pressure).  ``tune`` times every compiled variant on the
batch's own active solves (mhd_batch_time_fluid_tiles: the fluid pass alone,
which leaves the solves unchanged), picks the fastest and sets it; the pick
is cached per (GPU, precision, shape class) in a JSON file, so a later batch
of the same kind selects it at creation without timing.
"""
from __future__ import annotations

import json
import os

from . import capi

CACHE = os.path.join(os.path.expanduser("~"), ".cache", "mpcns_mercury_b200", "fluid_tiles.json")


def shape_class(cells) -> str:
    """Block-shape class of a batch: the median block's k and j extents, in
    buckets (a tile wastes lanes on extents that are not its multiples)."""
    ks = sorted(int(c[2]) for c in cells)
    js = sorted(int(c[1]) for c in cells)
    med = lambda v: v[len(v) // 2] if v else 0  # noqa: E731
    bucket = lambda x: "<=32" if x <= 32 else "<=64" if x <= 64 else "<=128" if x <= 128 else ">128"  # noqa: E731
    return f"k{bucket(med(ks))}-j{bucket(med(js))}"


def _gpu_name() -> str:
    try:
        import torch

        return torch.cuda.get_device_name()
    except Exception:
        return "gpu"


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def tune(batch, precision: int, cells, reps: int = 5, cache: str | None = CACHE, retune: bool = False):
    """Pick the fluid tile for `batch` (solves with steps requested); returns
    {"variant", "shape", "ms": per variant (None when cached), "default_ms",
    "cached", "key"}."""
    key = f"{_gpu_name()}|{'mixed' if precision else 'fp64'}|{shape_class(cells)}"
    table = _load(cache) if cache else {}
    if not retune and key in table:
        v = int(table[key]["variant"])
        batch.fluid_tile(v)
        return {"variant": v, "shape": capi.fluid_tile_shape(v), "ms": None, "default_ms": None, "cached": True,
                "key": key}
    ms = batch.time_fluid_tiles(reps)
    v = min(range(len(ms)), key=lambda q: ms[q])
    batch.fluid_tile(v)
    if cache:
        table[key] = {"variant": v, "shape": list(capi.fluid_tile_shape(v)), "ms": ms}
        try:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            tmp = cache + ".tmp"
            with open(tmp, "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
            os.replace(tmp, cache)
        except OSError:
            pass
    return {"variant": v, "shape": capi.fluid_tile_shape(v), "ms": ms, "default_ms": ms[0], "cached": False,
            "key": key}
