"""Autotuned plans: the device search runs in the library (zkg_tune_msm / zkg_tune_ntt); this
module caches its choices on disk, keyed by (device name, operation, size, group), so a process
pays for the search once per configuration.

    msm = tuned_msm(gpu, Group.G1, n, bases, scalars)   # Msm with the fastest (c, L, form, GLV)
    ntt = tuned_ntt(gpu, log_n, data)                   # Ntt with the fastest pass split

Cache: $ZK_GPU_TUNE_CACHE, else ~/.cache/zk_gpu/autotune.json.
"""
from __future__ import annotations

import ctypes
import json
import os

from ._lib import MsmTuning, check, lib
from .gpu import Buffer, Gpu
from .group import Group
from .msm import Msm
from .ntt import Ntt


def cache_path() -> str:
    return os.environ.get("ZK_GPU_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "zk_gpu",
                                                            "autotune.json"))


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(cache: dict) -> None:
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def search_msm(gpu: Gpu, group: Group, n: int, bases: Buffer, scalars: Buffer, reps: int = 2) -> list[dict]:
    """Every candidate the library timed, fastest first."""
    arr = (MsmTuning * 128)()
    count = ctypes.c_size_t()
    check(lib().zkg_tune_msm(gpu.handle, int(group), n, bases.handle, scalars.handle, reps, arr, 128,
                             ctypes.byref(count)))
    return [{"c": arr[i].c, "item_points": arr[i].item_points, "variant": arr[i].variant, "glv": arr[i].glv,
             "ms": arr[i].ms} for i in range(count.value)]


def tuned_msm(gpu: Gpu, group: Group, n: int, bases: Buffer, scalars: Buffer, reps: int = 2,
              refresh: bool = False) -> Msm:
    key = f"{gpu.adapter_name}|msm2|{int(group)}|{n}"
    cache = _load()
    if refresh or key not in cache:
        best = search_msm(gpu, group, n, bases, scalars, reps)[0]
        cache[key] = best
        _store(cache)
    p = cache[key]
    msm = Msm.for_group(gpu, group, n, p["c"], p["item_points"])
    msm.set_variant(p["variant"])
    msm.set_glv(bool(p.get("glv", 0)))
    return msm


def tuned_ntt(gpu: Gpu, log_n: int, data: Buffer, reps: int = 2, refresh: bool = False) -> Ntt:
    key = f"{gpu.adapter_name}|ntt3|{log_n}"
    cache = _load()
    if refresh or key not in cache:
        var, best, ms = ctypes.c_int(), ctypes.c_uint32(), ctypes.c_double()
        check(lib().zkg_tune_ntt(gpu.handle, log_n, data.handle, reps, ctypes.byref(var), ctypes.byref(best),
                                 ctypes.byref(ms)))
        cache[key] = {"variant": var.value, "max_stages": best.value, "ms": ms.value}
        _store(cache)
    ntt = Ntt(gpu, log_n)
    ntt.set_variant(cache[key]["variant"])
    check(lib().zkg_ntt_set_max_stages(ntt.handle, cache[key]["max_stages"]))
    return ntt
