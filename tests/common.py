"""Helpers shared by the test files: seeded inputs in the reference's memory format, and
one-call wrappers around the GPU MSM and NTT (the reference's tests/common/mod.rs:16-72)."""
from __future__ import annotations

import json
import os

import numpy as np

from oracle import bn254, cpu
from zk_gpu import Group, Msm, xyzz_to_affine, xyzz_to_affine_g2
from zk_gpu.msm import affine_words
from zk_gpu.synthetic import uniform_scalars

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
R = bn254.R


def quick() -> bool:
    """ZK_GPU_QUICK=1 trims the largest sizes (tests/common/mod.rs:20-23)."""
    return os.environ.get("ZK_GPU_QUICK") == "1"


def rng(seed: int) -> np.random.Generator:
    return np.random.default_rng(seed)


def fr_words(values) -> np.ndarray:
    return np.array([w for v in values for w in bn254.words32(int(v) % R)], dtype=np.uint32)


def random_fr(seed: int, n: int) -> np.ndarray:
    return uniform_scalars(n, seed)


def random_points(group: str, seed: int, n: int) -> np.ndarray:
    """n uniformly random group elements [k]G (plain affine words)."""
    return cpu.generator_multiples(group, uniform_scalars(n, seed + 7919))


def msm_ref(group: str, bases: np.ndarray, scalars: np.ndarray, mont256: bool = False) -> np.ndarray:
    return cpu.msm(group, bases, scalars, mont256=mont256)


def gpu_msm(gpu, bases: np.ndarray, scalars: np.ndarray, plan=None, group: Group = Group.G1,
            variant=None, glv=None) -> np.ndarray:
    """Upload plain bases and scalars, run one MSM and return the affine result words
    (zeros = infinity). plan = None uses the defaults; (c, item_points) overrides them;
    variant selects the accumulation kernel's form; glv switches the G1 GLV split on or off."""
    n = scalars.size // 8
    base_buf = Msm.upload_bases(gpu, bases)
    scalar_buf = gpu.buffer(scalars)
    if plan is None:
        msm = Msm.for_group(gpu, group, n, Msm.default_window(n))
    else:
        msm = Msm.for_group(gpu, group, n, plan[0], plan[1])
    if variant is not None:
        msm.set_variant(variant)
    if glv is not None:
        msm.set_glv(glv)
    out = msm.run(gpu, base_buf, scalar_buf)
    words = gpu.read(out, group.xyzz_words())
    if group == Group.G1:
        return affine_words(xyzz_to_affine(words), group)
    return affine_words(xyzz_to_affine_g2(words), group)


def gpu_ntt(gpu, ntt, data: np.ndarray, inverse: bool = False) -> np.ndarray:
    buf = gpu.buffer(data)
    (ntt.inverse if inverse else ntt.forward)(gpu, buf)
    return gpu.read(buf, data.size)


def load_golden(name: str):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)["cases"]


def hex_list_words(values) -> np.ndarray:
    return np.array([w for h in values for w in bn254.hex_words(h)], dtype=np.uint32)


def golden_msm_cases():
    out = []
    for c in load_golden("msm.json"):
        bases = np.array([w for x, y in c["bases"] for w in bn254.hex_words(x) + bn254.hex_words(y)], dtype=np.uint32)
        out.append((c["name"], bases, hex_list_words(c["scalars"]), hex_list_words(c["result"])))
    return out


def golden_ntt_cases():
    return [(c["log_n"], c["direction"] == "inverse", hex_list_words(c["input"]), hex_list_words(c["output"]))
            for c in load_golden("ntt.json")]
