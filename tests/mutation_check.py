#!/usr/bin/env python3
"""Mutation check over the CUDA library: shows that the GPU test suite catches real bugs.

Test infrastructure, restating the reference's tools/mutation_check.py:21-43 for this code base:
each mutant is one small deliberate bug (a dropped carry, a wrong special case, a missing
scaling...) applied to a copy of the library's sources; the copy is built into its own
libzkg.so and the GPU tests run against it (ZKG_LIB selects the library). A mutant under which
every test still passes ("SURVIVED") points at a hole in the tests.

Every mutant changes arithmetic only: no index, bound, address or loop-exit condition, so no
mutant can make a kernel read or write outside its buffers or spin without end.

    python tests/mutation_check.py --stale              # every mutant's text occurs exactly once (CPU, seconds)
    python tests/mutation_check.py --build OUT [names]  # build the mutant libraries (CPU: nvcc cross-compiles)
    python tests/mutation_check.py --run OUT [names]    # run the GPU tests against each built library
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = "zk-gpu_b200/csrc/"

# (name, file, text to find, replacement). The text must occur exactly once in the file.
MUTANTS = [
    ("digits-carry", CSRC + "msm_kernels.cuh", "      mag = (1u << c) - v;\n      *neg = true;\n      carry = 1;",
     "      mag = (1u << c) - v;\n      *neg = true;"),
    ("digits-mask", CSRC + "msm_kernels.cuh", "  return v & ((1u << c) - 1);\n}", "  return v & ((1u << c) - 2);\n}"),
    ("combine-shift", CSRC + "msm_kernels.cuh", "for (uint32_t k = 0; k < width; k++) acc = lane_double(acc, sm);",
     "for (uint32_t k = 1; k < width; k++) acc = lane_double(acc, sm);"),
    ("glv-round", CSRC + "msm_kernels.cuh", "const uint64_t t = p[3] + (1ull << 63);", "const uint64_t t = p[3];"),
    ("glv-sign", CSRC + "msm_kernels.cuh", "    *neg = neg_d != flip;", "    *neg = neg_d;"),
    ("glv-digits-carry", CSRC + "msm_kernels.cuh", "      neg_d = true;\n      carry = 1;", "      neg_d = true;"),
    ("sort-sign", CSRC + "msm_kernels.cuh", "code = (fixed ? slot[k] : slot[k] - w * half) | (neg[k] ? 0x8000u : 0u);",
     "code = (fixed ? slot[k] : slot[k] - w * half) | 0u;"),
    ("reduce-weights", CSRC + "msm_kernels.cuh",
     "      if (!empty) run = xyzz_add(run, load_xyzz<F>(in + slot * XW));\n      tot = xyzz_add(tot, run);",
     "      tot = xyzz_add(tot, run);\n      if (!empty) run = xyzz_add(run, load_xyzz<F>(in + slot * XW));"),
    ("madd-f64-no-doubling", CSRC + "msm_f64.cuh", "    if (!e_is_zero4(r)) return false;\n    XyzzT<E> t = acc.get();",
     "    return false;\n    XyzzT<E> t = acc.get();"),
    ("madd-no-doubling", CSRC + "curve.cuh",
     "  F r = s2 - p.y;\n  if (pp.is_zero()) {\n    if (r.is_zero()) return xyzz_double_call(p);",
     "  F r = s2 - p.y;\n  if (pp.is_zero()) {\n    if (r.is_zero()) return xyzz_infinity<F>();"),
    ("add-no-doubling", CSRC + "curve.cuh",
     "  F r = s2 - s1;\n  if (pp.is_zero()) {\n    if (r.is_zero()) return xyzz_double_call(p);",
     "  F r = s2 - s1;\n  if (pp.is_zero()) {\n    if (r.is_zero()) return xyzz_infinity<F>();"),
    ("madd-no-infinity", CSRC + "curve.cuh",
     "  if (is_infinity(q)) return p;\n  if (is_infinity(p)) return Xyzz<F>{q.x, q.y, F::one(), F::one()};",
     "  if (is_infinity(p)) return Xyzz<F>{q.x, q.y, F::one(), F::one()};"),
    ("field-sub-addback", CSRC + "field.cuh", '"r"(P::P0 & borrow), "r"(P::P1 & borrow)',
     '"r"(P::P0 & borrow), "r"(P::P1 & 0u)'),
    ("field-add-reduce", CSRC + "field.cuh",
     "  // borrow = 0xffffffff when s < p: keep s; otherwise take s - p.\n  Fp<P> r;\n#pragma unroll\n"
     "  for (int i = 0; i < 8; i++) r.w[i] = (s.w[i] & borrow) | (d.w[i] & ~borrow);",
     "  // borrow = 0xffffffff when s < p: keep s; otherwise take s - p.\n  Fp<P> r;\n#pragma unroll\n"
     "  for (int i = 0; i < 8; i++) r.w[i] = s.w[i];"),
    ("fp64-carry", CSRC + "field_f64.cuh", "    const uint64_t carry = (t + kM52) >> 52;", "    const uint64_t carry = t >> 52;"),
    ("g2-mul-cross", CSRC + "field.cuh", "  r1 = Fq2T<B>{ac1 - bd1, (cr1 - ac1) - bd1};", "  r1 = Fq2T<B>{ac1 - bd1, cr1 - ac1};"),
    ("g2-sqr", CSRC + "field.cuh", "  rx = Fq2T<B>{re_x, ab_x + ab_x};", "  rx = Fq2T<B>{re_x, ab_x};"),
    ("ntt-no-scaling", CSRC + "ntt.cu", "    const int scale_flag = last && inverse;\n    size_t ev",
     "    const int scale_flag = 0;\n    size_t ev"),
    ("ntt-twiddle-op", CSRC + "ntt.cu",
     "        const FqD o0 = fqd_mul<FrLimbs>(fqd_sub<2, FrLimbs>(x[0], y[0]), w[0]);",
     "        const FqD o0 = fqd_mul<FrLimbs>(fqd_reduce<FrLimbs>(fqd_add(x[0], y[0]), kr), w[0]);"),
    ("ntt-twiddle-index", CSRC + "ntt.cu", "          const uint32_t e = b & (size - 1);\n          w[k]",
     "          const uint32_t e = (b + 1) & (size - 1);\n          w[k]"),
    ("quotient-sign", CSRC + "ntt.cu", "  return (a * b - c * one) * zinv2;", "  return (a * b + c * one) * zinv2;"),
    ("upload-mont256", CSRC + "msm.cu", "  if (!mont256) rescale(ctx, out, host::fq().r2);",
     "  rescale(ctx, out, host::fq().r2);"),
]

# The GPU tests each mutant runs: everything but the full-size, fuzz-soak and serving tests
# (ZK_GPU_QUICK trims the largest sizes); -x stops at the first failure.
TEST_ARGS = ["tests", "-m", "gpu", "-x", "-q", "-k", "not full_size and not serving and not soak"]


def selected(names):
    known = {m[0] for m in MUTANTS}
    bad = [n for n in names if n not in known]
    if bad:
        sys.exit(f"unknown mutants: {bad}")
    return [m for m in MUTANTS if not names or m[0] in names]


def stale() -> list[str]:
    """Mutants whose text no longer occurs exactly once."""
    out = []
    for name, path, old, _ in MUTANTS:
        text = open(os.path.join(ROOT, path)).read()
        if text.count(old) != 1:
            out.append(f"{name}: {path} holds the text {text.count(old)} times")
    return out


def build(out_dir: str, names) -> None:
    jobs = str(max(1, os.cpu_count() or 1))
    for name, path, old, new in selected(names):
        tree = os.path.join(out_dir, name)
        shutil.rmtree(tree, ignore_errors=True)
        shutil.copytree(os.path.join(ROOT, "zk-gpu_b200", "csrc"), os.path.join(tree, "zk-gpu_b200", "csrc"))
        shutil.copy(os.path.join(ROOT, "zk-gpu_b200", "Makefile"), os.path.join(tree, "zk-gpu_b200", "Makefile"))
        shutil.copytree(os.path.join(ROOT, "include"), os.path.join(tree, "include"))
        target = os.path.join(tree, path)
        text = open(target).read()
        if text.count(old) != 1:
            sys.exit(f"{name}: mutation text must occur exactly once in {path}")
        open(target, "w").write(text.replace(old, new))
        r = subprocess.run(["make", "-s", "-C", os.path.join(tree, "zk-gpu_b200"), "-j", jobs], capture_output=True, text=True)
        print(("built     " if r.returncode == 0 else "BUILD FAILED ") + name, flush=True)


def run(out_dir: str, names) -> list[str]:
    survived = []
    for name, *_ in selected(names):
        lib = os.path.join(out_dir, name, "zk-gpu_b200", "libzkg.so")
        if not os.path.exists(lib):
            print(f"missing   {name}: not built", flush=True)
            continue
        env = dict(os.environ, ZKG_LIB=lib, ZK_GPU_QUICK="1")
        r = subprocess.run([sys.executable, "-m", "pytest", *TEST_ARGS], cwd=ROOT, env=env, capture_output=True,
                           text=True, timeout=1800)
        if r.returncode == 0:
            survived.append(name)
            print(f"SURVIVED  {name}: no test failed", flush=True)
        else:
            failed = [ln.split(" ")[1] for ln in r.stdout.splitlines() if ln.startswith("FAILED ")]
            print(f"caught    {name}: {', '.join(failed) or r.stdout.strip().splitlines()[-1][:100]}", flush=True)
    return survived


if __name__ == "__main__":
    args = sys.argv[1:]
    if args[:1] == ["--stale"]:
        problems = stale()
        print("\n".join(problems) or f"all {len(MUTANTS)} mutants apply")
        sys.exit(1 if problems else 0)
    if len(args) < 2 or args[0] not in ("--build", "--run"):
        sys.exit(__doc__)
    if args[0] == "--build":
        build(args[1], args[2:])
    else:
        lost = run(args[1], args[2:])
        print(f"{len(lost)} survived" + (f": {', '.join(lost)}" if lost else ""))
        sys.exit(1 if lost else 0)
