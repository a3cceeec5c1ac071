#!/usr/bin/env python
"""Benchmark: BN254 MSM and Fr NTT on B200, through the library's C ABI.

One step is the workload the headline metric names, with inputs resident in HBM:
    G1 MSM n = 2^24 + G1 MSM n = 2^20 (default_window, uniform scalars in [0, r),
    bases [k_i]G1 for seeded uniform k_i with 0.1% at infinity, kept in Montgomery form)
    + Fr NTT 2^24 forward then inverse (in place, natural order).
`value` is milliseconds per step (device time, CUDA events on the library's stream, max over
ranks); `e2e` is the same step through the public API with pinned host buffers: scalars and NTT
input copied host->device, MSM results and NTT outputs read back, every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's CPU path: the C restatement of zk-gpu's MSM and NTT
(oracle/, multi-threaded over every host core; the reference itself is Rust + wgpu and
cannot be built or run here) on the same step. Multi-GPU runs are independent replicas (the
MSM and NTT of one proof do not shard across GPUs here), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "zk-gpu_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

METRIC = "MSM 2^20/2^24 & NTT 2^24 ms, bit-exact; batched vs plain req/s, p50/p99 ms"
IMAD_PER_MULMOD = 264  # 8 rows x (16 product + 16 reduction multiply-adds + 1 m), field.cuh
FP64_PER_MULMOD = 170  # double-precision instructions per Fq product in limb form, field_f64.cuh
MULMODS_PER_MADD = 10  # madd-2008-s: 8M + 2S
# ncu DRAM traffic (read + write bytes) per launch. msm_accumulate_f64: captured on a G1 MSM of
# 2^22 points with the default plan (GLV split: 8.14 GB read + 0.11 GB written) and scaled by the
# entry count to 2^24 (x4); NTT forms 0, 1 and 2: the first pass captured on the 2^24 transform.
NCU_TRAFFIC = {
    "msm_accumulate_2^24": 33.0e9,
    "ntt_form0_2^24": 1.96e9,
    "ntt_form1_2^24": 2.18e9,
    "ntt_form2_2^24": 1.71e9,
}
# The pass kernel of each NTT form.
NTT_KERNEL = {0: "ntt_pass", 1: "ntt_pass_f64", 2: "ntt_pass_f64s", 3: "ntt_pass_f64s", 4: "ntt_pass_f64r4"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--log-msm", type=int, default=24, help="large MSM size (log2); 24 in the benchmark")
    ap.add_argument("--log-msm-small", type=int, default=20)
    ap.add_argument("--log-ntt", type=int, default=24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the batched-vs-plain request stream")
    ap.add_argument("--no-configs", action="store_true", help="skip the per-configuration timings")
    ap.add_argument("--serving-rates", default="1,20,60,200", help="Poisson arrival rates (req/s)")
    ap.add_argument("--serving-lanes", type=int, default=8)
    ap.add_argument("--profile-case", action="store_true",
                    help="run the small profiling case (Fq product probe, G1 MSM 2^22, Fr NTT 2^24 forward, "
                         "G2 MSM 2^20) and exit")
    ap.add_argument("--msm-form", type=int, choices=[0, 1, 2, 3, 4, 5, 6], default=None,
                    help="profiling case: G1 accumulation form (default: the plan's default)")
    ap.add_argument("--ntt-form", type=int, choices=[0, 1, 2, 3], default=None,
                    help="profiling case: NTT butterfly form (default: the plan's default)")
    ap.add_argument("--profile-parts", default="g1,ntt,g2,elementwise",
                    help="profiling case: which parts run (g1, g1_16, ntt, g2, elementwise), comma-separated; "
                         "g1_16 is three runs of a G1 MSM 2^16")
    return ap.parse_args()


def workload_name(a) -> str:
    return (f"BN254 G1 MSM n=2^{a.log_msm} + G1 MSM n=2^{a.log_msm_small} (default_window, uniform scalars in [0,r), "
            f"bases [k_i]G1 with 0.1% at infinity, resident in Montgomery form) + Fr NTT 2^{a.log_ntt} forward "
            f"then inverse (in place, natural order)")


# ---------------------------------------------------------------- distributed plumbing

class Dist:
    def __init__(self, n_gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        self.target = ids[local_rank] if local_rank < len(ids) else str(local_rank)
        self.proc = None
        # the raw samples (the JSON line carries their summary); ZKG_CLOCK_LOG_DIR chooses where
        log_dir = os.environ.get("ZKG_CLOCK_LOG_DIR") or tempfile.gettempdir()
        self.path = os.path.join(log_dir, f"clocks_rank{local_rank}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", self.target, "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons = [], [], set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(self.NAMES, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- our arm

def run_ours(a, d: Dist) -> dict | None:
    import torch

    from zk_gpu import Gpu, Group, Msm, Ntt, lib, xyzz_to_affine
    from zk_gpu._lib import StageTime, check
    from zk_gpu.msm import affine_words
    from zk_gpu.synthetic import generator_multiples, infinity_mask, uniform_scalars

    L = lib()
    torch.cuda.set_device(d.local_rank)
    gpu = Gpu(d.local_rank)
    stream = torch.cuda.ExternalStream(L.zkg_ctx_stream(gpu.handle), device=torch.device("cuda", d.local_rank))
    n24, n20, nn = 1 << a.log_msm, 1 << a.log_msm_small, 1 << a.log_ntt

    # inputs (seeded; identical on every rank: weak scaling, one replica per GPU)
    k = uniform_scalars(n24, 101).reshape(n24, 8)
    k[infinity_mask(n24, 0.001, 102)] = 0
    k = k.reshape(-1)
    bases = generator_multiples(gpu, Group.G1, k, mont256=True)  # resident proving key
    s24_host = uniform_scalars(n24, 103)
    s20_host = uniform_scalars(n20, 104)
    x_host = uniform_scalars(nn, 105)
    s24, s20, data = gpu.buffer(s24_host), gpu.buffer(s20_host), gpu.buffer(x_host)
    c24, c20 = Msm.default_window(n24), Msm.default_window(n20)
    msm24, msm20, ntt = Msm(gpu, n24, c24), Msm(gpu, n20, c20), Ntt(gpu, a.log_ntt)

    def step():
        msm24.run(gpu, bases, s24)
        msm20.run(gpu, bases, s20)  # the first 2^20 points of the same key
        ntt.forward(gpu, data)
        ntt.inverse(gpu, data)

    for _ in range(a.warmup):
        step()
    gpu.wait()
    res24 = affine_words(xyzz_to_affine(gpu.read(msm24.run(gpu, bases, s24), 32)))
    res20 = affine_words(xyzz_to_affine(gpu.read(msm20.run(gpu, bases, s20), 32)))
    round_trip = bool(np.array_equal(gpu.read(data, x_host.size), x_host))
    fwd_probe = gpu.buffer(x_host)
    ntt.forward(gpu, fwd_probe)
    ntt_fwd = gpu.read(fwd_probe, x_host.size)  # the whole forward output, checked against the CPU below
    del fwd_probe
    entries = ctypes.c_uint64()
    check(L.zkg_msm_last_entries(msm24.__dict__["_h"], ctypes.byref(entries)))

    # ---- timed region: device time of K steps
    for h in (msm24._h, msm20._h):
        check(L.zkg_msm_set_timing(h, 1))
    check(L.zkg_ntt_set_timing(ntt.handle, 1))
    clocks = ClockSampler(d.local_rank)
    clocks.start()
    time.sleep(0.4)
    d.barrier()
    torch.cuda.synchronize()
    launches0 = L.zkg_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    d.barrier()
    launches = L.zkg_launch_count() - launches0
    clk = clocks.stop()
    ms_total = e0.elapsed_time(e1)
    ms_step = d.max(ms_total / a.steps)

    def stage_times(fn, h, cap=16):
        arr = (StageTime * cap)()
        cnt, runs = ctypes.c_size_t(), ctypes.c_size_t()
        check(fn(h, arr, cap, ctypes.byref(cnt), ctypes.byref(runs)))
        return {arr[i].stage.decode(): arr[i].ms / max(runs.value, 1) for i in range(cnt.value)}, runs.value

    st24, _ = stage_times(L.zkg_msm_stage_times, msm24._h)
    st20, _ = stage_times(L.zkg_msm_stage_times, msm20._h)
    stn, nruns = stage_times(L.zkg_ntt_pass_times, ntt.handle)
    for h in (msm24._h, msm20._h):
        check(L.zkg_msm_set_timing(h, 0))
    check(L.zkg_ntt_set_timing(ntt.handle, 0))

    # ---- the same step as one batched graph launch: the two MSMs and the NTT pair on three lanes
    from zk_gpu import Batch
    batch = Batch(gpu)
    r24, r20 = gpu.empty_buffer(32), gpu.empty_buffer(32)
    batch.add_msm(msm24, bases, s24, r24, lane=0)
    batch.add_msm(msm20, bases, s20, r20, lane=1)
    batch.add_ntt(ntt, data, inverse=False, lane=2)
    batch.add_ntt(ntt, data, inverse=True, lane=2)
    batch.capture()
    for _ in range(a.warmup):
        batch.launch()
    torch.cuda.synchronize()
    d.barrier()
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record(stream)
    for _ in range(a.steps):
        batch.launch()
    b1.record(stream)
    torch.cuda.synchronize()
    batched_ms = d.max(b0.elapsed_time(b1) / a.steps)
    batched_ok = bool(np.array_equal(affine_words(xyzz_to_affine(gpu.read(r24, 32))), res24)
                      and np.array_equal(affine_words(xyzz_to_affine(gpu.read(r20, 32))), res20)
                      and np.array_equal(gpu.read(data, x_host.size), x_host))
    batch.close()

    # ---- integer-multiply pipe peak (measured here, the roofline denominator for the MSM)
    peaks = {}
    for v, name in [(0, "mad_lo"), (1, "mad_hi"), (2, "madc_chain"), (3, "fq_mulmod"), (9, "dfma"),
                    (11, "fq_mulmod_fp64")]:
        x = ctypes.c_double()
        check(L.zkg_bench_integer_pipe(gpu.handle, v, ctypes.byref(x)))
        peaks[name] = x.value
    imad_peak = max(peaks["mad_lo"], peaks["mad_hi"], peaks["madc_chain"])

    # ---- end to end through the public API with pinned host buffers
    def pinned(words: int) -> np.ndarray:
        ptr = ctypes.c_void_p()
        check(L.zkg_host_alloc(words * 4, ctypes.byref(ptr)))
        arr = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint32)), shape=(words,))
        pinned.ptrs.append(ptr)
        return arr
    pinned.ptrs = []
    p24, p20, px, pout = pinned(s24_host.size), pinned(s20_host.size), pinned(x_host.size), pinned(x_host.size)
    o24, o20 = pinned(32), pinned(32)
    p24[:], p20[:], px[:] = s24_host, s20_host, x_host

    # Queued copies on the upload and read-back streams (zkg_buf_write_async /
    # zkg_buf_read_async). The step's operations are independent, so they run smallest input
    # first: the 2^20 scalars (32 MiB) start the device while the NTT input (512 MiB) uploads;
    # the 2^24 scalars upload during the NTT pair; the NTT output (512 MiB) comes back while the
    # 2^24 MSM runs. wait=False queues the next step before this one's results are in
    # (steady-state throughput of back-to-back steps).
    def e2e_step(wait=True):
        s20.write_async(p20)
        r20 = msm20.run(gpu, bases, s20)
        gpu.read_async(r20, o20)
        data.write_async(px)
        ntt.forward(gpu, data)
        ntt.inverse(gpu, data)
        gpu.read_async(data, pout)
        s24.write_async(p24)
        r24 = msm24.run(gpu, bases, s24)
        gpu.read_async(r24, o24)
        if wait:
            gpu.wait()

    e2e_step()
    d.barrier()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        e2e_step()
    e2e_ms = d.max((time.perf_counter() - t0) * 1e3 / a.steps)
    e2e_ok = bool(np.array_equal(pout, x_host)
                  and np.array_equal(affine_words(xyzz_to_affine(o24)), res24)
                  and np.array_equal(affine_words(xyzz_to_affine(o20)), res20))
    d.barrier()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        e2e_step(wait=False)
    gpu.wait()
    e2e_pipe_ms = d.max((time.perf_counter() - t0) * 1e3 / a.steps)
    e2e_ok = e2e_ok and bool(np.array_equal(pout, x_host))
    for ptr in pinned.ptrs:
        L.zkg_host_free(ptr)

    # ---- rooflines
    acc_ms = st24.get("accumulate", float("nan"))
    acc_ops = entries.value * MULMODS_PER_MADD * IMAD_PER_MULMOD
    acc_achieved = acc_ops / (acc_ms * 1e-3)
    acc_fp64 = entries.value * MULMODS_PER_MADD * FP64_PER_MULMOD / (acc_ms * 1e-3)
    acc_variant = msm24.params()["variant"]
    n_pass = len(stn)
    ntt_pass_ms = sum(stn.values()) / max(n_pass, 1)  # mean pass duration (forward and inverse)
    ntt_bytes = 64 * nn  # each pass reads and writes 32 B per element
    ntt_products = a.log_ntt * nn // 2 - (nn - 1)  # butterflies with a twiddle other than 1
    hbm_peak = None
    try:
        hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        hbm_src = "measured"
    except Exception:
        hbm_peak, hbm_src = 6650.0, "fallback"
    ntt_gbs = ntt_bytes / (ntt_pass_ms * 1e-3) / 1e9

    out = {
        "metric": METRIC,
        "value": round(ms_step, 4),
        "unit": "ms",
        "n_gpus": d.world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": round(ms_step, 4),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32 (BN254 Fq/Fr Montgomery, 8x32-bit limbs)",
        "data": "synthetic (seeded)",
        "config": {
            "workload": workload_name(a),
            "parallelism": f"replicas x{d.world} (one full step per GPU)",
            "windows": {"msm_2^%d" % a.log_msm: c24, "msm_2^%d" % a.log_msm_small: c20},
            "msm_plans": {f"msm_2^{a.log_msm}": msm24.params(), f"msm_2^{a.log_msm_small}": msm20.params()},
            "l2": "inputs larger than L2 (2^24 MSM bases 1 GiB, scalars 512 MiB; NTT 512 MiB); no flush",
        },
        "parts_ms": {
            f"msm_g1_2^{a.log_msm}": round(sum(st24.values()), 4),
            f"msm_g1_2^{a.log_msm_small}": round(sum(st20.values()), 4),
            f"ntt_2^{a.log_ntt}_per_transform": round(sum(stn.values()), 4),
        },
        "stages_ms": {f"msm_2^{a.log_msm}": {k: round(v, 4) for k, v in st24.items()},
                      f"msm_2^{a.log_msm_small}": {k: round(v, 4) for k, v in st20.items()},
                      f"ntt_2^{a.log_ntt}": {k: round(v, 4) for k, v in stn.items()}},
        "roofline": {
            "kernel": (f"msm_accumulate_f64 (G1 MSM 2^{a.log_msm}; Fq products on the FP64 pipe)" if acc_variant >= 3
                       else f"msm_accumulate<Fq> (G1 MSM 2^{a.log_msm})"),
            "bound": "imad",
            "achieved": round(acc_achieved / 1e12, 3),
            "peak": round(imad_peak / 1e12, 3),
            "unit": "T int-mul-add/s",
            "frac": round(acc_achieved / imad_peak, 4),
            "traffic": NCU_TRAFFIC["msm_accumulate_2^24"],
            "algorithmic": f"{entries.value} nonzero digits x {MULMODS_PER_MADD} Fq products x "
                           f"{IMAD_PER_MULMOD} 32-bit multiply-adds (the integer-product equivalent of the work)",
            "peak_source": "measured in this run: best of mad.lo / mad.hi / carry-chain probes "
                           "(zkg_bench_integer_pipe)",
            "fp64_pipe": {"achieved": round(acc_fp64 / 1e12, 3), "peak": round(peaks["dfma"] / 1e12, 3),
                          "unit": "T FP64 instr/s", "frac": round(acc_fp64 / peaks["dfma"], 4),
                          "algorithmic": f"{FP64_PER_MULMOD} FP64 instructions per Fq product"},
        },
        "roofline_ntt": {
            "kernel": (f"{NTT_KERNEL.get(ntt.params()['variant'], 'ntt_pass')} (Fr NTT 2^{a.log_ntt}, {n_pass} passes, "
                       f"form {ntt.params()['variant']})"),
            "bound": "hbm",
            "achieved": round(ntt_gbs, 1),
            "peak": hbm_peak,
            "unit": "GB/s",
            "frac": round(ntt_gbs / hbm_peak, 4),
            "peak_source": hbm_src,
            "traffic": NCU_TRAFFIC.get(f"ntt_form{ntt.params()['variant']}_2^24"),
            "algorithmic": "64 B per element per pass (read + write); the first pass also reads its staged "
                           "twiddles, 40 B per element (form 2)",
            "transform_frac_of_hbm": round((ntt_bytes * n_pass / (sum(stn.values()) * 1e-3) / 1e9) / hbm_peak, 4),
            "product_rate": {
                "achieved": round(ntt_products / (sum(stn.values()) * 1e-3) / 1e9, 2),
                "peak": round(peaks["fq_mulmod_fp64"] / 1e9, 2),
                "unit": "G Fr products/s",
                "frac": round(ntt_products / (sum(stn.values()) * 1e-3) / peaks["fq_mulmod_fp64"], 4),
                "algorithmic": f"{ntt_products} twiddle products per forward transform (log2(n) n/2 butterflies "
                               "less the n - 1 with twiddle 1); peak: the measured rate of independent "
                               "double-precision-limb Montgomery products (zkg_bench_integer_pipe variant 11)",
            },
        },
        "integer_pipe_probe": {k: round(v / 1e12, 3) for k, v in peaks.items()},
        "e2e": {
            "value": round(e2e_ms, 3),
            "unit": "ms",
            "h2d_bytes_per_step": int(4 * (s24_host.size + s20_host.size + x_host.size)),
            "d2h_bytes_per_step": int(4 * (32 + 32 + x_host.size)),
            "copies": "page-locked host buffers, queued copies overlapping the kernels (smallest input first; the NTT output returns during the 2^24 MSM); one wait per step",
            "pipelined_ms": round(e2e_pipe_ms, 3),
        },
        "gpu_launches": int(launches),
        "step_batched": {"ms": round(batched_ms, 4), "lanes": 3, "graph_launches_per_step": 1,
                         "note": "the same step captured as one CUDA graph: MSM 2^24, MSM 2^20 and the NTT pair on "
                                 "independent lanes", "same_results": batched_ok},
        "clocks": clk,
        "bit_exact": {"ntt_round_trip": round_trip, "e2e_round_trip": e2e_ok},
    }
    # the per-configuration timings and the request stream are single-GPU measurements: a scaling
    # run (N > 1 replicas) reports the step alone and releases the GPUs sooner
    if not a.no_configs and d.world == 1:
        out["configs"] = run_configs(gpu, bases, stream, n24)
    if not a.no_serving and d.world == 1:
        out["serving"] = run_serving(a, gpu)
    if d.rank == 0 and d.world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"], checks = cpu_baseline(a, gpu, bases, k, s20_host, s24_host, x_host, res20, res24,
                                                   ntt_fwd)
        out["bit_exact"].update(checks)
    del msm24, msm20, ntt
    return out


# ---------------------------------------------------------------- served vs plain request stream

SERVING_KEYS = (18, 20, 21, 22)  # resident proving keys, log2 of their sizes
SERVING_K = (14, 22)             # circuit size m = 2^k, k uniform over these integers


def run_configs(gpu, bases, stream, n_max, cpu_too=True) -> dict:
    """Device time of one call at the other sizes of the benchmark configurations (outside the
    timed step; inputs resident; CUDA events on the library stream, best of three after a
    warm-up): G1 MSM 2^16..2^24 with default_window (uniform scalars, and the two skewed
    distributions at 2^24), G2 MSM 2^18..2^22 (Montgomery-2^256 upload), Fr NTT 2^16..2^26;
    for C0 (2^16) and C2 (2^18..2^22, three scalar distributions) also the autotuned plan and the
    CPU restatement of the reference's CPU path on all host threads (one call each)."""
    import torch

    from oracle import cpu
    from zk_gpu import Group, Msm, Ntt, xyzz_to_affine
    from zk_gpu.autotune import tuned_msm
    from zk_gpu.msm import affine_words
    from zk_gpu.synthetic import generator_multiples, scalar_distribution, uniform_scalars

    def device_ms(fn):
        fn()
        best = float("inf")
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return round(best, 3)

    out = {"method": "device time of one call, best of 3 after a warm-up; inputs resident in HBM; NTT hbm_gbs = "
                     "64 B per element per pass over the forward transform's time"}
    g1 = {}
    for lg in (16, 18, 20, 22, 24):
        n = 1 << lg
        if n > n_max:
            continue
        s = gpu.buffer(uniform_scalars(n, 300 + lg))
        msm = Msm(gpu, n, Msm.default_window(n))
        g1[f"2^{lg}"] = device_ms(lambda: msm.run(gpu, bases, s))  # the first n points of the key
        if lg == 24:
            for kind, seed in (("sparse", 1), ("r-1", 2)):
                sk = gpu.buffer(scalar_distribution(n, kind, 400 + seed))
                g1[f"2^{lg} {kind}"] = device_ms(lambda: msm.run(gpu, bases, sk))
                sk.free()
        msm.close()
        s.free()
    out["g1_msm_ms"] = g1
    # C0 and C2 per scalar distribution: default_window, autotuned, and the CPU port
    threads = os.cpu_count() or 1
    c2 = {"method": "one call each; GPU: device time, best of 3; autotuned: zkg_tune_msm over windows "
                    "default-2..default+2, points per thread and accumulation forms, tuned once per size on "
                    "uniform scalars; cpu: the oracle's C restatement of the reference's CPU MSM on "
                    f"{threads} host threads, one call, wall time; bit_exact: the GPU results (both plans) "
                    "equal the CPU result"}
    host_bases = gpu.read(bases, 16 * min(n_max, 1 << 22)) if cpu_too else None
    for lg in (16, 18, 20, 22):
        n = 1 << lg
        if n > n_max:
            continue
        plain = Msm(gpu, n, Msm.default_window(n))
        su = gpu.buffer(uniform_scalars(n, 1300 + lg))
        tuned = tuned_msm(gpu, Group.G1, n, bases, su, reps=1)
        su.free()
        for kind in ("uniform", "sparse", "r-1") if lg > 16 else ("uniform",):
            sh = scalar_distribution(n, kind, 1400 + lg)
            sk = gpu.buffer(sh)
            row = {"default_window": device_ms(lambda: plain.run(gpu, bases, sk)),
                   "autotuned": device_ms(lambda: tuned.run(gpu, bases, sk)), "tuned_plan": tuned.params()}
            if cpu_too:
                t0 = time.perf_counter()
                want = cpu.msm("G1", host_bases[: 16 * n], sh, mont256=True, nthreads=threads)
                row["cpu_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
                got_p = affine_words(xyzz_to_affine(gpu.read(plain.run(gpu, bases, sk), 32)))
                got_t = affine_words(xyzz_to_affine(gpu.read(tuned.run(gpu, bases, sk), 32)))
                row["bit_exact"] = bool(np.array_equal(got_p, want) and np.array_equal(got_t, want))
                row["cpu_over_gpu"] = round(row["cpu_ms"] / row["default_window"], 1)
            c2[f"2^{lg} {kind}"] = row
            sk.free()
        plain.close()
        tuned.close()
    out["g1_msm_c0_c2"] = c2
    # fixed-base tables over the resident key (one set of buckets for every window, no
    # combination): the table build once, then one call, uniform scalars
    fb = {"method": "zkg_msm_fixed_base_table once (wall time, device synchronised), then one call (device "
                    "time, best of 3); default_window; the same scalars as the default_window rows above"}
    for lg in (16, 20):
        n = 1 << lg
        if n > n_max:
            continue
        c = Msm.default_window(n)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        table = Msm.fixed_base_table(gpu, Group.G1, bases, n, c)
        gpu.wait()
        build_ms = (time.perf_counter() - t0) * 1e3
        msm = Msm(gpu, n, c)
        msm.set_fixed_base(True)
        sh = scalar_distribution(n, "uniform", 1400 + lg)
        sk = gpu.buffer(sh)
        row = {"ms": device_ms(lambda: msm.run(gpu, table, sk)), "table_build_ms": round(build_ms, 1),
               "table_bytes": int(table.words() * 4)}
        if cpu_too:
            got = affine_words(xyzz_to_affine(gpu.read(msm.run(gpu, table, sk), 32)))
            row["bit_exact"] = bool(np.array_equal(got, cpu.msm("G1", host_bases[: 16 * n], sh, mont256=True,
                                                                 nthreads=threads)))
        fb[f"2^{lg}"] = row
        msm.close()
        sk.free()
        table.free()
    out["g1_msm_fixed_base"] = fb
    g2 = {}
    n2 = 1 << 22
    b2 = generator_multiples(gpu, Group.G2, uniform_scalars(n2, 500), mont256=True)
    for lg in (18, 20, 22):
        n = 1 << lg
        s = gpu.buffer(uniform_scalars(n, 510 + lg))
        msm = Msm.for_group(gpu, Group.G2, n, Msm.default_window(n))
        g2[f"2^{lg}"] = device_ms(lambda: msm.run(gpu, b2, s))
        msm.close()
        s.free()
    b2.free()
    out["g2_msm_ms"] = g2
    nt = {}
    for lg in (16, 20, 22, 24, 26):
        x = gpu.buffer(uniform_scalars(1 << lg, 600 + lg))
        ntt = Ntt(gpu, lg)
        fwd = device_ms(lambda: ntt.forward(gpu, x))
        inv = device_ms(lambda: ntt.inverse(gpu, x))
        nt[f"2^{lg}"] = {"forward": fwd, "inverse": inv, "passes": ntt.params()["passes"],
                         "hbm_gbs": round(64 * (1 << lg) * ntt.params()["passes"] / (fwd * 1e-3) / 1e9, 1)}
        ntt.close()
        x.free()
    out["ntt_ms"] = nt
    return out


def request_device_ms(gpu, keys, pool) -> dict:
    """Summed kernel time of one Groth16-shaped request per size class k, measured alone with
    CUDA events on the library stream through the public API: three G1 MSMs and one G2 MSM on the
    smallest key that covers m, and the witness-map chain (3 inverse transforms with the coset
    shift, 2 forward transforms, the forward transform of c with the quotient, the inverse with
    the unshift); best of 3 after a warm-up."""
    import torch

    from zk_gpu import CosetShift, Group, Msm, Ntt, lib
    from oracle import bn254

    stream = torch.cuda.ExternalStream(lib().zkg_ctx_stream(gpu.handle), device=torch.device("cuda", 0))
    g = 7
    out = {}
    for k, req in sorted(pool.items()):
        m = 1 << k
        n_key, g1b, g2b = next(key for key in keys if key[0] >= m)
        m1 = Msm(gpu, m, Msm.default_window(m))
        m2 = Msm.for_group(gpu, Group.G2, m, Msm.default_window(m))
        g1_host = [req.g1[j].array.copy() for j in range(3)]
        for j in range(3):
            g1_host[j][8 * req.g1_counts[j]:] = 0  # the server zeroes the tail of a shorter vector too
        s1 = [gpu.buffer(h) for h in g1_host]
        s2 = gpu.buffer(req.g2.array)
        polys = [gpu.buffer(req.polys[j].array) for j in range(3)]
        ntt = Ntt(gpu, k + 1)
        shift = CosetShift(gpu, k + 1, g)
        unshift = CosetShift(gpu, k + 1, pow(g, bn254.R - 2, bn254.R))

        def chain():
            for j in range(3):
                m1.run(gpu, g1b, s1[j])
            m2.run(gpu, g2b, s2)
            for j in range(3):
                ntt.inverse_coset(gpu, polys[j], shift)
            ntt.forward(gpu, polys[0])
            ntt.forward(gpu, polys[1])
            ntt.forward_quotient(gpu, polys[2], polys[0], polys[1], g)
            ntt.inverse_coset(gpu, polys[2], unshift)

        chain()
        best = float("inf")
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            chain()
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        out[k] = best
        for b in s1 + [s2] + polys:
            b.free()
        for o in (m1, m2, ntt, shift, unshift):
            o.close()
    return out


def run_serving(a, gpu) -> dict:
    """The Groth16-shaped stream through the plain server (one request at a time, operations
    launched one by one) and the served one (lanes, graphs, continuous batching, HBM-budget
    admission), same requests, same Poisson arrival times per rate."""
    from zk_gpu import Group
    from zk_gpu.serving import ProofInputs, Server, run_stream
    from zk_gpu.synthetic import generator_multiples, uniform_scalars

    keys = []
    for lk in SERVING_KEYS:
        n = 1 << lk
        g1 = generator_multiples(gpu, Group.G1, uniform_scalars(n, 700 + lk), mont256=True)
        g2 = generator_multiples(gpu, Group.G2, uniform_scalars(n, 800 + lk), mont256=True)
        keys.append((n, g1, g2))
    # one input set per circuit size, reused by every request of that size
    pool = {}
    for k in range(SERVING_K[0], SERVING_K[1] + 1):
        m = 1 << k
        req = ProofInputs(k)
        g1 = [uniform_scalars(m, 900 + 3 * k + j) for j in range(3)]
        g1[2] = g1[2][: 8 * (m - 1024)]
        polys = [uniform_scalars(2 * m, 950 + 3 * k + j) for j in range(3)]
        pool[k] = req.fill(g1, uniform_scalars(m, 990 + k), polys)
    kernel_ms = request_device_ms(gpu, keys, pool)
    rates = [float(r) for r in a.serving_rates.split(",") if r]
    out = {"workload": "Groth16-shaped requests: m = 2^k, k uniform in {14..22}; 3 G1 MSMs (m, m, m-1024) + "
                       "1 G2 MSM (m) on resident keys 2^18/2^20/2^21/2^22 + 7 Fr NTTs of 2m with coset shifts "
                       "and the quotient; Poisson arrivals",
           "lanes": a.serving_lanes, "points": []}
    servers = {}
    for mode in ("plain", "batched"):
        sv = Server(gpu, lanes=a.serving_lanes, plain=(mode == "plain"))
        for n, g1, g2 in keys:
            sv.add_key(n, g1, g2)
        # warm every size class once (slot creation, graph capture) outside the timing; the
        # served mode runs several requests of one size at once, so it keeps three slots per size
        # ready (more are made on its builder thread when a stream needs them)
        for k in sorted(pool):
            sv.wait(sv.submit(pool[k]))
            if mode == "batched":
                sv.reserve(k, 3)
        servers[mode] = sv
    for rate in rates:
        rng = np.random.default_rng(int(rate * 1000) + 17)
        count = int(max(18, min(72, rate * 3)))
        ks = rng.integers(SERVING_K[0], SERVING_K[1] + 1, size=count)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=count))
        point = {"rate_req_per_s": rate, "requests": count}
        for mode in ("plain", "batched"):
            st0 = servers[mode].stats()
            r = run_stream(servers[mode], [pool[int(k)] for k in ks], arrivals)
            st1 = servers[mode].stats()
            point[mode] = {key: round(v, 3) for key, v in r.items() if key != "requests"}
            point[mode]["slots_made"] = st1["slots_created"] - st0["slots_created"]
            # device-busy fraction: the requests' summed kernel time (each measured alone) over
            # the stream's wall time; near 1, no schedule can serve the mix faster
            point[mode]["device_busy_frac"] = round(sum(kernel_ms[int(k)] for k in ks) / (r["wall_s"] * 1e3), 3)
            point[mode]["slot_build_ms"] = round(st1["build_ms"] - st0["build_ms"], 1)
        point["throughput_ratio"] = round(point["batched"]["req_per_s"] / point["plain"]["req_per_s"], 3)
        out["points"].append(point)
    for sv in servers.values():
        sv.close()
    out["request_kernel_ms"] = {f"k={k}": round(v, 3) for k, v in sorted(kernel_ms.items())}
    out["device_bound_req_per_s"] = round(1e3 * len(kernel_ms) / sum(kernel_ms.values()), 2)
    top = out["points"][-1]
    out["max_rate_ratio"] = top["throughput_ratio"]
    return out


# ---------------------------------------------------------------- CPU side (the oracle: baseline only)

def cpu_step(bases_m256, s24, s20, x, threads):
    """One step of the workload on the host cores with the C restatement of the reference's CPU
    path. Returns (seconds per part, results)."""
    from oracle import cpu

    t = {}
    t0 = time.perf_counter()
    r24 = cpu.msm("G1", bases_m256, s24, mont256=True, nthreads=threads)
    t["msm_2^24"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    r20 = cpu.msm("G1", bases_m256[: s20.size * 2], s20, mont256=True, nthreads=threads)
    t["msm_2^20"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    y = cpu.ntt(x, False, threads)
    t["ntt_fwd"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    cpu.ntt(y, True, threads)
    t["ntt_inv"] = time.perf_counter() - t0
    return t, (r24, r20, y)


def cpu_baseline(a, gpu, bases, k, s20, s24, x, res20, res24, ntt_fwd):
    from oracle import cpu

    threads = os.cpu_count() or 1
    bases_m256 = gpu.read(bases, 16 * (1 << a.log_msm))
    t, (r24, r20, y) = cpu_step(bases_m256, s24, s20, x, threads)
    total = sum(t.values())
    checks = {
        f"msm_2^{a.log_msm}_vs_cpu": bool(np.array_equal(r24, res24)),
        f"msm_2^{a.log_msm_small}_vs_cpu": bool(np.array_equal(r20, res20)),
        f"ntt_2^{a.log_ntt}_vs_cpu": bool(np.array_equal(y, ntt_fwd)),  # all 2^log_ntt outputs
    }
    return {"value": round(total * 1e3, 1), "unit": "ms", "cores": threads, "kind": "port",
            "sample": "one full step (both MSMs and the NTT pair) on the oracle's C restatement of the "
                      "reference's CPU algorithms", "parts_s": {k_: round(v, 3) for k_, v in t.items()}}, checks


def run_reference(a, d: Dist) -> dict | None:
    if d.rank != 0:
        return None
    from oracle import cpu
    from zk_gpu.synthetic import infinity_mask, uniform_scalars

    threads = os.cpu_count() or 1
    n24, n20, nn = 1 << a.log_msm, 1 << a.log_msm_small, 1 << a.log_ntt
    k = uniform_scalars(n24, 101).reshape(n24, 8)
    k[infinity_mask(n24, 0.001, 102)] = 0
    bases = cpu.generator_multiples("G1", k.reshape(-1), mont256=True, nthreads=threads)
    s24, s20, x = uniform_scalars(n24, 103), uniform_scalars(n20, 104), uniform_scalars(nn, 105)
    for _ in range(a.warmup):
        cpu_step(bases, s24, s20, x, threads)
    t0 = time.perf_counter()
    parts = []
    for _ in range(a.steps):
        t, _ = cpu_step(bases, s24, s20, x, threads)
        parts.append(t)
    ms = (time.perf_counter() - t0) * 1e3 / a.steps
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(ms, 1),
        "unit": "ms",
        "n_gpus": d.world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": round(ms, 1),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64 (BN254 Fq/Fr Montgomery, 4x64-bit limbs)",
        "data": "synthetic (seeded)",
        "config": {"workload": workload_name(a), "parallelism": "host cores (rank 0 only)"},
        "cpu_baseline": {"value": round(ms, 1), "unit": "ms", "cores": threads, "kind": "port",
                         "sample": "the full step, every step (C restatement of the reference's CPU algorithms; "
                                   "arkworks is not available here)"},
        "e2e": {"value": round(ms, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "parts_s": {key: round(statistics.mean(p[key] for p in parts), 3) for key in parts[0]},
    }


def profile_case(msm_form=None, ntt_form=None, parts="g1,ntt,g2,elementwise"):
    """The small case the ncu captures in profiles/ run: one Fq product probe launch set, one
    G1 MSM 2^22 (device-built bases, uniform scalars), one Fr NTT 2^24 forward, one G2 MSM 2^20
    (device-built bases, Montgomery-2^256 form, uniform scalars), and a coset shift and a quotient
    over 2^22 elements; `parts` selects which of them run."""
    from zk_gpu import Gpu, lib
    from zk_gpu._lib import check

    gpu = Gpu(0)
    parts = set(parts.split(","))
    if "g1" in parts:
        x = ctypes.c_double()
        check(lib().zkg_bench_integer_pipe(gpu.handle, 3, ctypes.byref(x)))
        profile_g1(gpu, msm_form)
    if "g1_16" in parts:
        profile_g1(gpu, msm_form, log_n=16, runs=3)
    if "ntt" in parts:
        profile_ntt(gpu, ntt_form)
    if "g2" in parts:
        profile_g2(gpu)
    if "elementwise" in parts:
        profile_elementwise(gpu)
    print("profile case done", flush=True)


def profile_g1(gpu, msm_form, log_n=22, runs=1):
    from zk_gpu import Group, Msm
    from zk_gpu.synthetic import generator_multiples, uniform_scalars

    n = 1 << log_n
    bases = generator_multiples(gpu, Group.G1, uniform_scalars(n, 1), mont256=True)
    s = gpu.buffer(uniform_scalars(n, 2))
    msm = Msm(gpu, n, Msm.default_window(n))
    if msm_form is not None:
        msm.set_variant(msm_form)
    for _ in range(runs):
        msm.run(gpu, bases, s)
    gpu.wait()
    msm.close()
    bases.free()
    s.free()


def profile_ntt(gpu, ntt_form):
    from zk_gpu import Ntt
    from zk_gpu.synthetic import uniform_scalars

    buf = gpu.buffer(uniform_scalars(1 << 24, 3))
    ntt = Ntt(gpu, 24)
    if ntt_form is not None:
        ntt.set_variant(ntt_form)
    ntt.forward(gpu, buf)
    gpu.wait()
    ntt.close()
    buf.free()


def profile_g2(gpu):
    from zk_gpu import Group, Msm
    from zk_gpu.synthetic import generator_multiples, uniform_scalars

    n2 = 1 << 20
    bases2 = generator_multiples(gpu, Group.G2, uniform_scalars(n2, 4), mont256=True)
    s2 = gpu.buffer(uniform_scalars(n2, 5))
    msm2 = Msm.for_group(gpu, Group.G2, n2, Msm.default_window(n2))
    msm2.run(gpu, bases2, s2)
    gpu.wait()
    msm2.close()
    bases2.free()
    s2.free()


def profile_elementwise(gpu):
    """The elementwise kernels of the witness map at 2^22: coset shift and quotient (unfused)."""
    from zk_gpu import CosetShift, quotient
    from zk_gpu.synthetic import uniform_scalars

    ln = 22
    a_, b_, c_ = (gpu.buffer(uniform_scalars(1 << ln, 6 + j)) for j in range(3))
    CosetShift(gpu, ln, 7).shift(gpu, a_)
    quotient(gpu, a_, b_, c_, ln, 7)
    gpu.wait()


def main():
    a = parse()
    if a.profile_case:
        return profile_case(a.msm_form, a.ntt_form, a.profile_parts)
    d = Dist(a.gpus)
    try:
        out = run_reference(a, d) if a.impl == "reference" else run_ours(a, d)
        if d.rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        d.close()


if __name__ == "__main__":
    main()
