"""Proving-request server over zkg_server: resident proving keys, HBM-footprint admission and
continuous batching of Groth16-shaped requests (see include/zkg.h, "serving").

    server = Server(gpu, lanes=8)              # or Server(gpu, plain=True): one call at a time
    server.add_key(n, g1_bases_buf, g2_bases_buf)
    req = ProofInputs(log_m)                   # page-locked host buffers
    req.fill(g1_scalars, g2_scalars, polys)    # numpy arrays in the memory format
    rid = server.submit(req); times = server.wait(rid)
    req.points(), req.h()                      # outputs

`run_stream` submits a list of requests at given arrival times and reports throughput and
latency percentiles.
"""
from __future__ import annotations

import ctypes
import threading
import time

import numpy as np

from ._lib import ProofRequest, RequestTimes, ServerConfig, ServerStats, check, lib, vp
from .gpu import Buffer, Gpu


class PinnedWords:
    """A page-locked host array of u32 words (zkg_host_alloc)."""

    def __init__(self, words: int):
        self._p = ctypes.c_void_p()
        check(lib().zkg_host_alloc(max(words, 1) * 4, ctypes.byref(self._p)))
        self.array = np.ctypeslib.as_array(ctypes.cast(self._p, ctypes.POINTER(ctypes.c_uint32)), shape=(words,))
        self.words = words

    @property
    def ptr(self) -> int:
        return self._p.value

    def free(self):
        if self._p:
            lib().zkg_host_free(self._p)
        self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class ProofInputs:
    """Host buffers of one request of size m = 2^log_m: three G1 scalar vectors (counts m, m,
    m - 1024 by default), one G2 scalar vector (m), three evaluation vectors of N = 2m elements,
    and the outputs (4 XYZZ points, N coefficients)."""

    def __init__(self, log_m: int, g1_counts=None):
        self.log_m = log_m
        m = 1 << log_m
        self.m, self.N = m, 2 * m
        self.g1_counts = list(g1_counts or [m, m, m - 1024])
        self.g1 = [PinnedWords(8 * m) for _ in range(3)]
        self.g2 = PinnedWords(8 * m)
        self.polys = [PinnedWords(8 * self.N) for _ in range(3)]
        self.out_points = PinnedWords(3 * 32 + 64)
        self.out_h = PinnedWords(8 * self.N)

    def fill(self, g1_scalars, g2_scalars, polys):
        for j in range(3):
            s = np.asarray(g1_scalars[j], dtype=np.uint32)
            self.g1[j].array[: s.size] = s
        self.g2.array[:] = np.asarray(g2_scalars, dtype=np.uint32)
        for j in range(3):
            self.polys[j].array[:] = np.asarray(polys[j], dtype=np.uint32)
        return self

    def descriptor(self) -> ProofRequest:
        d = ProofRequest()
        d.log_m = self.log_m
        for j in range(3):
            d.g1_scalars[j] = self.g1[j].ptr
            d.g1_count[j] = self.g1_counts[j]
            d.polys[j] = self.polys[j].ptr
        d.g2_scalars = self.g2.ptr
        d.out_points = self.out_points.ptr
        d.out_h = self.out_h.ptr
        return d

    def points(self) -> np.ndarray:
        return self.out_points.array.copy()

    def h(self) -> np.ndarray:
        return self.out_h.array.copy()


class Server:
    def __init__(self, gpu: Gpu, lanes: int = 8, plain: bool = False, hbm_budget_bytes: int = 0, coset_g: int = 7):
        cfg = ServerConfig()
        cfg.lanes = lanes
        cfg.plain = int(plain)
        cfg.hbm_budget_bytes = hbm_budget_bytes
        for i in range(8):
            cfg.coset_g[i] = (coset_g >> (32 * i)) & 0xFFFFFFFF
        h = vp()
        check(lib().zkg_server_new(gpu.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h.value
        self._keep = []

    def add_key(self, n: int, g1_bases: Buffer, g2_bases: Buffer) -> None:
        check(lib().zkg_server_add_key(self._h, n, g1_bases.handle, g2_bases.handle))
        self._keep += [g1_bases, g2_bases]

    def submit(self, req: ProofInputs) -> int:
        rid = ctypes.c_uint64()
        d = req.descriptor()
        check(lib().zkg_server_submit(self._h, ctypes.byref(d), ctypes.byref(rid)))
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1) -> dict:
        t = RequestTimes()
        check(lib().zkg_server_wait(self._h, rid, timeout_ms, ctypes.byref(t)))
        return {"queued_ms": t.queued_ms, "device_ms": t.device_ms, "total_ms": t.total_ms}

    def reserve(self, log_m: int, count: int) -> None:
        """Makes idle slots of size 2^log_m until the server holds `count` of them."""
        check(lib().zkg_server_reserve(self._h, log_m, count))

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().zkg_server_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def close(self):
        if self._h:
            lib().zkg_server_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_stream(server: Server, requests, arrivals_s) -> dict:
    """Submits requests[i] at arrivals_s[i] seconds after the start. Returns requests/s over
    the whole run and latency percentiles (submit -> done). One request object may appear more
    than once: its inputs are only read, but overlapping uses write the same output arrays, so
    its outputs are meaningful only when its uses do not overlap."""
    n = len(requests)
    ids = [None] * n
    lat = [None] * n
    t0 = time.perf_counter()

    def waiter():
        for i in range(n):
            while ids[i] is None:
                time.sleep(0.0002)
            lat[i] = server.wait(ids[i])["total_ms"]

    th = threading.Thread(target=waiter)
    th.start()
    for i, (req, at) in enumerate(zip(requests, arrivals_s)):
        delay = t0 + at - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        ids[i] = server.submit(req)
    th.join()
    wall = time.perf_counter() - t0
    lat_arr = np.array(lat)
    return {
        "requests": n,
        "wall_s": wall,
        "req_per_s": n / wall,
        "p50_ms": float(np.percentile(lat_arr, 50)),
        "p99_ms": float(np.percentile(lat_arr, 99)),
        "mean_ms": float(lat_arr.mean()),
    }
