"""Autotuner for the NTT tile kernels.

Each plan can run one of several instantiated kernel shapes (threads per CTA,
polynomials per tile, single- or double-buffered TMA staging); all give
identical residues.  :func:`tune_ntt` times every variant on the caller's
batch with CUDA events (device-resident buffers larger than L2, warm-up first)
and pins the fastest on the plan.  Results are cached per (plan shape, count).
"""
from __future__ import annotations

import ctypes as C

from . import _lib

NUM_VARIANTS = 7  # LC_NTT_NUM_VARIANTS
VARIANT_SHAPES = {
    0: "CTA-wide TMA ring: 128 threads, 2 stages",
    1: "CTA-wide TMA ring: 128 threads, 3 stages",
    2: "CTA-wide TMA ring: 256 threads, 2 stages",
    3: "warp-autonomous TMA rings: 4 warps/CTA, 2 stages",
    4: "warp-autonomous TMA rings: 4 warps/CTA, 3 stages",
    5: "CTA-wide TMA ring: 128 threads, 2 stages, swizzled vector transpose (u32, d = 256)",
    6: "CTA-wide TMA ring: 128 threads, 2 stages, swizzled vector transpose, lane twiddles in registers",
}
_cache: dict = {}


def time_variants(plan, count: int, reps: int = 10, warmup: int = 3, inverse: bool = False):
    """Return {variant: mean ms per launch} for ``count`` polynomials per modulus."""
    import torch
    L = _lib.lib()
    elems = plan.n * plan.num_moduli * count
    dtype = torch.int64 if plan.elem_dtype.__name__ == "uint64" else torch.int32
    x = torch.zeros(elems, dtype=dtype, device="cuda")
    y = torch.empty_like(x)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    fn = L.lc_ntt_inverse if inverse else L.lc_ntt_forward
    out = {}
    for v in range(NUM_VARIANTS):
        _lib.check(L.lc_ntt_plan_set_variant(plan.handle, v), "set_variant")
        for _ in range(warmup):
            _lib.check(fn(plan.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), count,
                          st), "tune")
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn(plan.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), count, st)
        b.record()
        torch.cuda.synchronize()
        out[v] = a.elapsed_time(b) / reps
    _lib.check(L.lc_ntt_plan_check(plan.handle, st), "tune check")
    return out


def tune_ntt(plan, count: int, reps: int = 10) -> int:
    """Time every variant on this batch size and keep the fastest on ``plan``."""
    key = (plan.n, plan.num_moduli, plan.elem_dtype.__name__, count)
    if key not in _cache:
        fwd = time_variants(plan, count, reps)
        inv = time_variants(plan, count, reps, inverse=True)
        _cache[key] = (min(fwd, key=lambda v: fwd[v] + inv[v]), fwd, inv)
    best = _cache[key][0]
    _lib.check(_lib.lib().lc_ntt_plan_set_variant(plan.handle, best), "set_variant")
    return best


def last_results(plan, count: int):
    key = (plan.n, plan.num_moduli, plan.elem_dtype.__name__, count)
    return _cache.get(key)


# ------------------------------------------------------------------ commit batches

BATCH_CHUNKS = (1024, 2048, 4096, 8192, 16384)
BATCH_CTAS = (1, 2, 3, 4)
BATCH_CLAIMS = (1, 4)


def _time_batch(batch, reps: int) -> float:
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch.run()  # warm-up (and graph capture for a new configuration)
    a.record()
    for _ in range(reps):
        batch.run()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune_batch(batch, reps: int = 2):
    """Pick the product chunk (CUDA-core products only), the CTAs per SM of
    the persistent launches and the work items per claim for this batch: a
    coordinate search (chunk at 2 CTAs/SM, then CTAs/SM, then the claim
    size) timed with CUDA events.
    Leaves the best configuration on ``batch``; returns (config, timings)."""
    timings = {}

    def t(cfg):
        if cfg not in timings:
            batch.set_config(*cfg)
            timings[cfg] = _time_batch(batch, reps)
        return timings[cfg]

    # the chunk only shapes the CUDA-core products; the tensor-core form
    # splits its items at the exact-int32 bound instead
    chunks = BATCH_CHUNKS if batch.products == batch.PRODUCTS_INT64 else (batch.config[0],)
    best = min(((c, 2, 1) for c in chunks), key=t)
    best = min(((best[0], n, 1) for n in BATCH_CTAS), key=t)
    best = min(((best[0], best[1], k) for k in BATCH_CLAIMS), key=t)
    batch.set_config(*best)
    batch.check()
    return best, {f"{c[0]}/{c[1]}/{c[2]}": ms for c, ms in timings.items()}
