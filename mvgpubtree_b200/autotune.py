"""Autotuner of the persistent batch path: picks the launch shape -- tile width (threads per node)
and resident blocks per SM -- that runs a sample of the caller's workload fastest on this GPU.

Each candidate runs on its own clone of the tree (mvbt_clone), so tuning leaves the tree as it
was and every candidate starts from the same state. On the clone, the first sample step runs
untimed (it also loads the kernel variant), the remaining steps are timed with CUDA events around
the persistent kernel; the candidate with the least kernel time wins and is set on the plan.

Knobs: tile width 8 or 16 (the node is 16 pairs, so an 8-lane tile reads it with 16-byte lane
loads and a 16-lane tile with 8-byte loads) and blocks per SM (0 = full occupancy of the
unconstrained kernel, 4 / 6 / 8 = register-capped variants with more resident warps).
"""
from __future__ import annotations

import numpy as np

DEFAULT_CANDIDATES = ((8, 0), (8, 4), (8, 6), (16, 0), (16, 4), (16, 6))


def _dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    return torch.from_numpy(a.view(np.int32)).cuda()


def autotune_batches(tree, samples, candidates=DEFAULT_CANDIDATES, plan=None) -> dict:
    """samples: at least two workload.Batches steps (the first warms, the rest are timed).
    Returns {"tile_width", "blocks_per_sm", "kernel_ms": {"W<w>/bps<b>": ms}}; when `plan` is
    given, its launch shape is set to the winner."""
    import torch

    if len(samples) < 2:
        raise ValueError("autotune_batches needs at least two sample steps")
    max_ops = max(b.num_ops for b in samples)
    max_batches = max(b.num_batches for b in samples)
    max_pairs = max(max(1, b.range_pairs) for b in samples)
    dsamples = [[_dev(torch, a) for a in (b.type, b.key, b.arg, b.out_off, b.range_cap)] for b in samples]
    result = torch.empty(max_ops, dtype=torch.int32, device="cuda")
    range_out = torch.empty(max_pairs * 2, dtype=torch.int32, device="cuda")
    timings = {}
    best = None
    for w, bps in candidates:
        clone = tree.clone()
        p = clone.batch_plan(max_ops, max_batches)
        p.set_launch(w, bps)
        p.run(samples[0].batch_off, *dsamples[0], result, range_out)
        p.enable_timing(True)
        for b, d in zip(samples[1:], dsamples[1:]):
            p.run(b.batch_off, *d, result, range_out)
        ms = sum(p.kernel_times())
        clone.check_errors()
        p.close()
        clone.close()
        timings[f"W{w}/bps{bps}"] = round(ms, 3)
        if best is None or ms < best[0]:
            best = (ms, w, bps)
    del dsamples, result, range_out
    torch.cuda.empty_cache()
    if plan is not None:
        plan.set_launch(best[1], best[2])
    return {"tile_width": best[1], "blocks_per_sm": best[2], "kernel_ms": timings}
