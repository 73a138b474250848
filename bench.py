#!/usr/bin/env python
"""Benchmark: mixed-op batches on a 40M-key multiversion B-link tree (one B200 per rank).

Workload (one step): 256 independent batches of mixed ops -- erase 10 % (present keys),
insert 20 % (new keys), find 50 % (half hits), range query 20 % (length L geometric with mean 32,
clipped to [1, 1024], upper bound = lower + L * 107) -- with lognormal batch sizes (median 16K ops,
sigma 1.5, clipped to [1K, 4M]), on a versioned tree that starts with 40M distinct uniform keys
from [1, 2^32 - 3], one snapshot per batch. Inputs are synthetic and seeded (no dataset exists
for this workload); each step gets fresh batches, generated against the evolving key set.

value    : Mops/s of the batched path (one persistent launch per step, ops resident in HBM).
e2e      : Mops/s through the public batch API with host buffers: per step the op arrays are
           copied from pinned host memory, the captured CUDA graph is replayed, and the results
           (values, counts) and the range pairs that exist (packed on the device) are copied
           back; two steps are in flight, so copies overlap the next step's run.
plain    : the same W warm-up + K timed steps as one snapshot + one launch per batch (the drop-in
           method), on an identical tree, so both arms time the same steps on trees of the same age.
roofline : algorithmic bytes of the persistent kernel per launch / its CUDA-event time.
verified : every result of every step, batched against plain (range pairs on the warm-up steps);
           step 0 in full (find values, range counts and pairs) against the CPU oracle and against
           the reference implementation's own CUDA build; configs 1-3 against the oracle.
serving  : continuous batching of Poisson-arriving requests (lognormal sizes, median 256 ops) at
           offered loads of 10 / 50 / 200 M ops/s for a short window each, on a 40M-key tree with
           reclamation; p50 / p99 / p999 latency (arrival to results on the host) and achieved
           throughput, beside the plain mode with one request per launch on an identical tree.
configs  : the other workloads of the reference's benchmarks, measured alone before the above:
           c1 plain-tree insert + finds (2^20 keys), c2 versioned insert / update / finds at two
           snapshots (2^25 keys), c3 inserts + range queries at the snapshot before them on 40M
           keys (9 mixes; one concurrent_insert_range call, and insert then range_query).

With --impl reference the script times the reference implementation's own CUDA build
(oracle/_ref/ref_driver, built by oracle/ref_build.py from the reference's unmodified headers) on
the same batches through its public host API, one batch at a time (take_snapshot, find(ts),
range_query(ts), insert, erase), and reports the oracle's multiversion ordered map
(key-range partitioned over all host cores, one full step) as its cpu_baseline. Without the
reference build its value is null and the line says why.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mops/s mixed ops @40M keys, batched vs plain launch, bit-exact; serving p99 µs"
UNIT = "Mops/s"
KEYS_40M = 40_000_000
HBM_FALLBACK_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--initial-keys", type=int, default=KEYS_40M)
    ap.add_argument("--batches", type=int, default=256)
    ap.add_argument("--seed", type=int, default=20240611)
    ap.add_argument("--tile-width", type=int, default=8)
    ap.add_argument("--blocks-per-sm", type=int, default=0,
                    help="0 = full occupancy of the default kernel; 6 / 8 = register-capped variants")
    ap.add_argument("--e2e-steps", type=int, default=12,
                    help="timed steps of the end-to-end pipeline (two in flight; more steps amortise its fill and drain)")
    ap.add_argument("--pool-gb", type=float, default=30.0,
                    help="node pool of each tree of the batched, plain and e2e arms")
    ap.add_argument("--serve-pool-gb", type=float, default=24.0,
                    help="node pool of the serving sessions (the memory cap of config 5)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep --tile-width / --blocks-per-sm instead of tuning the launch shape")
    ap.add_argument("--serve-loads", default="10,50,200",
                    help="offered loads (M ops/s) of the serving sessions; empty = no serving run")
    ap.add_argument("--serve-seconds", type=float, default=4.0,
                    help="arrival window of each serving session, capped at --serve-max-ops ops of trace")
    ap.add_argument("--serve-max-ops", type=float, default=50e6,
                    help="most ops of one serving session's trace (the whole trace and its range "
                         "output slots are held in pinned host memory)")
    ap.add_argument("--serve-max-lag", type=int, default=1 << 22,
                    help="serving admission: most version copies waiting for reclamation")
    ap.add_argument("--no-reclaim-arm", action="store_true",
                    help="skip the batched steps with reclamation inside the persistent launch")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the c1-c3 workloads (plain finds, finds at snapshots, concurrent "
                         "insert + range) reported under \"configs\"")
    ap.add_argument("--config-reps", type=int, default=2,
                    help="timed experiments per c1-c3 measurement (after one untimed)")
    ap.add_argument("--profile-case", choices=["sorted-insert-16M", "update-find-16M"], default=None,
                    help="run only a small case of one kernel for a profiler capture and exit: "
                         "sorted-insert-16M = a 16M-key bulk-loaded versioned tree, a snapshot, "
                         "then one insert call of 3.6M new keys (the u90 mix of config 3 at 0.4x); "
                         "update-find-16M = a 2^24-key bulk-loaded versioned tree, a snapshot, 2^22 "
                         "updates and then 2^22 finds at the snapshot, both through the unsorted "
                         "path (k_insert, k_find)")
    return ap.parse_args()


def run_profile_case(args) -> None:
    """A small case of one kernel, sized for an ncu capture (about 1 GB on the device)."""
    import torch
    import mvgpubtree_b200 as mv
    import workload as wl

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b)

    seed = args.seed
    out = {"case": args.profile_case, "tile_width": args.tile_width}
    if args.profile_case == "sorted-insert-16M":
        n, m = 16_000_000, 3_600_000
        keys = wl.distinct_keys(seed, 0, n)
        ins = wl.distinct_keys(seed, n, m)
        t = mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=args.tile_width)
        t.insert(dev(keys), dev(wl.values_for(keys, seed)))
        t.take_snapshot()
        di, dv = dev(ins), dev(wl.values_for(ins, seed))
        ms = timed(lambda: t.insert(di, dv))
        out.update({"ms": round(ms, 3), "mops": round(m / ms / 1e3, 1)})
    else:
        n, m = 1 << 24, 1 << 22
        keys = wl.distinct_keys(seed, 0, n)
        t = mv.gpu_versioned_btree(pool_bytes=1 << 30, tile_width=args.tile_width)
        t.insert(dev(keys), dev(wl.values_for(keys, seed)))
        s0 = t.take_snapshot()
        t.set_frontend(mv.FRONTEND_UNSORTED)
        upd = wl.shuffle(seed + 3, keys)[:m]
        du, duv = dev(upd), dev(wl.values_for(upd, seed ^ 1))
        q = dev(wl.shuffle(seed + 5, keys)[:m])
        r = torch.empty(m, dtype=torch.int32, device="cuda")
        ms_u = timed(lambda: t.insert(du, duv))
        ms_f = timed(lambda: t.find(q, r, timestamp=s0))
        out.update({"update_ms": round(ms_u, 3), "update_mops": round(m / ms_u / 1e3, 1),
                    "find_ms": round(ms_f, 3), "find_mops": round(m / ms_f / 1e3, 1)})
    t.check_errors()
    print(json.dumps(out), flush=True)
    t.close()


# ------------------------------------------------------------------------------------------------
# process group (one process per GPU; replicas: no data-path collective)
# ------------------------------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend):
        if self.world > 1:
            import datetime
            import torch.distributed as td
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = td

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.reader = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.reader.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_gbs():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return HBM_FALLBACK_GBS, "fallback"


# ------------------------------------------------------------------------------------------------
# workload
# ------------------------------------------------------------------------------------------------
def make_workload(seed: int, initial: int, steps: int, batches: int):
    import workload as wl
    t0 = time.time()
    init = wl.distinct_keys(seed, 0, initial)
    vals = wl.values_for(init, 0)
    gen = wl.MixGenerator(seed, initial, stride=wl.stride_for(KEYS_40M))
    out = [gen.generate(batches) for _ in range(steps)]
    return init, vals, out, time.time() - t0


def op_bytes(b, result: np.ndarray, height: int, leaf_fill: float) -> float:
    """Algorithmic bytes touched by one step's ops (node = 128 B, H = tree height):
    find 128 H + 8; insert 128 (H + 1) + 256 + 8 (descent, locked reload, version copy, leaf
    write, key + value); erase 128 (H + 1) + 256 + 4; range 128 H + 128 (leaves - 1) + 8 count + 8
    with leaves = 1 + count / (keys per leaf)."""
    t = b.type
    n_find = int(np.count_nonzero(t == 0))
    n_ins = int(np.count_nonzero(t == 1))
    n_er = int(np.count_nonzero(t == 2))
    cnt = result[t == 3].astype(np.float64)
    H = float(height)
    total = n_find * (128 * H + 8) + n_ins * (128 * (H + 1) + 256 + 8) + n_er * (128 * (H + 1) + 256 + 4)
    total += float(np.sum(128 * H + 128 * (cnt / leaf_fill) + 8 * cnt + 8))
    return total


def valid_pair_positions(torch, d_type, d_result, d_off, d_cap):
    """Device positions (pair index into the step's range output) of every pair the step's range
    queries wrote: query i's first min(count_i, cap_i) slots from out_off[i]."""
    r = d_type == 3
    off = d_off[r]
    take = torch.minimum(d_result[r].long() & 0xFFFFFFFF, d_cap[r].long() & 0xFFFFFFFF)
    total = int(take.sum())
    if total == 0:
        return torch.empty(0, dtype=torch.int64, device=d_type.device)
    starts = torch.cumsum(take, 0) - take
    return torch.repeat_interleave(off - starts, take) + torch.arange(total, device=d_type.device)


def run_ours(args, dist: Dist):
    import torch
    import mvgpubtree_b200 as mv

    torch.cuda.set_device(dist.local)
    dist.init("nccl")
    seed = args.seed + 7919 * dist.rank
    W, K = max(3, args.warmup), args.steps
    We, Ke = 2, max(1, args.e2e_steps)  # e2e warm-up: one step per buffer set (graph capture, scratch)
    V = min(W, 3)  # warm-up steps whose range pairs are compared between the batched and plain arms
    n_steps = W + K + We + Ke
    init, vals, steps, gen_s = make_workload(seed, args.initial_keys, n_steps, args.batches)

    def dev(a):
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint64:
            return torch.from_numpy(a.view(np.int64)).cuda()
        return torch.from_numpy(a.view(np.int32)).cuda()

    pool = int(args.pool_gb * (1 << 30))
    max_ops = max(b.num_ops for b in steps)
    max_pairs = max(b.range_pairs for b in steps)
    trees = {}
    for name in ("batched", "plain"):
        t = mv.gpu_versioned_btree(pool_bytes=pool, tile_width=args.tile_width,
                                   blocks_per_sm=args.blocks_per_sm if name == "batched" else 0)
        t.insert(dev(init), dev(vals))
        t.check_errors()
        trees[name] = t
    torch.cuda.synchronize()
    plans = {k: t.batch_plan(max_ops, args.batches) for k, t in trees.items()}
    # launch shape of the persistent path: autotuned on clones of the tree with the first two
    # steps of the workload (the timed steps come later and are not part of the sample)
    tune = None
    if not args.no_autotune:
        from mvgpubtree_b200.autotune import autotune_batches
        tune = autotune_batches(trees["batched"], steps[:2], plan=plans["batched"])
    range_out = {k: torch.empty(max(1, max_pairs) * 2, dtype=torch.int32, device="cuda") for k in trees}
    stream = torch.cuda.current_stream()

    # Both arms run the same W warm-up + K timed steps on identical trees, so their timed steps
    # meet trees of the same age. Results (find values, range counts) of every step are kept for
    # the batched-vs-plain comparison; range pairs are compared on the first V warm-up steps.
    dsteps = [[dev(b.type), dev(b.key), dev(b.arg), dev(b.out_off), dev(b.range_cap)] for b in steps[: W + K]]
    results = {k: [torch.empty(b.num_ops, dtype=torch.int32, device="cuda") for b in steps[: W + K]]
               for k in trees}
    positions, saved_pairs, step0 = [], [], None

    def run_arm(name, mode, on_warm):
        plan = plans[name]
        for s in range(W):
            plan.run(steps[s].batch_off, *dsteps[s], results[name][s], range_out[name], mode=mode)
            on_warm(s)
        trees[name].check_errors()
        plan.enable_timing(name == "batched")
        clocks = ClockSampler(dist.local)
        clocks.start()
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in range(W, W + K):
            plan.run(steps[s].batch_off, *dsteps[s], results[name][s], range_out[name], mode=mode)
        e1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        clk = clocks.stop()
        kms = plan.kernel_times() if name == "batched" else []
        plan.enable_timing(False)
        trees[name].check_errors()
        return dist.max(e0.elapsed_time(e1)), clk, kms

    def batched_warm(s):
        nonlocal step0
        if s >= V:
            return
        d = dsteps[s]
        pos = valid_pair_positions(torch, d[0], results["batched"][s], d[3], d[4])
        positions.append(pos)
        saved_pairs.append(range_out["batched"].view(-1, 2)[pos].clone())
        if s == 0:  # the first full step, checked against the oracle and the reference build
            n = steps[0].range_pairs
            step0 = (results["batched"][0].cpu().numpy().view(np.uint32).copy(),
                     range_out["batched"][: 2 * n].cpu().numpy().view(np.uint32).reshape(n, 2).copy())

    pair_mismatch = []

    def plain_warm(s):
        if s < V:
            got = range_out["plain"].view(-1, 2)[positions[s]]
            pair_mismatch.append(int((got != saved_pairs[s]).any(dim=1).sum()))

    # ---- batched, device-resident: W warm-up + K timed steps, one persistent launch each ----
    plan = plans["batched"]
    ms_max, clk, kernel_ms = run_arm("batched", mv.BATCH_PERSISTENT, batched_warm)
    ops_timed = sum(steps[s].num_ops for s in range(W, W + K))
    ops_all = ops_timed * dist.world
    value = ops_all / (ms_max * 1e-3) / 1e6

    # ---- plain: one snapshot + one launch per batch, the same steps on an identical tree ----
    plain_ms, plain_clk, _ = run_arm("plain", mv.BATCH_PER_LAUNCH, plain_warm)
    plain_value = ops_all / (plain_ms * 1e-3) / 1e6
    result_mismatch = [int((results["batched"][s] != results["plain"][s]).sum()) for s in range(W + K)]
    batched_vs_plain = {
        "steps_compared": W + K, "result_mismatches": int(sum(result_mismatch)),
        "pair_steps_compared": V, "pairs_compared": int(sum(int(p.numel()) for p in positions)),
        "pair_mismatches": int(sum(pair_mismatch)),
        "identical": sum(result_mismatch) == 0 and sum(pair_mismatch) == 0}
    del saved_pairs, positions

    # range counts of the timed steps (for the roofline bytes), read after the timed region
    host_res = [results["batched"][s].cpu().numpy().view(np.uint32) for s in range(W, W + K)]
    plans["plain"].close()
    trees["plain"].close()
    del plans["plain"], trees["plain"], range_out["plain"], results["plain"]
    torch.cuda.empty_cache()

    # ---- the same steps with reclamation inside the persistent launch, on a tree created with
    # reclamation: copies freed while the launch runs and handed out again by the same launch ----
    reclaim_inside = None
    if not args.no_reclaim_arm:
        tr = mv.gpu_versioned_btree(pool_bytes=pool, tile_width=args.tile_width, reclaim=True)
        tr.insert(dev(init), dev(vals))
        pr = tr.batch_plan(max_ops, args.batches)
        if tune:
            pr.set_launch(tune["tile_width"], tune["blocks_per_sm"])
        pr.set_reclaim(True)
        rr = torch.empty(max_ops, dtype=torch.int32, device="cuda")
        nodes, live_lo, live_hi, mism = [], None, None, 0
        for s in range(W):
            pr.run(steps[s].batch_off, *dsteps[s], rr[: steps[s].num_ops], range_out["batched"], mode=mv.BATCH_PERSISTENT)
            mism += int((rr[: steps[s].num_ops] != results["batched"][s]).sum())
        tr.check_errors()
        pr.enable_timing(True)
        torch.cuda.synchronize()
        r0e, r1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        outs_r = [torch.empty(steps[s].num_ops, dtype=torch.int32, device="cuda") for s in range(W, W + K)]
        r0e.record(stream)
        for j, s in enumerate(range(W, W + K)):
            pr.run(steps[s].batch_off, *dsteps[s], outs_r[j], range_out["batched"], mode=mv.BATCH_PERSISTENT)
        r1e.record(stream)
        torch.cuda.synchronize()
        rms = dist.max(r0e.elapsed_time(r1e))
        pr.enable_timing(False)
        tr.check_errors()
        ser = pr.memory_series().astype(np.int64)  # the last timed step, per batch
        live = ser[:, 1] - ser[:, 2]
        mism += sum(int((outs_r[j] != results["batched"][s]).sum()) for j, s in enumerate(range(W, W + K)))
        st = tr.stats()
        reclaim_inside = {
            "value": round(ops_all / (rms * 1e-3) / 1e6, 2), "unit": UNIT, "steps": K,
            "results_identical_to_batched": mism == 0,
            "nodes_taken_from_pool": int(tr.compute_memory_usage()["nodes_allocated"]),
            "nodes_taken_without_reclamation": int(trees["batched"].compute_memory_usage()["nodes_allocated"]),
            "copies_freed": int(st["reclaimed"]), "freed_nodes_reused": int(st["reused"]),
            "live_nodes_last_step": {"first_batch": int(live[0]), "last_batch": int(live[-1]),
                                     "min": int(live.min()), "max": int(live.max())},
            "how": "the batched arm's steps on a tree created with reclamation; copies freed inside "
                   "each persistent launch once the batches that read them have finished"}
        outs_r.clear()
        pr.close()
        tr.close()
        del rr
    del dsteps, results
    torch.cuda.empty_cache()

    # ---- e2e: public API with pinned host buffers, CUDA graph replay, two steps in flight ----
    # Step s: its op arrays cross on the input stream, its graph replay and the packing of its
    # range pairs run on the compute stream, and its results and packed pairs cross back on the
    # output stream once the host has its pair count, while step s + 1 runs. Buffers and plans
    # alternate between two sets.
    e2e_steps = steps[W + K:]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64 if a.dtype == np.uint64 else np.int32)).pin_memory()
    bufs = []
    for k in range(2):
        bp = plan if k == 0 else trees["batched"].batch_plan(max_ops, args.batches)
        if k and tune:
            bp.set_launch(tune["tile_width"], tune["blocks_per_sm"])
        bufs.append({
            "ops": [torch.empty(max_ops, dtype=torch.int32, device="cuda") for _ in range(3)],
            "off": torch.empty(max_ops, dtype=torch.int64, device="cuda"),
            "cap": torch.empty(max_ops, dtype=torch.int32, device="cuda"),
            "res": torch.empty(max_ops, dtype=torch.int32, device="cuda"),
            "rout": range_out["batched"] if k == 0 else torch.empty(max(1, max_pairs) * 2, dtype=torch.int32, device="cuda"),
            "comp": torch.empty(max(1, max_pairs) * 2, dtype=torch.int32, device="cuda"),
            "h_res": torch.empty(max_ops, dtype=torch.int32).pin_memory(),
            "h_comp": torch.empty(max(1, max_pairs) * 2, dtype=torch.int32).pin_memory(),
            "plan": bp, "ev_in": torch.cuda.Event(), "ev_k": torch.cuda.Event(), "ev_out": torch.cuda.Event()})
    h_in = [[pin(b.type), pin(b.key), pin(b.arg), pin(b.out_off), pin(b.range_cap)] for b in e2e_steps]
    h_total = torch.zeros(len(e2e_steps), dtype=torch.int64).pin_memory()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    # per-step stage marks (CUDA events on each stage's stream): input copy, run + packing, output
    # copy; and the host's wait for each step's pair count
    tev = lambda: torch.cuda.Event(enable_timing=True)
    marks = [{k: tev() for k in ("in0", "in1", "k0", "k1", "o0", "o1")} for _ in e2e_steps]
    host_wait = [0.0] * len(e2e_steps)
    host_run = [0.0] * len(e2e_steps)

    def finish(q):
        bq, b = bufs[q % 2], e2e_steps[q]
        t0 = time.perf_counter()
        bq["ev_k"].synchronize()  # step q's run and packing are done; its pair count is on the host
        host_wait[q] = 1e3 * (time.perf_counter() - t0)
        tot = int(h_total[q])
        with torch.cuda.stream(s_out):
            s_out.wait_event(bq["ev_k"])
            marks[q]["o0"].record(s_out)
            bq["h_res"][: b.num_ops].copy_(bq["res"][: b.num_ops], non_blocking=True)
            bq["h_comp"][: 2 * tot].copy_(bq["comp"][: 2 * tot], non_blocking=True)
            marks[q]["o1"].record(s_out)
            bq["ev_out"].record(s_out)
        out_bytes_of[q] = b.num_ops * 4 + 8 + tot * 8
        return out_bytes_of[q]

    ev0, ev1 = tev(), tev()
    h2d = d2h = 0
    in_bytes = [sum(int(h.numel() * h.element_size()) for h in hs) for hs in h_in]
    out_bytes_of = [0] * len(e2e_steps)
    for s, b in enumerate(e2e_steps):
        bs, n = bufs[s % 2], b.num_ops
        if s == We:
            if s:
                finish(s - 1)
            dist.barrier()
            torch.cuda.synchronize()
            ev0.record(stream)
        with torch.cuda.stream(s_in):
            s_in.wait_event(bs["ev_k"])  # the run two steps back has read these buffers
            marks[s]["in0"].record(s_in)
            dst = [bs["ops"][0][:n], bs["ops"][1][:n], bs["ops"][2][:n], bs["off"][:n], bs["cap"][:n]]
            for d, h in zip(dst, h_in[s]):
                d.copy_(h, non_blocking=True)
            marks[s]["in1"].record(s_in)
            bs["ev_in"].record(s_in)
        stream.wait_event(bs["ev_in"])
        stream.wait_event(bs["ev_out"])  # its results from two steps back have crossed
        marks[s]["k0"].record(stream)
        t_run = time.perf_counter()
        bs["plan"].run(b.batch_off, bs["ops"][0], bs["ops"][1], bs["ops"][2], bs["off"], bs["cap"], bs["res"],
                       bs["rout"], mode=mv.BATCH_GRAPH, stream=stream)
        # the pair count goes straight to pinned host memory: no copy queued behind the big ones
        bs["plan"].compact_ranges(n, bs["ops"][0], bs["res"], bs["off"], bs["cap"], bs["rout"], bs["comp"],
                                  h_total[s:s + 1], stream=stream)
        host_run[s] = 1e3 * (time.perf_counter() - t_run)
        marks[s]["k1"].record(stream)
        bs["ev_k"].record(stream)
        if s >= We:
            h2d += in_bytes[s]
        if s >= 1 and s != We:
            out_bytes = finish(s - 1)
            if s - 1 >= We:
                d2h += out_bytes
    d2h += finish(len(e2e_steps) - 1)
    ev1.record(s_out)
    torch.cuda.synchronize()
    trees["batched"].check_errors()
    e2e_ms = dist.max(ev0.elapsed_time(ev1))
    e2e_ops = sum(b.num_ops for b in e2e_steps[We:]) * dist.world
    e2e_value = e2e_ops / (e2e_ms * 1e-3) / 1e6
    e2e_stages = [{"in_ms": round(m["in0"].elapsed_time(m["in1"]), 2),
                   "in_gbs": round(in_bytes[i] / max(1e-6, m["in0"].elapsed_time(m["in1"])) / 1e6, 1),
                   "run_ms": round(m["k0"].elapsed_time(m["k1"]), 2),
                   "out_ms": round(m["o0"].elapsed_time(m["o1"]), 2),
                   "out_gbs": round(out_bytes_of[i] / max(1e-6, m["o0"].elapsed_time(m["o1"])) / 1e6, 1),
                   "run_start_ms": round(ev0.elapsed_time(m["k0"]), 2),
                   "gap_before_run_ms": round(marks[i - 1]["k1"].elapsed_time(m["k0"]), 2),
                   "host_run_call_ms": round(host_run[i], 2),
                   "host_wait_ms": round(host_wait[i], 2)}
                  for i, m in enumerate(marks) if i >= We]
    copy_peak = pinned_copy_peak(torch)

    # ---- roofline of the persistent kernel ----
    rep = trees["batched"].validate_tree_structure()
    fill = rep["keys"] / max(1, rep["leaves"])
    bytes_per = [op_bytes(steps[W + i], host_res[i], rep["height"], fill) for i in range(K)]
    kms = kernel_ms[-K:] if len(kernel_ms) >= K else kernel_ms
    avg_bytes = sum(bytes_per) / len(bytes_per)
    avg_kms = sum(kms) / len(kms)
    peak, peak_kind = measured_hbm_gbs()
    achieved = avg_bytes / (avg_kms * 1e-3) / 1e9
    mean_ops = sum(steps[s].num_ops for s in range(W, W + K)) / K
    # DRAM bytes per launch: an ncu capture of one full-size launch of this kernel on this
    # workload (profiles/k_batched_traffic.json), per op, times the mean ops of the timed launches
    traffic = None
    tf = ROOT / "profiles" / "k_batched_traffic.json"
    if tf.exists():
        try:
            traffic = int(json.loads(tf.read_text())["dram_bytes_per_op"] * mean_ops)
        except Exception:
            traffic = None
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": dist.world,
        "steps": K, "warmup": W, "ms_per_step": round(ms_max / K, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
        "config": {
            "workload": "mixed batches (erase 10 %, insert 20 %, find 50 % with 50 % hits, range "
                        f"20 % with L~geometric(32) clipped [1,1024], stride 107) on a "
                        f"{args.initial_keys / 1e6:g}M-key versioned B-link tree, one snapshot per batch",
            "initial_keys": args.initial_keys, "batches_per_step": args.batches,
            "batch_size": "lognormal median 16384, sigma 1.5, clipped [1024, 4194304]",
            "mean_ops_per_step": int(mean_ops), "mode": "persistent launch, device work queue",
            "tile_width": tune["tile_width"] if tune else args.tile_width,
            "blocks_per_sm": tune["blocks_per_sm"] if tune else args.blocks_per_sm,
            "autotune": tune,
            "parallelism": f"replicas x{dist.world}",
            "l2": "inputs larger than L2 (tree of %d nodes = %.1f GB; ops %.0f MB per step)" % (
                rep["nodes_allocated"], rep["nodes_allocated"] * 128 / 1e9, mean_ops * 24 / 1e6),
            "tree_height": rep["height"], "workload_gen_s": round(gen_s, 1),
        },
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT,
                "h2d_bytes_per_step": int(h2d / max(1, Ke)), "d2h_bytes_per_step": int(d2h / max(1, Ke)),
                "mode": "CUDA graph replay via the public batch API, pinned host buffers, two steps in "
                        "flight: op arrays in, results and the range pairs that exist (packed by "
                        "mvbt_batch_compact_ranges) back, overlapping the next step's run",
                "stages": e2e_stages,
                "copy_gbs": {"h2d": round(sum(in_bytes[We:]) / max(1e-6, sum(x["in_ms"] for x in e2e_stages)) / 1e6, 1),
                             "d2h": round(sum(out_bytes_of[We:]) / max(1e-6, sum(x["out_ms"] for x in e2e_stages)) / 1e6, 1),
                             "pinned_peak_h2d": copy_peak[0], "pinned_peak_d2h": copy_peak[1],
                             "peak_how": "1 GiB pinned <-> device copy, best of 3, CUDA events, same process"}},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "kernel": "k_batched", "kernel_ms": round(avg_kms, 3),
                     "algorithmic_bytes_per_launch": int(avg_bytes), "peak_source": peak_kind},
        "clocks": clk,
        "gpu_launches": 5 * K,
        "verified": {"batched_vs_plain": batched_vs_plain},
    }
    if reclaim_inside is not None:
        out["reclaim_inside_launch"] = reclaim_inside
    plain = {"value": round(plain_value, 2), "unit": UNIT, "steps": K, "warmup": W,
             "ms_per_step": round(plain_ms / K, 3), "batched_over_plain": round(value / plain_value, 3),
             "same_steps_as_batched": True, "clocks": plain_clk,
             "how": "the same W warm-up + K timed steps as the batched arm, on an identical tree "
                    "(one snapshot + one mixed launch per batch)"}
    del plans, plan, bufs, h_in, range_out
    trees.clear()
    torch.cuda.empty_cache()
    if args.serve_loads:
        out["serving"] = run_serving(args, seed, init, vals, dev,
                                     verify=dist.world == 1 and not args.no_cpu_baseline)
        out["serving_p99_us"] = out["serving"]["headline"]["p99_us"]
        checks = [r["batched"]["oracle_check"] for r in out["serving"]["per_load"] if "oracle_check" in r["batched"]]
        if checks:
            out["verified"]["serving_vs_oracle"] = {
                "identical": all(c["identical"] for c in checks),
                "results_compared": sum(c["results_compared"] for c in checks),
                "pairs_compared": sum(c["pairs_compared"] for c in checks),
                "how": "every batched serving session replayed on the partitioned oracle: the requests "
                       "that share a snapshot as one batch, in snapshot order, carrying the state across "
                       "the offered loads; every find value, range count and range pair compared"}
    return out, plain, (init, vals, steps[0], step0)


def pinned_copy_peak(torch, nbytes: int = 1 << 30):
    """Best-of-3 GB/s of one pinned host -> device and one device -> pinned host copy of nbytes."""
    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    best = [0.0, 0.0]
    for _ in range(3):
        for k, (dst, src) in enumerate(((d, h), (h, d))):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            dst.copy_(src, non_blocking=True)
            b.record()
            b.synchronize()
            best[k] = max(best[k], nbytes / (a.elapsed_time(b) * 1e-3) / 1e9)
    del h, d
    return round(best[0], 1), round(best[1], 1)


def latency_summary(arrival_ns, done_ns, ops: int) -> dict:
    lat = (done_ns.astype(np.int64) - arrival_ns.astype(np.int64)) / 1e3
    span = float(done_ns.max()) / 1e9
    return {"achieved_mops": round(ops / span / 1e6, 2), "p50_us": round(float(np.percentile(lat, 50)), 1),
            "p99_us": round(float(np.percentile(lat, 99)), 1),
            "p999_us": round(float(np.percentile(lat, 99.9)), 1), "max_us": round(float(lat.max()), 1)}


def run_serving(args, seed: int, init, vals, dev, verify: bool = True) -> dict:
    """Serving (continuous batching) at each offered load: Poisson arrivals of mixed requests
    (lognormal sizes, median 256 ops, clipped [1, 64K]) for args.serve_seconds, on a 40M-key tree
    with reclamation; beside it the plain mode (one request per launch) on an identical tree.
    Latency = arrival to results on the host; throughput = ops / (start to last completion).
    Every result of the batched sessions is replayed on the partitioned oracle (verify=True): the
    requests that share a snapshot form one batch, applied in snapshot order, and every find value,
    range count and range pair is compared."""
    import torch
    import mvgpubtree_b200 as mv
    import workload as wl
    loads = [float(x) for x in str(args.serve_loads).split(",") if x.strip()]
    pool = int(args.serve_pool_gb * (1 << 30))
    trees = {"batched": mv.gpu_versioned_btree(pool_bytes=pool, tile_width=args.tile_width, reclaim=True),
             "plain": mv.gpu_versioned_btree(pool_bytes=pool, tile_width=args.tile_width)}
    for t in trees.values():
        t.insert(dev(init), dev(vals))
        t.check_errors()
    replay = None
    if verify:
        import oracle
        replay = oracle.PartitionedMVMap(os.cpu_count() or 1, versioned=True)
        replay.insert(init, vals)
    gen = wl.serving_generator(seed, args.initial_keys, wl.stride_for(KEYS_40M))  # the trees' key set
    mean_size = 657.0  # mean of the request-size distribution (lognormal median 256, sigma 1.5)
    per_load = []
    for k, load in enumerate(loads):
        seconds = min(args.serve_seconds, args.serve_max_ops / (load * 1e6))
        R = max(16, int(load * 1e6 * seconds / mean_size))
        b, arrival = wl.serving_trace(seed + 11 * (k + 1), 0, R, load, 0, generator=gen)
        res = {"offered_mops": load, "seconds": round(seconds, 3), "requests": R, "ops": int(b.num_ops)}
        for name, t in trees.items():
            kw = ({"reclaim_in_launch": 1, "max_reclaim_lag": args.serve_max_lag} if name == "batched"
                  else {})
            o = t.serve(b, arrival, mode=mv.BATCH_PERSISTENT if name == "batched" else mv.BATCH_PER_LAUNCH, **kw)
            t.check_errors()
            summ = latency_summary(arrival, o["done_ns"], b.num_ops)
            summ.update({k: o["stats"][k] for k in ("launches", "reclaims", "max_waiting", "memory_waits",
                                                     "max_reclaim_lag", "lag_waits", "nodes_high_water")})
            if name == "batched" and replay is not None:
                summ["oracle_check"] = serving_replay_check(replay, wl, b, o)
            res[name] = summ
        per_load.append(res)
    st = trees["batched"].stats()
    use = trees["batched"].compute_memory_usage()
    head = next((r for r in per_load if r["offered_mops"] == 50.0), per_load[-1])
    gen.close()
    if replay is not None:
        replay.close()
    return {"mode": "continuous batching: the requests that arrived while the previous launch ran "
                    "form the next launch, one snapshot per admitted batch (reads at it, writes after), "
                    "reclamation inside every launch, admission by free nodes and by reclamation lag",
            "request_size": "lognormal median 256 ops, sigma 1.5, clipped [1, 65536]",
            "arrivals": "Poisson", "seconds_per_load": "min(serve_seconds, serve_max_ops / load)",
            "serve_seconds": args.serve_seconds, "serve_max_ops": args.serve_max_ops, "pool_gb": args.serve_pool_gb,
            "per_load": per_load,
            "headline": {"offered_mops": head["offered_mops"], **{k: head["batched"][k] for k in
                         ("achieved_mops", "p50_us", "p99_us", "p999_us")}},
            "reclaimed_nodes": st["reclaimed"], "reused_nodes": st["reused"],
            "nodes_high_water": use["nodes_allocated"]}


def serving_replay_check(m, wl, b, o) -> dict:
    """The batched serving session `o` over trace `b` replayed on the partitioned oracle `m` (which
    holds the tree's state before the session): requests that share a snapshot are one batch."""
    snaps = o["snapshot"].astype(np.int64)
    R = snaps.size
    steps = np.diff(snaps)
    ordered = bool(np.all((steps == 0) | (steps == 1)))
    starts = np.concatenate([[0], np.nonzero(steps)[0] + 1, [R]])
    g = wl.Batches(b.batch_off[starts].astype(np.uint64), b.type, b.key, b.arg, b.out_off, b.range_cap,
                   b.range_pairs)
    res, out = m.run_batches(g, with_pairs=True)
    r = b.type == 3
    take = np.minimum(res[r], b.range_cap[r]).astype(np.int64)
    pos = np.repeat(b.out_off[r].astype(np.int64) - (np.cumsum(take) - take), take) + np.arange(int(take.sum()))
    bad_res = int(np.count_nonzero(res != o["result"][: res.size]))
    bad_pairs = int(np.count_nonzero((out.reshape(-1, 2)[pos] != o["range_out"][pos]).any(axis=1)))
    return {"groups": int(len(starts) - 1), "snapshots_in_order": ordered, "results_compared": int(res.size),
            "result_mismatches": bad_res, "pairs_compared": int(pos.size), "pair_mismatches": bad_pairs,
            "identical": ordered and bad_res == 0 and bad_pairs == 0}


# ------------------------------------------------------------------------------------------------
# CPU side: the oracle (the reference-side CPU implementation of the path), timed on host cores
# ------------------------------------------------------------------------------------------------
REF_DRIVER = Path(__file__).resolve().parent / "oracle" / "_ref" / "ref_driver"

# ------------------------------------------------------------------------------------------------
# the other workloads of the reference's own benchmarks, in both arms (configs 1-3)
#   c1: plain B-link tree, 2^20 keys inserted, 2^20 finds (half hits)
#   c2: versioned tree, 2^25 keys, 2^22 in-place updates, 2^25 finds at the snapshot before and
#       at the snapshot after the updates
#   c3: versioned tree of 40M keys, 10M ops (each an insert with probability u, else a range query
#       of length L at the snapshot taken before the inserts), u in {5, 50, 90} %, L in {8, 32, 128};
#       "concurrent" = one concurrent_insert_range call, "sequence" = insert, then range_query
# Every phase is timed alone with CUDA events, after one untimed experiment, mean of --config-reps.
# ------------------------------------------------------------------------------------------------
C1_KEYS, C2_KEYS, C2_UPDATES = 1 << 20, 1 << 25, 1 << 22
C3_OPS, C3_UPDATE, C3_LENGTHS = 10_000_000, (0.05, 0.5, 0.9), (8, 32, 128)
C3_REF_CONCURRENT_UNAVAILABLE = (
    "the reference's concurrent_insert_range raised an illegal memory access on a B200 with "
    "in-bounds inputs (262144 keys, 54000 inserts + 6000 range queries of L = 128), so it is not "
    "run; its plain form (insert, then range_query at the snapshot before) is timed instead")


def hit_miss_queries(wl, seed: int, keys: np.ndarray) -> np.ndarray:
    n = keys.size
    hits = wl.shuffle(seed + 1, keys)[: n // 2]
    miss = wl.distinct_keys(seed, wl.MISS_INDEX_BASE, n - n // 2)
    return wl.shuffle(seed + 2, np.concatenate([hits, miss]))


def c3_combos(seed: int):
    """(u, L, inserts, ranges) of config 3: each of the 10M ops is an insert with probability u."""
    out = []
    for u in C3_UPDATE:
        n_ins = int((np.random.default_rng(seed).random(C3_OPS) < u).sum())
        out += [(u, L, n_ins, C3_OPS - n_ins) for L in C3_LENGTHS]
    return out


def _hmean(xs):
    return len(xs) / sum(1.0 / x for x in xs)


def run_configs_ours(args) -> dict:
    """Configs 1-3 through this library's reference-named host API, tile widths 8 and 16 (the
    faster is reported). Every result is checked against the oracle at full size: each c1 and c2
    find, and each c3 range count and range pair (all 9 mixes, 40M keys, 10M ops) at the snapshot
    taken before the inserts (oracle.SortedSnapshot of the initial keys)."""
    import torch
    import mvgpubtree_b200 as mv
    import oracle
    import workload as wl

    seed, reps = args.seed, max(1, args.config_reps)
    stream = torch.cuda.current_stream()

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    def mean_runs(make, phases):
        """1 untimed + reps timed experiments of make() -> tree, then phases(tree) -> [ms...]."""
        acc = None
        for r in range(1 + reps):
            t = make()
            ms = phases(t)
            t.check_errors()
            t.close()
            if r:
                acc = ms if acc is None else [x + y for x, y in zip(acc, ms)]
        return [x / reps for x in acc]

    out = {}
    # ---- c1 ----
    n = C1_KEYS
    keys = wl.distinct_keys(seed, 0, n)
    vals = wl.values_for(keys, seed)
    q = hit_miss_queries(wl, seed, keys)
    expect = oracle.SortedSnapshot(keys, vals).find(q)
    dk, dv, dq = dev(keys), dev(vals), dev(q)
    r0 = torch.empty(n, dtype=torch.int32, device="cuda")
    FE = {"auto": mv.FRONTEND_AUTO, "unsorted": mv.FRONTEND_UNSORTED}
    rows = []
    for fe, w in [(f, w) for f in FE for w in (8, 16)]:
        ms = mean_runs(lambda: mv.gpu_blink_tree(pool_bytes=1 << 30, tile_width=w, frontend=FE[fe]),
                       lambda t: [timed(lambda: t.insert(dk, dv)), timed(lambda: t.find(dq, r0))])
        ok = bool(np.array_equal(r0.cpu().numpy().view(np.uint32), expect))
        rows.append({"frontend": fe, "tile_width": w, "insert_mops": round(n / ms[0] / 1e3, 1),
                     "find_mops": round(n / ms[1] / 1e3, 1), "verified": ok})
    out["c1_plain_2^20"] = config_summary(rows, "find_mops", ["insert_mops", "find_mops"])
    del dk, dv, dq, r0

    # ---- c2 ----
    n, u = C2_KEYS, C2_UPDATES
    keys = wl.distinct_keys(seed, 0, n)
    upd = wl.shuffle(seed + 3, keys)[:u]
    q = hit_miss_queries(wl, seed, keys)
    v0 = wl.values_for(keys, seed)
    e0 = oracle.SortedSnapshot(keys, v0).find(q)
    v1 = v0.copy()
    v1[np.isin(keys, upd, assume_unique=True)] = wl.values_for(keys[np.isin(keys, upd, assume_unique=True)], seed ^ 1)
    e1 = oracle.SortedSnapshot(keys, v1).find(q)
    del v0, v1
    dk, dv, du, duv, dq = dev(keys), dev(wl.values_for(keys, seed)), dev(upd), dev(wl.values_for(upd, seed ^ 1)), dev(q)
    r0 = torch.empty(n, dtype=torch.int32, device="cuda")
    r1 = torch.empty(n, dtype=torch.int32, device="cuda")
    rows = []
    for fe, w in [(f, w) for f in FE for w in (8, 16)]:
        def phases(t):
            a = timed(lambda: t.insert(dk, dv))
            s0 = t.take_snapshot()
            b = timed(lambda: t.insert(du, duv))
            s1 = t.take_snapshot()
            return [a, b, timed(lambda: t.find(dq, r0, timestamp=s0)), timed(lambda: t.find(dq, r1, timestamp=s1))]
        ms = mean_runs(lambda: mv.gpu_versioned_btree(pool_bytes=4 << 30, tile_width=w, frontend=FE[fe]), phases)
        ok = bool(np.array_equal(r0.cpu().numpy().view(np.uint32), e0)
                  and np.array_equal(r1.cpu().numpy().view(np.uint32), e1))
        rows.append({"frontend": fe, "tile_width": w, "insert_mops": round(n / ms[0] / 1e3, 1),
                     "update_mops": round(u / ms[1] / 1e3, 1), "find_s0_mops": round(n / ms[2] / 1e3, 1),
                     "find_s1_mops": round(n / ms[3] / 1e3, 1), "verified": ok})
    out["c2_versioned_2^25"] = config_summary(rows, "find_s1_mops",
                                              ["insert_mops", "update_mops", "find_s0_mops", "find_s1_mops"])
    del dk, dv, du, duv, dq, r0, r1
    torch.cuda.empty_cache()

    # ---- c3: concurrent insert + range query on clones of one 40M-key tree per tile width ----
    N = args.initial_keys
    stride = wl.stride_for(N)
    keys = wl.distinct_keys(seed, 0, N)
    kvals = wl.values_for(keys, seed)
    dk, dv = dev(keys), dev(kvals)
    # the oracle's state at the snapshot every c3 range query reads: the initial keys
    snap = oracle.SortedSnapshot(keys, kvals)
    d_sk, d_sv = dev(snap.keys), dev(snap.values)
    del kvals
    base, insert_mops, insert_per_op = {}, {}, {}
    for w in (8, 16):
        for fe in (mv.FRONTEND_UNSORTED, mv.FRONTEND_AUTO):
            ms = []
            for r in range(1 + reps):
                t = mv.gpu_versioned_btree(pool_bytes=8 << 30, tile_width=w, frontend=fe)
                ms.append(timed(lambda: t.insert(dk, dv)))
                if r < reps or fe == mv.FRONTEND_UNSORTED:
                    t.close()
            (insert_per_op if fe == mv.FRONTEND_UNSORTED else insert_mops)[w] = round(N / (sum(ms[1:]) / reps) / 1e3, 1)
        base[w] = t
    del dk, dv
    runs = {8: {}, 16: {}}
    seq = {8: {}, 16: {}}
    checks = {}
    lo_start = (None, None)
    for u, L, n_ins, n_rq in c3_combos(seed):
        ins = wl.distinct_keys(seed, N, n_ins)
        lo = wl.uniform_keys(seed + 1, n_rq)
        hi = wl.upper_bounds(lo, L, stride)
        if lo_start[0] != n_rq:  # the lower bounds of a given u are shared by its three lengths
            lo_start = (n_rq, snap.lower_bound(lo))
        a = lo_start[1]
        c = np.maximum(snap.lower_bound(hi) - a, 0)
        d_a, d_c = torch.from_numpy(a).cuda(), torch.from_numpy(c).cuda()
        di, div, dlo, dhi = dev(ins), dev(wl.values_for(ins, seed)), dev(lo), dev(hi)
        pairs = torch.empty(n_rq * 2 * L * 2, dtype=torch.int32, device="cuda")
        counts = torch.empty(n_rq, dtype=torch.int32, device="cuda")
        name = f"u{int(u * 100)}_L{L}"

        def sequence(t):
            s = t.take_snapshot()
            return [timed(lambda: (t.insert(di, div), t.range_query(dlo, dhi, pairs, counts, 2 * L, n_rq, s)))]

        chk = {"queries": n_rq, "pairs": int(np.minimum(c, 2 * L).sum()), "max_count": int(c.max()) if n_rq else 0}
        for w in (8, 16):
            ms = mean_runs(lambda: base[w].clone(),
                           lambda t: [timed(lambda: t.concurrent_insert_range(
                               di, div, n_ins, dlo, dhi, n_rq, pairs, 2 * L, counts))])
            runs[w][name] = round(C3_OPS / ms[0] / 1e3, 1)
            chk[f"w{w}_concurrent_bad"] = check_ranges_device(torch, counts, pairs, d_a, d_c, 2 * L, d_sk, d_sv)
            ms = mean_runs(lambda: base[w].clone(), sequence)
            seq[w][name] = round(C3_OPS / ms[0] / 1e3, 1)
            chk[f"w{w}_sequence_bad"] = check_ranges_device(torch, counts, pairs, d_a, d_c, 2 * L, d_sk, d_sv)
        checks[name] = chk
        del di, div, dlo, dhi, pairs, counts, d_a, d_c
        torch.cuda.empty_cache()
    for t in base.values():
        t.close()
    del d_sk, d_sv
    w = max(runs, key=lambda k: _hmean(list(runs[k].values())))
    ws = max(seq, key=lambda k: _hmean(list(seq[k].values())))
    wi = max(insert_mops, key=insert_mops.get)
    bad = sum(sum(x for k, v in ch.items() if k.endswith("_bad") for x in v) for ch in checks.values())
    out["c3_insert_range_40M"] = {
        "tile_width": w, "insert_40M_mops": insert_mops[wi], "insert_tile_width": wi,
        "insert_40M_mops_by_width": insert_mops,
        "insert_40M_per_op_mops_by_width": insert_per_op,
        "frontend": "auto (the 40M-key tree is a bulk load; the mixes sort their calls)",
        "concurrent_mops": runs[w], "concurrent_hmean_mops": round(_hmean(list(runs[w].values())), 1),
        "sequence_tile_width": ws,
        "sequence_mops": seq[ws], "sequence_hmean_mops": round(_hmean(list(seq[ws].values())), 1),
        "hmean_by_width": {str(x): {"concurrent": round(_hmean(list(runs[x].values())), 1),
                                    "sequence": round(_hmean(list(seq[x].values())), 1)} for x in runs},
        "verified": bad == 0,
        "check": {"how": "every range count and every pair min(count, 2L) of every query, both tile "
                         "widths, concurrent and sequence forms, against the oracle's state at the "
                         "launch snapshot (the initial 40M keys)",
                  "per_mix": checks}}
    torch.cuda.empty_cache()
    return out


def config_summary(rows, key: str, metrics) -> dict:
    """The AUTO front-end's best tile width (by `key`) as the headline row, each metric's best over
    the tile widths per front-end beside it, and every row. AUTO sorts large calls on the device
    and bulk-loads an insert into a pristine tree; UNSORTED runs every op from the root in the
    caller's order (the per-op path)."""
    auto = [r for r in rows if r["frontend"] == "auto"]
    best = dict(max(auto, key=lambda r: r[key]))
    best["best_by_frontend"] = {fe: {m: max(r[m] for r in rows if r["frontend"] == fe) for m in metrics}
                                for fe in sorted({r["frontend"] for r in rows})}
    best["verified"] = all(r["verified"] for r in rows)
    best["rows"] = rows
    return best


def check_ranges_device(torch, counts, pairs, d_start, d_count, cap, d_keys, d_values, chunk=1 << 18):
    """[count mismatches, pair mismatches] of range results against the oracle's answer: query i
    holds d_count[i] hits, the keys d_keys[d_start[i] : d_start[i] + d_count[i]] (sorted snapshot
    arrays from oracle.SortedSnapshot, shipped to the device) with their values; its first
    min(count, cap) pairs sit at pairs[i * cap ...]. The comparison gathers on the device, so the
    tens of GB of fixed-size slots never cross to the host."""
    got = counts.long() & 0xFFFFFFFF
    bad_counts = int((got != d_count).sum())
    P = pairs.view(-1, 2)
    bad_pairs = 0
    n = int(d_count.numel())
    for q0 in range(0, n, chunk):
        q1 = min(n, q0 + chunk)
        take = torch.clamp(d_count[q0:q1], max=cap)
        total = int(take.sum())
        if total == 0:
            continue
        starts = torch.cumsum(take, 0) - take
        j = torch.arange(total, device=take.device) - torch.repeat_interleave(starts, take)
        qi = torch.repeat_interleave(torch.arange(q0, q1, device=take.device), take)
        g = P[qi * cap + j]
        e = d_start[qi] + j
        bad_pairs += int(((g[:, 0] != d_keys[e]) | (g[:, 1] != d_values[e])).sum())
    return [bad_counts, bad_pairs]


def run_configs_reference(args) -> dict:
    """Configs 1-3 on the reference implementation's own CUDA build (oracle/_ref/ref_driver): the
    same inputs and phases as run_configs_ours, through the reference's public host API."""
    if not REF_DRIVER.exists():
        return {"unavailable": "reference build not present"}
    reps = str(max(1, args.config_reps))
    common = ["--seed", str(args.seed), "--warmup", "1", "--reps", reps]

    def drive(*a):
        out = subprocess.run([str(REF_DRIVER), *a, *common], capture_output=True, text=True, timeout=1200)
        if out.returncode != 0:
            raise RuntimeError(f"ref_driver {a[0]} failed ({out.returncode}): {out.stderr.strip()[-300:]}")
        return json.loads(out.stdout.strip().splitlines()[-1])

    res = {}
    try:
        c1 = drive("c1", "--n", str(C1_KEYS))
        res["c1_plain_2^20"] = {"insert_mops": round(c1["insert_mops"], 1), "find_mops": round(c1["find_mops"], 1)}
        c2 = drive("c2", "--initial", str(C2_KEYS), "--updates", str(C2_UPDATES))
        res["c2_versioned_2^25"] = {"insert_mops": round(c2["insert_mops"], 1), "update_mops": round(c2["update_mops"], 1),
                                    "find_s0_mops": round(c2["find0_mops"], 1), "find_s1_mops": round(c2["find1_mops"], 1)}
        combos = c3_combos(args.seed)
        spec = ",".join(f"{i}:{r}:{L}:{2 * L}" for _, L, i, r in combos)
        c3 = drive("c3", "--initial", str(args.initial_keys), "--combos", spec, "--checksums", "0")
        ops = {f"u{int(u * 100)}_L{L}": round(x["ops_mops"], 1) for (u, L, _, _), x in zip(combos, c3["runs"])}
        res["c3_insert_range_40M"] = {
            "insert_40M_mops": round(statistics.mean(x["insert_mops"] for x in c3["runs"]), 1),
            "concurrent_mops": None,
            "concurrent_unavailable": C3_REF_CONCURRENT_UNAVAILABLE,
            "sequence_mops": ops, "sequence_hmean_mops": round(_hmean(list(ops.values())), 1)}
    except (RuntimeError, subprocess.TimeoutExpired) as e:
        res["error"] = str(e)[-300:]
    return res


def reference_build_time(args, W: int, K: int):
    """The reference implementation's own CUDA build (oracle/_ref/ref_driver, compiled from the
    reference's unmodified headers) on this workload: same generator, seed and batches, each batch
    issued through the reference's public host API in its plain form (take_snapshot, find(ts),
    range_query(ts), insert, erase). Returns its JSON line, or (None, why)."""
    if not REF_DRIVER.exists():
        return None, "reference build not present (oracle/ref_build.py builds it where the reference sources are)"
    cmd = [str(REF_DRIVER), "c4", "--initial", str(args.initial_keys), "--batches", str(args.batches),
           "--steps", str(K), "--warmup", str(W), "--seed", str(args.seed), "--checksums", "0"]
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=1200)
    except subprocess.TimeoutExpired:
        return None, "reference build timed out"
    if out.returncode != 0:
        return None, f"reference build failed ({out.returncode}): {out.stderr.strip()[-300:]}"
    return json.loads(out.stdout.strip().splitlines()[-1]), None


def run_reference(args, dist: Dist):
    """Reference arm (rank 0 only): the reference implementation's own CUDA build
    (oracle/_ref/ref_driver, from its unmodified headers) on this B200 and this workload, through
    its public host API. The oracle port on the host cores (one full step) is reported beside it as
    cpu_baseline. Without a reference build the arm reports value null with the reason. This
    process loads no library of this repository's product: the workload generator is the host-only
    workload/libworkload.so and the CPU map is oracle/liboracle.so."""
    if dist.rank != 0:
        return None
    W, K = max(3, args.warmup), args.steps
    configs = None if args.no_configs else run_configs_reference(args)
    ref, why = reference_build_time(args, W, K)
    init, vals, steps, _ = make_workload(args.seed, args.initial_keys, 1, args.batches)
    cpu = None
    if not args.no_cpu_baseline:
        import oracle
        cores = os.cpu_count() or 1
        m = oracle.PartitionedMVMap(cores, versioned=True)
        t0 = time.time()
        m.insert(init, vals)
        build_s = time.time() - t0
        t0 = time.perf_counter()
        m.run_batches(steps[0], with_pairs=True)
        run_s = time.perf_counter() - t0
        m.close()
        cpu = {"value": round(steps[0].num_ops / run_s / 1e6, 3), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"one full step ({steps[0].num_ops} ops in {steps[0].num_batches} batches) on the "
                         f"40M-key oracle map, {cores} threads; build {build_s:.1f} s untimed"}
    config = {"workload": "mixed batches on a 40M-key versioned tree, one snapshot per batch "
                          "(same generator, seed and batches as the GPU arm)",
              "initial_keys": args.initial_keys, "batches_per_step": args.batches,
              "implementation": "reference CUDA build (unmodified headers, nvcc sm_100a, its own "
                                "flags) through its public host API, one batch at a time: "
                                "take_snapshot, find(ts), range_query(ts), insert(in_place), erase; "
                                "op arrays resident on the device"}
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": dist.world, "steps": K,
            "warmup": W, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded)", "config": config}
    if ref is None:
        line.update({"value": None, "unavailable": why})
    else:
        value = round(ref["mops"], 3)
        config["ops_timed"] = ref["ops_timed"]
        line.update({"value": value, "ms_per_step": round(ref["ms"] / K, 3),
                     "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if configs is not None:
        line["configs"] = configs
    return line


def oracle_step_check(init, vals, b, gpu_result, gpu_pairs):
    """One full step of mixed batches on the partitioned oracle (all host cores; the map is built
    from the initial keys, untimed): its run is timed (the CPU baseline) and every result -- find
    value, range count, and each of the first min(count, cap) pairs of every range query -- is
    compared with the GPU's results of the same step on the same initial tree."""
    import oracle
    cores = os.cpu_count() or 1
    m = oracle.PartitionedMVMap(cores, versioned=True)
    t0 = time.time()
    m.insert(init, vals)
    build_s = time.time() - t0
    t0 = time.perf_counter()
    res, out = m.run_batches(b, with_pairs=True)
    run_s = time.perf_counter() - t0
    m.close()
    r = b.type == 3
    take = np.minimum(res[r], b.range_cap[r]).astype(np.int64)
    pos = np.repeat(b.out_off[r].astype(np.int64) - (np.cumsum(take) - take), take) + np.arange(int(take.sum()))
    exp_pairs = out.reshape(-1, 2)[pos]
    got_pairs = gpu_pairs[pos]
    bad_res = int(np.count_nonzero(res != gpu_result))
    bad_pairs = int(np.count_nonzero((exp_pairs != got_pairs).any(axis=1)))
    check = {"ops": int(b.num_ops), "results_compared": int(res.size), "result_mismatches": bad_res,
             "pairs_compared": int(pos.size), "pair_mismatches": bad_pairs,
             "identical": bad_res == 0 and bad_pairs == 0,
             "how": "step 0 (256 batches) of the bench workload from the initial 40M-key tree, GPU "
                    "(persistent launch) against the partitioned multiversion-map oracle"}
    cpu = {"value": round(b.num_ops / run_s / 1e6, 3), "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"one full step ({b.num_ops} ops in {b.num_batches} batches) on the 40M-key oracle "
                     f"map, {cores} threads; build {build_s:.1f} s untimed"}
    return check, cpu


def reference_step_check(args, seed: int, b, gpu_result, gpu_pairs) -> dict:
    """Checksums of every result of step 0 from the reference implementation's own CUDA build
    (oracle/_ref/ref_driver, same generator, seed and initial tree, each batch through its public
    host API) against the same sums of this library's step 0 (oracle/refsums.py)."""
    from oracle import refsums
    if not REF_DRIVER.exists():
        return {"unavailable": "reference build not present"}
    try:
        ref = refsums.run_driver("c4", "--initial", str(args.initial_keys), "--batches", str(args.batches),
                                 "--steps", "1", "--warmup", "0", "--seed", str(seed), "--checksums", "1",
                                 timeout=900)
    except (RuntimeError, subprocess.TimeoutExpired) as e:
        return {"unavailable": str(e)[-300:]}
    ours = refsums.step_sums(b, gpu_result, gpu_pairs)
    theirs = [int(x) for x in ref["step_checksums"][0]]
    return {"identical": ours == theirs, "ours": [str(x) for x in ours], "reference": [str(x) for x in theirs],
            "how": "find / range-count / range-pair checksums of step 0 (256 batches, same seed) from "
                   "the reference's CUDA build (take_snapshot, find(ts), range_query(ts), insert, erase "
                   "per batch) and from this library's persistent launch"}


def main():
    args = parse_args()
    dist = Dist()
    if args.profile_case:
        run_profile_case(args)
        return
    if args.impl == "reference":
        out = run_reference(args, dist)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    configs = None
    if dist.world == 1 and not args.no_configs:
        configs = run_configs_ours(args)
    out, plain, (init, vals, b0, step0) = run_ours(args, dist)
    if dist.rank == 0 and dist.world == 1:
        res0, pairs0 = step0
        if not args.no_cpu_baseline:
            check, cpu = oracle_step_check(init, vals, b0, res0, pairs0)
            out["verified"]["c4_step0_vs_oracle"] = check
            out["cpu_baseline"] = cpu
        out["verified"]["c4_step0_vs_reference_build"] = reference_step_check(args, args.seed, b0, res0, pairs0)
    v = out["verified"]
    out["verified"]["all"] = bool(v["batched_vs_plain"]["identical"]
                                  and v.get("c4_step0_vs_oracle", {}).get("identical", False)
                                  and v.get("serving_vs_oracle", {}).get("identical", True)
                                  and all(c.get("verified", False) for c in (configs or {}).values()))
    # the comparison with the plain per-batch launch and the other configs go last on the line
    if configs is not None:
        out["configs"] = configs
    out["plain_per_batch"] = plain
    if dist.rank == 0:
        print(json.dumps(out), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
