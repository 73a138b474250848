"""B200-native multiversion B-link tree.

Python mirror of the reference's host API (owensgroup/MVGpuBTree: ``GpuBTree::gpu_blink_tree`` in
include/gpu_blink_tree.hpp and ``GpuBTree::gpu_versioned_btree`` in
include/gpu_versioned_blink_tree.hpp) over the C ABI of ``libmvbt.so`` (include/mvbt.h). Method
names, argument order and meaning follow the reference; arrays are CUDA tensors, pinned host
tensors or raw device pointers (ints), exactly as the reference's methods take device (or UVA
pinned) pointers. Every operation runs the library's sm_100a kernels; there is no CPU fallback:
importing this package fails if the library has not been built.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

__all__ = [
    "LATEST", "NOT_FOUND", "MVBTError", "lib", "library_path", "gpu_blink_tree",
    "gpu_versioned_btree", "gpu_versioned_blink_tree", "pair_dtype_words", "BatchPlan",
    "BATCH_PERSISTENT", "BATCH_PER_LAUNCH", "BATCH_GRAPH", "NOALLOC_MAX_OPS", "NOALLOC_MAX_BATCHES",
    "FRONTEND_AUTO", "FRONTEND_UNSORTED", "FRONTEND_SORTED",
    "RECLAIM_ALL", "SERVE_SNAPSHOT_PER_BATCH", "SERVE_SNAPSHOT_PER_REQUEST", "load",
]

LATEST = 0xFFFFFFFF
FRONTEND_AUTO, FRONTEND_UNSORTED, FRONTEND_SORTED = 0, 1, 2  # MVBT_FRONTEND_*
NOT_FOUND = 0xFFFFFFFF
pair_dtype_words = 2  # a result pair is two uint32 words {key, value}

_HERE = Path(__file__).resolve().parent
library_path = _HERE / "libmvbt.so"

if not library_path.exists():
    raise ImportError(
        f"{library_path} is missing: build it with `python mvgpubtree_b200/build.py` "
        "(the tree has no CPU implementation)")

lib = ctypes.CDLL(str(library_path))

_u32, _u64, _i32, _vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p


class mvbt_config(ctypes.Structure):
    _fields_ = [("pool_bytes", _u64), ("device", _i32), ("tile_width", _i32),
                ("block_size", _i32), ("spin_limit", _u32), ("chunk_nodes", _u32),
                ("blocks_per_sm", _u32), ("max_blocks", _u32), ("wait_ms", _u32),
                ("reclaim", _u32), ("frontend", _u32), ("reserved", _u32 * 2)]


class mvbt_report(ctypes.Structure):
    _fields_ = [("height", _u32), ("reserved0", _u32), ("keys", _u64), ("leaves", _u64),
                ("interior", _u64), ("nodes_allocated", _u64), ("key_checksum", _u64),
                ("locked_nodes", _u32), ("violations", _u32)]


class mvbt_device_view(ctypes.Structure):
    _fields_ = [("pool", _vp), ("control", _vp), ("versioned", _u32), ("capacity", _u32),
                ("reclaim", _u32), ("reserved", _u32)]


class mvbt_serve_config(ctypes.Structure):
    _fields_ = [("max_ops_per_launch", _u64), ("max_range_pairs", _u64),
                ("max_requests_per_launch", _u32), ("pipeline_depth", _u32), ("mode", _u32),
                ("reclaim_every", _u32), ("nodes_per_write", _u32), ("snapshots", _u32),
                ("reserve_nodes", _u64), ("reclaim_in_launch", _u32), ("pad0", _u32),
                ("max_reclaim_lag", _u64), ("reserved", _u64 * 2)]


class mvbt_serve_stats(ctypes.Structure):
    _fields_ = [(n, _u64) for n in ("requests", "ops", "launches", "reclaims", "span_ns", "max_waiting",
                                     "memory_waits", "max_launch_ops", "max_reclaim_lag", "lag_waits",
                                     "nodes_high_water")] + [("reserved", _u64 * 5)]


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_P = _vp
_sig("mvbt_config_init", None, ctypes.POINTER(mvbt_config))
_sig("mvbt_create", ctypes.c_int, ctypes.c_int, ctypes.POINTER(mvbt_config), ctypes.POINTER(_vp))
_sig("mvbt_destroy", ctypes.c_int, _vp)
_sig("mvbt_set_frontend", ctypes.c_int, _vp, _u32)
_sig("mvbt_insert", ctypes.c_int, _vp, _P, _P, _u32, _vp, ctypes.c_int)
_sig("mvbt_find", ctypes.c_int, _vp, _P, _P, _u32, _u32, _vp, ctypes.c_int)
_sig("mvbt_erase", ctypes.c_int, _vp, _P, _u32, _vp, ctypes.c_int)
_sig("mvbt_range_query", ctypes.c_int, _vp, _P, _P, _P, _P, _u32, _u32, _u32, _vp, ctypes.c_int)
_sig("mvbt_concurrent_insert_range", ctypes.c_int, _vp, _P, _P, _u32, _P, _P, _u32, _P, _u32, _P, _vp)
_sig("mvbt_concurrent_find_erase", ctypes.c_int, _vp, _P, _P, _u32, _P, _u32, _vp)
_sig("mvbt_take_snapshot", ctypes.c_int, _vp, _vp, ctypes.POINTER(_u32))
_sig("mvbt_take_snapshot_async", ctypes.c_int, _vp, _vp, _P)
_sig("mvbt_check_errors", ctypes.c_int, _vp, _vp, ctypes.POINTER(_u32))
_sig("mvbt_clear_errors", ctypes.c_int, _vp, _vp)
_sig("mvbt_memory_usage", ctypes.c_int, _vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64), ctypes.POINTER(_u64))
_sig("mvbt_validate", ctypes.c_int, _vp, _u32, ctypes.POINTER(mvbt_report))
_sig("mvbt_get_device_view", ctypes.c_int, _vp, ctypes.POINTER(mvbt_device_view))
_sig("mvbt_copy_pool", ctypes.c_int, _vp, _vp, _u64, ctypes.POINTER(_u64))
_sig("mvbt_validate_image", ctypes.c_int, _vp, _u64, ctypes.c_int, _u32, ctypes.POINTER(mvbt_report))
_sig("mvbt_validate_image_detail", ctypes.c_int, _vp, _u64, ctypes.c_int, _u32, ctypes.POINTER(mvbt_report),
     ctypes.c_char_p, _u64)
_sig("mvbt_get_info", ctypes.c_int, _vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
     ctypes.POINTER(ctypes.c_int))
_sig("mvbt_batch_plan_create", ctypes.c_int, _vp, _u64, _u32, ctypes.POINTER(_vp))
_sig("mvbt_batch_plan_destroy", ctypes.c_int, _vp)
_sig("mvbt_batch_run", ctypes.c_int, _vp, _u32, _vp, _P, _P, _P, _P, _P, _P, _P, ctypes.c_int, _vp)
_sig("mvbt_batch_plan_timing", ctypes.c_int, _vp, ctypes.c_int)
_sig("mvbt_batch_plan_set_reclaim", ctypes.c_int, _vp, ctypes.c_int, _u32)
_sig("mvbt_batch_plan_memory_series", ctypes.c_int, _vp, _vp, _u32, ctypes.POINTER(_u32))
_sig("mvbt_batch_plan_kernel_times", ctypes.c_int, _vp, ctypes.POINTER(ctypes.c_float), _u32,
     ctypes.POINTER(_u32))
_sig("mvbt_stats", ctypes.c_int, _vp, ctypes.POINTER(_u64), _u32)
_sig("mvbt_reclaim", ctypes.c_int, _vp, _u32, _vp)
_sig("mvbt_clone", ctypes.c_int, _vp, ctypes.POINTER(_vp))
_sig("mvbt_bulk_build", ctypes.c_int, _vp, _P, _P, _u64, _u32, _vp)
_sig("mvbt_save", ctypes.c_int, _vp, ctypes.c_char_p)
_sig("mvbt_load", ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_vp))
_sig("mvbt_batch_plan_set_launch", ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int)
_sig("mvbt_batch_compact_ranges", ctypes.c_int, _vp, _u64, _P, _P, _P, _P, _P, _P, _P, _vp)
_sig("mvbt_serve_config_init", None, ctypes.POINTER(mvbt_serve_config))
_sig("mvbt_serve_trace", ctypes.c_int, _vp, ctypes.POINTER(mvbt_serve_config), _u32, _vp, _vp, _vp, _vp,
     _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(mvbt_serve_stats))
_sig("mvbt_batch_run_noalloc", ctypes.c_int, _vp, _u32, _P, _u64, _P, _P, _P, _P, _P, _P, _P, _vp)
_sig("mvbt_last_error", ctypes.c_char_p)
_sig("mvbt_status_string", ctypes.c_char_p, ctypes.c_int)


class MVBTError(RuntimeError):
    """A C ABI call returned a non-zero status."""

    def __init__(self, status: int, where: str):
        self.status = status
        msg = lib.mvbt_status_string(status).decode()
        detail = lib.mvbt_last_error().decode()
        super().__init__(f"{where}: {msg} ({status}){': ' + detail if detail else ''}")


def _check(status: int, where: str) -> None:
    if status != 0:
        raise MVBTError(status, where)


PAIRS = 0  # word_bytes of a pair buffer: {key, value} uint32 pairs held in 4- or 8-byte elements


def _ptr(x, word_bytes: int = 4, name: str = "array"):
    """Device address of a CUDA tensor, a pinned host tensor or a raw pointer (int).

    word_bytes is the element size the C ABI reads through the pointer: 4 for uint32 arrays, 8 for
    uint64 arrays (offsets, totals; an integer dtype is required), PAIRS for pair buffers. A tensor
    of another element size is rejected: the kernels would read it with the wrong stride, past
    its end."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        es = x.element_size()
        if word_bytes == PAIRS:
            if es not in (4, 8):
                raise TypeError(f"{name}: a pair buffer needs 32- or 64-bit elements, got {es} bytes")
        elif es != word_bytes:
            raise TypeError(f"{name}: expected {8 * word_bytes}-bit elements, got {8 * es}-bit ones")
        if word_bytes == 8 and (x.is_floating_point() or x.is_complex()):
            raise TypeError(f"{name}: expected an integer dtype, got {x.dtype}")
        if not x.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
        if not x.is_cuda and not x.is_pinned():
            raise ValueError(f"{name} must be a CUDA tensor or pinned host memory; "
                             "pageable host memory cannot be read by the kernels")
        return x.data_ptr()
    raise TypeError(f"{name}: expected a torch tensor or an integer device pointer")


def _numel(x) -> int:
    return int(x.numel()) if hasattr(x, "numel") else 0


def _stream(stream) -> int:
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available() and torch.cuda.is_initialized():
                return int(torch.cuda.current_stream().cuda_stream)
        except Exception:
            pass
        return 0
    if isinstance(stream, int):
        return stream
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    raise TypeError("stream must be None, an int handle or a torch.cuda.Stream")


class _TreeBase:
    """Shared host methods of both trees (one handle owns one device tree)."""

    _kind = -1
    branching_factor = 16  # node pairs, as GpuBTree::*::branching_factor

    def __init__(self, pool_bytes: int = 4 << 30, tile_width: int = 8, device: int | None = None,
                 block_size: int = 256, spin_limit: int = 0, chunk_nodes: int = 0,
                 blocks_per_sm: int = 0, max_blocks: int = 0, wait_ms: int = 0,
                 reclaim: bool = False, frontend: int = 0):
        cfg = mvbt_config()
        lib.mvbt_config_init(ctypes.byref(cfg))
        cfg.pool_bytes = int(pool_bytes)
        cfg.tile_width = int(tile_width)
        cfg.block_size = int(block_size)
        cfg.device = -1 if device is None else int(device)
        cfg.spin_limit = int(spin_limit)
        cfg.chunk_nodes = int(chunk_nodes)
        cfg.blocks_per_sm = int(blocks_per_sm)
        cfg.max_blocks = int(max_blocks)
        if wait_ms:
            cfg.wait_ms = int(wait_ms)
        cfg.reclaim = 1 if reclaim else 0
        cfg.frontend = int(frontend)
        h = _vp()
        _check(lib.mvbt_create(self._kind, ctypes.byref(cfg), ctypes.byref(h)), "mvbt_create")
        self._h = h
        self.tile_width = int(tile_width)

    @classmethod
    def _adopt(cls, handle) -> "_TreeBase":
        """Wraps a tree handle the library created (clone, load)."""
        obj = cls.__new__(cls)
        obj._h = handle
        kind, w, dev = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib.mvbt_get_info(handle, ctypes.byref(kind), ctypes.byref(w), ctypes.byref(dev)), "get_info")
        obj.tile_width = int(w.value)
        return obj

    def bulk_build(self, keys, values, num_keys: int | None = None, fill: int = 0, stream=None) -> None:
        """Builds this fresh tree from pairs with keys sorted strictly increasing (device tensors);
        leaves hold `fill` pairs (0 = 8, half full, as the reference's bulk-build constructor,
        include/gpu_blink_tree.hpp:85-136)."""
        n = _numel(keys) if num_keys is None else int(num_keys)
        _check(lib.mvbt_bulk_build(self._h, _ptr(keys, name="keys"), _ptr(values, name="values"), n,
                                   int(fill), _stream(stream)), "bulk_build")

    def set_frontend(self, frontend: int) -> None:
        """Batch front-end of the bulk calls: FRONTEND_AUTO, FRONTEND_UNSORTED or FRONTEND_SORTED
        (sort the call's keys on the device and run each tile over a contiguous run of them)."""
        _check(lib.mvbt_set_frontend(self._h, int(frontend)), "set_frontend")

    def clone(self) -> "_TreeBase":
        """A copy of the tree (every version, allocator and reclamation state) with the same
        configuration; changing one leaves the other as it was."""
        h = _vp()
        _check(lib.mvbt_clone(self._h, ctypes.byref(h)), "clone")
        return type(self)._adopt(h)

    def save(self, path) -> None:
        """Checkpoint of the tree to a file (mvbt_save); load() restores it."""
        _check(lib.mvbt_save(self._h, str(path).encode()), "save")

    # -- lifetime --
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.mvbt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return int(self._h.value)

    # -- host bulk operations (reference: gpu_blink_tree.hpp:218-265) --
    def insert(self, keys, values, num_keys: int | None = None, stream=None, in_place: bool = True):
        n = _numel(keys) if num_keys is None else int(num_keys)
        _check(lib.mvbt_insert(self._h, _ptr(keys, name="keys"), _ptr(values, name="values"), n,
                               _stream(stream), int(bool(in_place))), "insert")

    def find(self, keys, values, num_keys: int | None = None, timestamp: int = LATEST, stream=None,
             concurrent: bool = False):
        n = _numel(keys) if num_keys is None else int(num_keys)
        _check(lib.mvbt_find(self._h, _ptr(keys, name="keys"), _ptr(values, name="values"), n,
                             int(timestamp), _stream(stream), int(bool(concurrent))), "find")

    def erase(self, keys, num_keys: int | None = None, stream=None, concurrent: bool = False):
        n = _numel(keys) if num_keys is None else int(num_keys)
        _check(lib.mvbt_erase(self._h, _ptr(keys, name="keys"), n, _stream(stream),
                              int(bool(concurrent))), "erase")

    def range_query(self, lower_bound, upper_bound, result, counts, average_range_length: int,
                    num_keys: int | None = None, timestamp: int = LATEST, stream=None,
                    concurrent: bool = False):
        n = _numel(lower_bound) if num_keys is None else int(num_keys)
        _check(lib.mvbt_range_query(self._h, _ptr(lower_bound, name="lower"), _ptr(upper_bound, name="upper"),
                                    _ptr(result, PAIRS, "result"), _ptr(counts, name="counts"),
                                    int(average_range_length), n, int(timestamp), _stream(stream),
                                    int(bool(concurrent))), "range_query")

    def concurrent_insert_range(self, keys, values, num_insertion: int, lower_bound, upper_bound,
                                num_ranges: int, result, average_range_length: int, counts=None,
                                stream=None):
        _check(lib.mvbt_concurrent_insert_range(
            self._h, _ptr(keys, name="keys"), _ptr(values, name="values"), int(num_insertion),
            _ptr(lower_bound, name="lower"), _ptr(upper_bound, name="upper"), int(num_ranges),
            _ptr(result, PAIRS, "result"), int(average_range_length), _ptr(counts, name="counts"),
            _stream(stream)), "concurrent_insert_range")

    def concurrent_find_erase(self, find_keys, find_results, num_finds: int, erase_keys,
                              num_erasures: int, stream=None):
        _check(lib.mvbt_concurrent_find_erase(
            self._h, _ptr(find_keys, name="find_keys"), _ptr(find_results, name="find_results"),
            int(num_finds), _ptr(erase_keys, name="erase_keys"), int(num_erasures), _stream(stream)),
            "concurrent_find_erase")

    # -- status, statistics, validation --
    def check_errors(self, stream=None, raise_on_error: bool = True) -> int:
        bits = _u32(0)
        st = lib.mvbt_check_errors(self._h, _stream(stream), ctypes.byref(bits))
        if st and raise_on_error:
            raise MVBTError(st, "device error")
        return int(bits.value)

    def clear_errors(self, stream=None) -> None:
        _check(lib.mvbt_clear_errors(self._h, _stream(stream)), "clear_errors")

    def compute_memory_usage(self) -> dict:
        a, b, c = _u64(), _u64(), _u64()
        _check(lib.mvbt_memory_usage(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "memory_usage")
        return {"nodes_allocated": a.value, "bytes_allocated": b.value, "pool_bytes": c.value}

    def validate_tree_structure(self, timestamp: int = LATEST, raise_on_error: bool = True) -> dict:
        rep = mvbt_report()
        st = lib.mvbt_validate(self._h, int(timestamp), ctypes.byref(rep))
        out = {f: getattr(rep, f) for f, _ in mvbt_report._fields_ if not f.startswith("reserved")}
        if st and raise_on_error:
            raise MVBTError(st, f"validate_tree_structure {out}")
        return out

    def validate_detail(self, timestamp: int = LATEST) -> tuple[dict, str]:
        """Host walk of a pool copy; returns the report and a description of the first violations."""
        img = self.copy_pool()
        rep = mvbt_report()
        buf = ctypes.create_string_buffer(8192)
        lib.mvbt_validate_image_detail(img.ctypes.data, img.shape[0], int(self._kind == 1),
                                       int(timestamp), ctypes.byref(rep), buf, 8192)
        out = {f: getattr(rep, f) for f, _ in mvbt_report._fields_ if not f.startswith("reserved")}
        return out, buf.value.decode()

    def copy_pool(self):
        """Host image of the allocated nodes: numpy uint32 array [nodes, 32]."""
        import numpy as np
        usage = self.compute_memory_usage()
        img = np.empty((int(usage["nodes_allocated"]), 32), np.uint32)
        n = _u64(0)
        _check(lib.mvbt_copy_pool(self._h, img.ctypes.data, img.shape[0], ctypes.byref(n)), "copy_pool")
        return img[: n.value]

    def stats(self) -> dict:
        """Device counters: versions copied, splits, longest walks, epoch, error bits per site."""
        buf = (_u64 * 43)()
        _check(lib.mvbt_stats(self._h, buf, 43), "stats")
        v = list(buf)
        sites = v[6:22] + v[27:43]
        return {"cow": v[0], "splits": v[1], "max_hops": v[2], "max_descent": v[3], "epoch": v[4],
                "error_bits": v[5], "error_sites": {i: x for i, x in enumerate(sites) if x},
                "restarts": v[22], "reclaimed": v[23], "free_nodes": v[24], "reused": v[25],
                "log_dropped": v[26]}

    def reclaim(self, min_live_snapshot: int = 0xFFFFFFFF, stream=None) -> None:
        """Frees version copies no snapshot id >= min_live_snapshot reads (RECLAIM_ALL: keep only
        the newest state and later snapshots). Stream-ordered; no writer may run concurrently.
        Needs reclaim=True at construction (reference: the DEBR reclaimer,
        include/memory_reclaimer.hpp:70-410)."""
        _check(lib.mvbt_reclaim(self._h, int(min_live_snapshot) & 0xFFFFFFFF, _stream(stream)), "reclaim")

    def device_view(self) -> mvbt_device_view:
        v = mvbt_device_view()
        _check(lib.mvbt_get_device_view(self._h, ctypes.byref(v)), "device_view")
        return v


class gpu_blink_tree(_TreeBase):
    """Plain concurrent B-link tree (reference: include/gpu_blink_tree.hpp:63-67)."""

    _kind = 0


class gpu_versioned_btree(_TreeBase):
    """Multiversion B-link tree with snapshots (reference: include/gpu_versioned_blink_tree.hpp:71-75)."""

    _kind = 1

    def take_snapshot(self, stream=None) -> int:
        """Takes a snapshot and returns its id; synchronises the stream (reference 297-302)."""
        ts = _u32(0)
        _check(lib.mvbt_take_snapshot(self._h, _stream(stream), ctypes.byref(ts)), "take_snapshot")
        return int(ts.value)

    def batch_plan(self, max_ops: int, max_batches: int) -> "BatchPlan":
        """Scratch for mixed op batches of up to max_ops ops in max_batches batches."""
        return BatchPlan(self, max_ops, max_batches)

    def batch_run_noalloc(self, batch_off, num_ops: int, type, key, arg, out_off, range_cap, result,
                          range_out, stream=None) -> None:
        """Mixed batches for callers that cannot allocate device memory on their call path (a
        latency-bound serving loop, a host that owns every allocation): the scratch lives in a
        fixed array inside the library, so this call allocates nothing. At most NOALLOC_MAX_OPS
        ops in NOALLOC_MAX_BATCHES batches; batch_off is a DEVICE tensor of num_batches + 1
        64-bit offsets. Calls that overlap on the GPU share the array and race."""
        if not hasattr(batch_off, "numel"):
            raise TypeError("batch_off must be a device tensor of num_batches + 1 offsets")
        _check(lib.mvbt_batch_run_noalloc(
            self._h, int(batch_off.numel()) - 1, _ptr(batch_off, 8, "batch_off"), int(num_ops),
            _ptr(type, name="type"), _ptr(key, name="key"), _ptr(arg, name="arg"),
            _ptr(out_off, 8, "out_off"), _ptr(range_cap, name="range_cap"),
            _ptr(result, name="result"), _ptr(range_out, PAIRS, "range_out"), _stream(stream)),
            "batch_run_noalloc")

    def serve(self, batches, arrival_ns, **config) -> dict:
        """Serving session over a trace (mvbt_serve_trace): request r is batch r of `batches`
        (workload.Batches, generated in one call so range slots increase) and
        arrives arrival_ns[r] after the session start. Config keys are the mvbt_serve_config
        fields (mode, snapshots: SERVE_SNAPSHOT_PER_BATCH or _PER_REQUEST, pipeline_depth,
        max_ops_per_launch, max_requests_per_launch, max_range_pairs, reclaim_every,
        nodes_per_write, reserve_nodes). Returns numpy arrays
        result (per op), range_out (pairs, uint32 [n, 2]), done_ns and snapshot (per request),
        and the stats as a dict. Host buffers are pinned when torch is available."""
        import numpy as np
        cfg = mvbt_serve_config()
        lib.mvbt_serve_config_init(ctypes.byref(cfg))
        for k, v in config.items():
            if not hasattr(cfg, k) or k.startswith("reserved"):
                raise ValueError(f"unknown serving option {k}")
            setattr(cfg, k, int(v))
        R = int(batches.num_batches)
        n = int(batches.num_ops)
        pairs = max(1, int(batches.range_pairs))
        try:
            import torch
            pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
            empty = lambda count, dt: torch.empty(count, dtype=dt).pin_memory()
            i32, i64 = torch.int32, torch.int64
            view = lambda t, dt: t.numpy().view(dt)
            addr = lambda t: t.data_ptr()
        except ImportError:  # pageable numpy buffers: the copies run synchronously
            pin = np.ascontiguousarray
            empty = lambda count, dt: np.empty(count, dt)
            i32, i64 = np.int32, np.int64
            view = lambda t, dt: t.view(dt)
            addr = lambda t: t.ctypes.data
        held = [pin(batches.batch_off.view(np.int64)), pin(np.asarray(arrival_ns, np.uint64).view(np.int64)),
                pin(batches.type.view(np.int32)), pin(batches.key.view(np.int32)),
                pin(batches.arg.view(np.int32)), pin(batches.out_off.view(np.int64)),
                pin(batches.range_cap.view(np.int32))]
        res, rout = empty(max(1, n), i32), empty(pairs * 2, i32)
        done, snap = empty(R, i64), empty(R, i32)
        st = mvbt_serve_stats()
        _check(lib.mvbt_serve_trace(self._h, ctypes.byref(cfg), R, *[addr(h) for h in held], addr(res),
                                    addr(rout), addr(done), addr(snap), ctypes.byref(st)), "serve_trace")
        stats = {f: int(getattr(st, f)) for f, _ in mvbt_serve_stats._fields_ if f != "reserved"}
        return {"result": view(res, np.uint32)[:n].copy(), "range_out": view(rout, np.uint32).reshape(-1, 2).copy(),
                "done_ns": view(done, np.uint64).copy(), "snapshot": view(snap, np.uint32).copy(),
                "stats": stats}

    def take_snapshot_async(self, d_out, stream=None) -> None:
        """Stream-ordered snapshot; writes the id to the device word d_out."""
        _check(lib.mvbt_take_snapshot_async(self._h, _stream(stream), _ptr(d_out, name="d_out")),
               "take_snapshot_async")


BATCH_PERSISTENT, BATCH_PER_LAUNCH, BATCH_GRAPH = 0, 1, 2


def load(path, device: int | None = None):
    """A tree restored from a file that save() wrote (mvbt_load), as gpu_blink_tree or
    gpu_versioned_btree."""
    h = _vp()
    _check(lib.mvbt_load(str(path).encode(), -1 if device is None else int(device), ctypes.byref(h)), "load")
    kind = ctypes.c_int()
    _check(lib.mvbt_get_info(h, ctypes.byref(kind), None, None), "get_info")
    return (gpu_versioned_btree if kind.value == 1 else gpu_blink_tree)._adopt(h)
NOALLOC_MAX_OPS, NOALLOC_MAX_BATCHES = 1 << 20, 1024  # MVBT_NOALLOC_MAX_OPS / _BATCHES
RECLAIM_ALL = 0xFFFFFFFF  # MVBT_RECLAIM_ALL
SERVE_SNAPSHOT_PER_BATCH, SERVE_SNAPSHOT_PER_REQUEST = 0, 1  # MVBT_SERVE_SNAPSHOT_*


class BatchPlan:
    """Device scratch and launch plan for running many mixed op batches on a versioned tree.

    run() takes the batch offsets as a host array (numpy uint64, num_batches + 1 entries) and the
    op arrays as device tensors: type/key/arg (uint32 words), out_off (64-bit), range_cap,
    result and range_out (pairs). mode: BATCH_PERSISTENT (one persistent launch fed by a device
    work queue), BATCH_GRAPH (that launch captured once and replayed as a CUDA graph) or
    BATCH_PER_LAUNCH (the plain method: one snapshot and one launch per batch).
    """

    def __init__(self, tree: "gpu_versioned_btree", max_ops: int, max_batches: int):
        h = _vp()
        _check(lib.mvbt_batch_plan_create(tree._h, int(max_ops), int(max_batches), ctypes.byref(h)),
               "batch_plan_create")
        self._h = h
        self.tree = tree  # keeps the tree alive while the plan exists
        self.max_batches = int(max_batches)

    def run(self, batch_off, type, key, arg, out_off, range_cap, result, range_out,
            mode: int = BATCH_PERSISTENT, stream=None):
        import numpy as np
        off = np.ascontiguousarray(batch_off, dtype=np.uint64)
        _check(lib.mvbt_batch_run(self._h, len(off) - 1, off.ctypes.data, _ptr(type, name="type"),
                                  _ptr(key, name="key"), _ptr(arg, name="arg"),
                                  _ptr(out_off, 8, "out_off"), _ptr(range_cap, name="range_cap"),
                                  _ptr(result, name="result"), _ptr(range_out, PAIRS, "range_out"),
                                  int(mode), _stream(stream)), "batch_run")

    def compact_ranges(self, num_ops: int, type, result, out_off, range_cap, range_out, compact, total,
                       stream=None) -> None:
        """Packs the first min(count, cap) pairs of every range query, in op order, into `compact`
        (a CUDA tensor or pinned host memory, which the kernel then writes directly) and the pair
        count into `total` (one 64-bit word). Query i's pairs start at the sum of min(count, cap)
        over the range queries before it."""
        _check(lib.mvbt_batch_compact_ranges(self._h, int(num_ops), _ptr(type, name="type"),
                                             _ptr(result, name="result"), _ptr(out_off, 8, "out_off"),
                                             _ptr(range_cap, name="range_cap"), _ptr(range_out, PAIRS, "range_out"),
                                             _ptr(compact, PAIRS, "compact"), _ptr(total, 8, "total"),
                                             _stream(stream)), "compact_ranges")

    def set_launch(self, tile_width: int = 0, blocks_per_sm: int = -1) -> None:
        """Launch shape of the persistent path: tile width 8 / 16 (0 = the tree's) and resident
        blocks per SM (-1 = the tree's, 0 = full occupancy, 4 / 6 / 8 = register-capped variants)."""
        _check(lib.mvbt_batch_plan_set_launch(self._h, int(tile_width), int(blocks_per_sm)), "set_launch")
        self.launch = (int(tile_width), int(blocks_per_sm))

    def set_reclaim(self, enable: bool = True, min_live_snapshot: int = 0xFFFFFFFF) -> None:
        """Reclamation inside this plan's persistent runs (the tree needs reclaim=True):
        min_live_snapshot is the oldest snapshot still read outside the runs (RECLAIM_ALL: none)."""
        _check(lib.mvbt_batch_plan_set_reclaim(self._h, int(bool(enable)), int(min_live_snapshot)), "set_reclaim")

    def memory_series(self):
        """Per batch of the last persistent run with reclamation on, sampled when its writes had
        finished: uint64 array [batches, 4] = epoch, nodes taken from the pool, freed nodes waiting
        in the free ring, nodes freed so far (live nodes = column 1 - column 2)."""
        import numpy as np
        out = np.zeros((self.max_batches, 4), np.uint64)
        n = _u32(0)
        _check(lib.mvbt_batch_plan_memory_series(self._h, out.ctypes.data, self.max_batches, ctypes.byref(n)),
               "memory_series")
        return out[: n.value]

    def enable_timing(self, on: bool = True) -> None:
        """CUDA events around the persistent kernel of each BATCH_PERSISTENT run."""
        _check(lib.mvbt_batch_plan_timing(self._h, int(bool(on))), "batch_plan_timing")

    def kernel_times(self) -> list:
        """Persistent-kernel times (ms) of the runs since the last call (waits for them)."""
        buf = (ctypes.c_float * 64)()
        n = _u32(0)
        _check(lib.mvbt_batch_plan_kernel_times(self._h, buf, 64, ctypes.byref(n)),
               "batch_plan_kernel_times")
        return [float(buf[i]) for i in range(n.value)]

    def close(self):
        if getattr(self, "_h", None):
            lib.mvbt_batch_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


gpu_versioned_blink_tree = gpu_versioned_btree
