"""Deterministic synthetic workloads (numpy front-end of workload/mvbt_workload.h).

The counterpart of the reference's key generator (include/rkg.hpp): distinct uniform keys in
[1, 2^32 - 3], values fmix32(key ^ salt), range bounds [k, k + L * stride) saturated at
0xFFFFFFFF, and the mixed erase/insert/find/range batch generator.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .build import LIB, build

if not LIB.exists():
    build()
lib = ctypes.CDLL(str(LIB))

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u64, _u32, _vp = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p

MISS_INDEX_BASE = 0x80000000
OP_FIND, OP_INSERT, OP_ERASE, OP_RANGE = 0, 1, 2, 3
KEY_DOMAIN_MAX = 0xFFFFFFFD  # keys are drawn from [1, 2^32 - 3]


class mvbt_mix_params(ctypes.Structure):
    _fields_ = [("p_erase", ctypes.c_double), ("p_insert", ctypes.c_double),
                ("p_find", ctypes.c_double), ("p_range", ctypes.c_double),
                ("find_hit", ctypes.c_double), ("batch_median", ctypes.c_double),
                ("batch_sigma", ctypes.c_double), ("batch_min", _u32), ("batch_max", _u32),
                ("range_mean", ctypes.c_double), ("range_min", _u32), ("range_max", _u32),
                ("stride", _u32), ("value_salt", _u32), ("fixed_batch", _u32),
                ("erase_lag", _u32), ("reserved", _u32 * 2)]


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)


_sig("mvbt_wl_splitmix64", _u64, ctypes.POINTER(_u64))
_sig("mvbt_wl_fmix32", _u32, _u32)
_sig("mvbt_wl_distinct_keys", None, _u64, _u64, _u64, _u32p)
_sig("mvbt_wl_values", None, _u32p, _u64, _u32, _u32p)
_sig("mvbt_wl_uniform_keys", None, _u64, _u64, _u32p)
_sig("mvbt_wl_shuffle", None, _u64, _u32p, _u64)
_sig("mvbt_wl_upper_bounds", None, _u32p, _u64, _u64, _u64, _u32p)
_sig("mvbt_wl_mix_default", None, ctypes.POINTER(mvbt_mix_params))
_sig("mvbt_wl_mix_create", _vp, ctypes.POINTER(mvbt_mix_params), _u64, _u64)
_sig("mvbt_wl_mix_destroy", None, _vp)
_sig("mvbt_wl_mix_generate", _u64, _vp, _u32, ctypes.POINTER(_u64))
_sig("mvbt_wl_mix_copy", None, _vp, _u64p, _u32p, _u32p, _u32p, _u64p, _u32p)
_sig("mvbt_wl_mix_present", _u64, _vp)


def fmix32(h: int) -> int:
    return int(lib.mvbt_wl_fmix32(h & 0xFFFFFFFF))


def distinct_keys(seed: int, start: int, n: int) -> np.ndarray:
    out = np.empty(n, np.uint32)
    if n:
        lib.mvbt_wl_distinct_keys(seed, start, n, out)
    return out


def values_for(keys: np.ndarray, salt: int) -> np.ndarray:
    keys = np.ascontiguousarray(keys, np.uint32)
    out = np.empty_like(keys)
    if keys.size:
        lib.mvbt_wl_values(keys, keys.size, salt & 0xFFFFFFFF, out)
    return out


def uniform_keys(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.uint32)
    if n:
        lib.mvbt_wl_uniform_keys(seed, n, out)
    return out


def shuffle(seed: int, a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, np.uint32).copy()
    if a.size:
        lib.mvbt_wl_shuffle(seed, a, a.size)
    return a


def upper_bounds(lower: np.ndarray, length: int, stride: int) -> np.ndarray:
    lower = np.ascontiguousarray(lower, np.uint32)
    out = np.empty_like(lower)
    if lower.size:
        lib.mvbt_wl_upper_bounds(lower, lower.size, int(length), int(stride), out)
    return out


def stride_for(num_keys: int) -> int:
    """floor((2^32 - 3) / num_keys): key spacing that makes a range of length L hold ~L keys."""
    return KEY_DOMAIN_MAX // max(1, int(num_keys))


def mix_params(**overrides) -> mvbt_mix_params:
    p = mvbt_mix_params()
    lib.mvbt_wl_mix_default(ctypes.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


@dataclass
class Batches:
    """num_batches batches of mixed ops; batch b holds ops [batch_off[b], batch_off[b+1])."""

    batch_off: np.ndarray  # uint64 [B + 1]
    type: np.ndarray       # uint32 [n] OP_*
    key: np.ndarray        # uint32 [n] key or lower bound
    arg: np.ndarray        # uint32 [n] value (insert) or upper bound (range)
    out_off: np.ndarray    # uint64 [n] range output offset in pairs
    range_cap: np.ndarray  # uint32 [n] range output capacity in pairs
    range_pairs: int       # total range output capacity in pairs

    @property
    def num_batches(self) -> int:
        return len(self.batch_off) - 1

    @property
    def num_ops(self) -> int:
        return int(self.batch_off[-1])


class MixGenerator:
    """Stateful generator of mixed batches over a present-key set (initial keys = distinct keys
    [0, initial_keys) of `seed`): erases hit present keys, inserts are new keys, finds hit present
    keys with probability find_hit (else never-inserted keys), ranges are [k, k + L * stride)."""

    def __init__(self, seed: int, initial_keys: int, **params):
        self.params = mix_params(**params)
        self._h = lib.mvbt_wl_mix_create(ctypes.byref(self.params), seed, initial_keys)

    def generate(self, num_batches: int) -> Batches:
        rp = _u64(0)
        n = int(lib.mvbt_wl_mix_generate(self._h, num_batches, ctypes.byref(rp)))
        b = Batches(np.empty(num_batches + 1, np.uint64), np.empty(n, np.uint32),
                    np.empty(n, np.uint32), np.empty(n, np.uint32), np.empty(n, np.uint64),
                    np.empty(n, np.uint32), int(rp.value))
        lib.mvbt_wl_mix_copy(self._h, b.batch_off, b.type, b.key, b.arg, b.out_off, b.range_cap)
        return b

    @property
    def present(self) -> int:
        return int(lib.mvbt_wl_mix_present(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib.mvbt_wl_mix_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def serving_generator(seed: int, initial_keys: int, stride: int, batch_median: float = 256.0,
                      batch_sigma: float = 1.5, batch_min: int = 1, batch_max: int = 65536,
                      erase_lag: int = 4096):
    """Request generator of the serving workload (the batched mix; request sizes lognormal,
    median 256 ops, clipped [1, 64K]) over the distinct keys [0, initial_keys) of `seed`. A key a
    request inserts can be erased (or picked as a find hit) only erase_lag requests later, more
    than one launch admits, so requests that share a snapshot never write the same key."""
    return MixGenerator(seed, initial_keys, stride=stride, batch_median=float(batch_median),
                        batch_sigma=float(batch_sigma), batch_min=int(batch_min), batch_max=int(batch_max),
                        erase_lag=int(erase_lag))


def serving_trace(seed: int, initial_keys: int, num_requests: int, offered_mops: float, stride: int,
                  batch_median: float = 256.0, batch_sigma: float = 1.5, batch_min: int = 1,
                  batch_max: int = 65536, generator: "MixGenerator | None" = None,
                  erase_lag: int = 4096):
    """Requests for a serving session: num_requests mixed batches from `generator` (default: a new
    serving_generator over the distinct keys [0, initial_keys) of `seed`; pass one to continue a
    key set across sessions), and Poisson arrival times (ns from the session start, the first at
    0) at an offered load of offered_mops million ops per second (request rate = load / mean
    request size). Returns (Batches, arrival_ns)."""
    gen = generator or serving_generator(seed, initial_keys, stride, batch_median, batch_sigma,
                                         batch_min, batch_max, erase_lag)
    b = gen.generate(int(num_requests))
    if generator is None:
        gen.close()
    sizes = np.diff(b.batch_off.astype(np.int64))
    mean = max(1.0, float(sizes.mean()))
    rate_per_ns = offered_mops * 1e6 / mean / 1e9
    rng = np.random.default_rng(seed ^ 0x5E12)
    gaps = rng.exponential(1.0 / rate_per_ns, int(num_requests))
    gaps[0] = 0.0
    return b, np.cumsum(gaps).astype(np.uint64)
