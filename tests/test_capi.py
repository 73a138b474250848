"""CPU tier: the C-ABI library loads, exports every declared symbol and validates arguments."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        if "namespace" in text:  # C++ wrapper headers (inline code over the C ABI) export nothing
            continue
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(mvbt_[a-z0-9_]+)\s*\(", text):
            names.append(m.group(1))
    return sorted(set(names))


def test_headers_declare_the_boundary():
    names = declared_functions()
    for required in ("mvbt_create", "mvbt_destroy", "mvbt_insert", "mvbt_find", "mvbt_erase",
                     "mvbt_range_query", "mvbt_concurrent_insert_range",
                     "mvbt_concurrent_find_erase", "mvbt_take_snapshot", "mvbt_validate"):
        assert required in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_symbol(name):
    import mvgpubtree_b200 as mv
    assert hasattr(mv.lib, name), f"{name} declared in include/*.h but not exported"


def test_status_strings_and_config_defaults():
    import mvgpubtree_b200 as mv
    assert mv.lib.mvbt_status_string(0) == b"ok"
    assert b"exhausted" in mv.lib.mvbt_status_string(3)
    cfg = mv.mvbt_config()
    mv.lib.mvbt_config_init(ctypes.byref(cfg))
    assert cfg.tile_width == 8 and cfg.block_size == 256 and cfg.pool_bytes == 4 << 30


def test_create_rejects_bad_arguments_without_touching_a_gpu():
    import mvgpubtree_b200 as mv
    h = ctypes.c_void_p()
    assert mv.lib.mvbt_create(7, None, ctypes.byref(h)) == 1  # bad kind
    cfg = mv.mvbt_config()
    mv.lib.mvbt_config_init(ctypes.byref(cfg))
    cfg.tile_width = 12
    assert mv.lib.mvbt_create(1, ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert b"tile_width" in mv.lib.mvbt_last_error()
    # null handles are rejected before any CUDA call
    assert mv.lib.mvbt_insert(None, None, None, 0, None, 1) == 1
    assert mv.lib.mvbt_find(None, None, None, 0, 0, None, 0) == 1


def test_pageable_host_memory_is_rejected():
    torch = pytest.importorskip("torch")
    import mvgpubtree_b200 as mv
    with pytest.raises(ValueError, match="pageable"):
        mv._ptr(torch.zeros(4, dtype=torch.int32))
    with pytest.raises(TypeError):
        mv._ptr([1, 2, 3])
    assert mv._ptr(1234) == 1234


def test_cpp_drop_in_header_compiles_and_links():
    """A reference-style C++ caller (tests/cpp/drop_in_example.cpp) builds against gpu_btree.h."""
    import sys
    sys.path.insert(0, str(ROOT / "tests" / "cpp"))
    from build import build
    exe = build()
    assert exe.exists()
