"""The C ABI library loads and exports what include/bt.h declares (no GPU)."""
import ctypes
import os
import re

import pytest

import bundling_thingy_b200 as bt

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "bt.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bt_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name


def test_bindings_cover_the_header(lib):
    assert set(declared_functions()) == set(bt.SIGNATURES)


def test_abi_version(lib):
    header = open(HEADER).read()
    version = int(re.search(r"#define BT_ABI_VERSION (\d+)", header).group(1))
    assert lib.bt_abi_version() == version
    # The ctypes mirrors keep the C layouts (no padding holes in either).
    assert ctypes.sizeof(bt._Options) == 96
    assert ctypes.sizeof(bt._Info) == 64
    assert ctypes.sizeof(bt._ServerOptions) == 48
    assert bt._ServerOptions.reserve_bytes.offset == 24
    assert bt._Options.wait_seconds.offset == 88


def test_options_defaults_match_reference(lib):
    o = bt._Options()
    lib.bt_options_init(ctypes.byref(o))
    assert (o.width, o.height) == (1600, 1600)            # gpu.rs:21
    assert o.max_graph_memory_bytes == 1024 * 1024 * 1024   # main.rs:87-89
    assert o.color_by == bt.COLOR_BY_DENSITY and o.neighbor_radius == 0
    assert o.use_graphs == 1


@pytest.mark.parametrize(
    "field,value,message",
    [
        ("width", 0, "dimensions must be nonzero"),
        ("height", 40000, "texture limits"),
        ("max_graph_memory_bytes", 0, "budget must be nonzero"),
        ("blur_sigma", 100.0, "blur sigma"),
        ("sample_spacing", -1.0, "spacing"),
        ("wait_seconds", -1.0, "wait_seconds"),
        ("wait_seconds", float("inf"), "wait_seconds"),
    ],
)
def test_create_rejects_invalid_options_before_touching_cuda(lib, field, value, message):
    o = bt._Options()
    lib.bt_options_init(ctypes.byref(o))
    setattr(o, field, value)
    h = ctypes.c_void_p()
    status = lib.bt_create(ctypes.byref(o), ctypes.byref(h))
    assert status == 3
    assert message in lib.bt_last_error(None).decode()
    assert not h.value


def test_budget_check_mirrors_resampler_new(lib):
    # resampling.rs:85-89: grid + staging must stay below the budget.
    o = bt._Options()
    lib.bt_options_init(ctypes.byref(o))
    o.neighbor_radius = 1
    o.max_graph_memory_bytes = 1 << 20
    h = ctypes.c_void_p()
    assert lib.bt_create(ctypes.byref(o), ctypes.byref(h)) == 5
    assert "exceed --max-graph-memory-mib" in lib.bt_last_error(None).decode()


def test_null_arguments_are_errors(lib):
    assert lib.bt_create(None, None) == 3
    assert lib.bt_upload(None, None, 0, None, 0, None) == 3
    assert lib.bt_iterate(None, 1) == 3
    lib.bt_destroy(None)
