"""CPU checks of the C ABI: the library builds for sm_100a, loads, and exports every
function include/green_b200.h declares (no device calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(gg_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from green_gpu_b200 import build, native
    path = build.build()
    return ctypes.CDLL(path), native


def test_header_declares_entry_points():
    names = _declared()
    for n in ("gg_create", "gg_gw_sigma", "gg_hf_fock", "gg_hf_exchange", "gg_symmetry_unfold"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    so, native = lib
    for n in _declared():
        assert hasattr(so, n), n
    assert sorted(native.EXPORTS) == sorted(_declared())


def test_version_string(lib):
    _, native = lib
    v = native.load().gg_version().decode()
    assert "sm_100a" in v


def test_create_without_device_reports_error(lib):
    _, native = lib
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    with pytest.raises(native.GreenError):
        native.Context(2, 2, 2, 2, 4, 1, 4, 3)


def test_bad_shape_rejected_before_device_use(lib):
    _, native = lib
    # odd nts is rejected by the shape check (gw_gpu_kernel.h:67) whatever the device state
    with pytest.raises(native.GreenError) as e:
        native.Context(2, 2, 2, 2, 4, 1, 5, 3)
    assert e.value.code == native.GG_ERR_ARG


def test_split_slice_default_is_the_same_everywhere():
    # library default, Python binding and both plugin mirrors agree on five slices: the smallest
    # count that keeps Sigma, P0 and K within 1e-8 of FP64 (four gives ~5e-8)
    txt = open(os.path.join(ROOT, "include", "green_b200.h")).read()
    m = re.search(r"#define\s+GG_DEFAULT_SPLIT_SLICES\s+(\d+)", txt)
    assert m and int(m.group(1)) == 5
    ctx_src = open(os.path.join(ROOT, "green_gpu_b200", "csrc", "context.cuh")).read()
    assert "int slices = GG_DEFAULT_SPLIT_SLICES;" in ctx_src
    from green_gpu_b200 import gpu_factory, native
    assert native.DEFAULT_SPLIT_SLICES == 5
    p = {}
    gpu_factory.custom_kernel_parameters(p)
    assert p["split_slices"] == 5
    drop_in = open(os.path.join(ROOT, "include", "green", "gpu", "gpu_factory.h")).read()
    assert "set_split_slices(GG_DEFAULT_SPLIT_SLICES)" in drop_in
