"""The C-ABI library builds, loads and exports every symbol of include/fbp_b200.h.
No GPU needed: only entry points that make no CUDA call are invoked."""
import ctypes
import os
import re

import pytest

from spikesorting_fullpursuit_b200 import build as B
from spikesorting_fullpursuit_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header="fbp_b200.h"):
    src = open(os.path.join(REPO, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char \*)\s*(fbp_\w+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return _lib.lib()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions() + declared_functions("fbp_prepost.h")
    assert len(names) >= 27
    for nm in names:
        assert hasattr(lib, nm), nm


def test_binding_table_covers_header():
    assert set(declared_functions()) == set(_lib.SIGNATURES)
    assert set(declared_functions("fbp_prepost.h")) == set(_lib.PREPOST_SIGNATURES)


def test_version_and_error_text(lib):
    assert lib.fbp_version() == 100
    assert lib.fbp_last_error() == b""


def test_workspace_size_is_host_only(lib):
    b = ctypes.c_size_t(0)
    assert lib.fbp_pursuit_workspace_bytes(1000, 4, 8, 31, 30, 0, ctypes.byref(b)) == 0
    # voltage-length likelihood for 8 templates dominates
    assert b.value >= 8 * 1000 * 4
    assert lib.fbp_pursuit_workspace_bytes(0, 4, 8, 31, 30, 0, ctypes.byref(b)) == _lib.FBP_ERR_BAD_ARG
    assert b"bad arguments" in lib.fbp_last_error()


def test_null_arguments_rejected_before_any_cuda_call(lib):
    n1, n2 = ctypes.c_uint32(0), ctypes.c_uint32(0)
    rc = lib.fbp_pursuit_chunk(None, 100, 4, None, 8, 31, None, None, 30, 1, 0, 0, 10, None, 0,
                               None, None, 0, None, ctypes.byref(n1), ctypes.byref(n2), 0, None, None)
    assert rc == _lib.FBP_ERR_BAD_ARG
    assert b"null pointer" in lib.fbp_last_error()


def test_scan_scratch(lib):
    assert lib.fbp_scan_scratch_bytes(4096) == 8
    assert lib.fbp_scan_scratch_bytes(4097) == 12


def test_test_limits_host_only(lib):
    _lib.set_test_limits(refine_list_cap=5, contender_pool_cap=7, wait_polls=0)
    _lib.reset_test_limits()
    assert lib.fbp_last_error() == b""


def test_bounds_entry_rejects_null_arguments(lib):
    rc = lib.fbp_tc_likelihood_bounds(None, 100, 4, None, 8, 31, None, None, 0, None, None, None)
    assert rc == _lib.FBP_ERR_BAD_ARG
    assert b"null pointer" in lib.fbp_last_error()


def test_plan_knobs_are_host_only_and_checked(lib):
    """The per-thread tensor-core plan knobs take their documented values and
    reject others with FBP_ERR_BAD_ARG, without touching a device."""
    for layout in (_lib.TC_LAYOUT_AUTO, _lib.TC_LAYOUT_SAMPLES, _lib.TC_LAYOUT_WIDE):
        assert lib.fbp_set_tc_layout(layout) == 0
    assert lib.fbp_set_tc_layout(3) == _lib.FBP_ERR_BAD_ARG
    assert b"unknown layout" in lib.fbp_last_error()
    assert lib.fbp_set_tc_layout(_lib.TC_LAYOUT_AUTO) == 0
    for gs in (0, 16, 32, 256):
        assert lib.fbp_set_tc_group_size(gs) == 0
    for gs in (8, 24, 272):
        assert lib.fbp_set_tc_group_size(gs) == _lib.FBP_ERR_BAD_ARG
    assert lib.fbp_set_tc_group_size(0) == 0
    assert lib.fbp_last_error() == b""
