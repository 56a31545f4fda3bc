"""Serving-loop host surface on CPU: record layouts and argument checks that
fail before any device work."""
import ctypes

import pytest

import gatlas_b200 as g


def test_record_layouts_match_the_c_abi():
    assert g.request_dtype().itemsize == 72 and g.request_dtype().fields["arrival_ns"][1] == 64
    assert g.result_dtype().itemsize == 48 and g.result_dtype().fields["result"][1] == 32
    assert ctypes.sizeof(g.ServerConfig) == 32 and ctypes.sizeof(g.ServerStats) == 112


def test_create_rejects_bad_configurations():
    with pytest.raises(g.GatlasError, match="no grouped kernel"):
        g.Server(1 << 30, engine="tc_split6")
    with pytest.raises(g.GatlasError, match="budget"):
        g.Server(100)
