"""The C ABI without a GPU: the library loads, exports every entry point include/twinsb200.h
declares, builds worlds in a host-only context (device -1) with ns-3's ECMP hashes, and reports
bad input and missing devices as error codes (never by exiting)."""
import csv
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, manifest
from twins_b200 import api


def declared_entry_points():
    text = (ROOT / "include" / "twinsb200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(tb_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported(native_lib):
    names = declared_entry_points()
    assert len(names) >= 12
    lib = api.load_library(native_lib)
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(n for n, _, _ in api.ENTRY_POINTS) == names


def host_ctx(lib):
    import ctypes
    ctx = ctypes.c_void_p()
    assert lib.tb_ctx_create(-1, 0, ctypes.byref(ctx)) == api.TB_OK
    return ctx


def add_world(lib, ctx, topo, flows, params):
    import ctypes
    t, keep = topo._c()
    p = params._c()
    wid = ctypes.c_int(-1)
    r = lib.tb_world_add_tcp(ctx, ctypes.byref(t), len(flows), api._ptr(flows.src, ctypes.c_int), api._ptr(flows.dst, ctypes.c_int),
                             api._ptr(flows.size, ctypes.c_longlong), api._ptr(flows.start_ns, ctypes.c_longlong),
                             api._ptr(flows.conn, ctypes.c_longlong), None, None, ctypes.byref(p), ctypes.byref(wid))
    return r, wid.value


@pytest.mark.parametrize("case", [c for c in manifest() if c["variant"] in ("base", "spray") and c["tcp"] == "dctcp"],
                         ids=lambda c: c["name"])
def test_hashes_equal_ns3(native_lib, case):
    """ECMP hashes computed by the library for every connection equal ns-3's hash columns
    (reference validation/check_hashes.sh)."""
    import ctypes
    lib = api.load_library(native_lib)
    ctx = host_ctx(lib)
    topo = api.Topology.from_args(case["args"], base=GOLDEN)
    flows = api.Flows.load(GOLDEN / case["flows"], topo.hosts)
    r, w = add_world(lib, ctx, topo, flows, api.TcpParams.from_args(case["args"]))
    assert r == api.TB_OK, lib.tb_last_error()
    hd = np.zeros(len(flows), dtype=np.uint32)
    ha = np.zeros(len(flows), dtype=np.uint32)
    assert lib.tb_hashes(ctx, w, api._ptr(hd, ctypes.c_uint), api._ptr(ha, ctypes.c_uint)) == api.TB_OK
    with open(GOLDEN / case["ns3"]) as f:
        rows = list(csv.reader(f))[1:]
    assert [int(r[6]) for r in rows] == hd.tolist()
    assert [int(r[7]) for r in rows] == ha.tolist()
    # a host-only context cannot run
    assert lib.tb_run(ctx, 10) == -4
    lib.tb_ctx_destroy(ctx)


def test_bad_inputs_are_errors(native_lib):
    lib = api.load_library(native_lib)
    ctx = host_ctx(lib)
    topo = api.Topology.fattree(4)
    # a host out of range
    r, _ = add_world(lib, ctx, topo, api.Flows.from_arrays([0], [99], [1000], [0]), api.TcpParams())
    assert r == -1
    assert b"out of range" in lib.tb_last_error()
    # messages of one connection between different hosts
    r, _ = add_world(lib, ctx, topo, api.Flows.from_arrays([0, 1], [2, 2], [10, 10], [0, 5], [7, 7]), api.TcpParams())
    assert r == -1
    # a FatTree k that is not a power of two
    r, _ = add_world(lib, ctx, api.Topology.fattree(6), api.Flows.from_arrays([0], [1], [10], [0]), api.TcpParams())
    assert r == -1
    # an unreachable topology file (two islands)
    t = api.Topology(kind=api.TOPO_GRAPH, n_hosts=2, n_switches=2, links=[(0, -1), (1, -2)])
    r, _ = add_world(lib, ctx, t, api.Flows.from_arrays([0], [1], [10], [0]), api.TcpParams())
    assert r == -1 and b"cannot reach" in lib.tb_last_error()
    # results before any run
    import ctypes
    assert lib.tb_results(ctx, 0, None, None) in (-1, -4)
    lib.tb_ctx_destroy(ctx)


def test_no_device_is_an_error_not_an_exit(native_lib):
    import ctypes
    import torch
    lib = api.load_library(native_lib)
    ctx = ctypes.c_void_p()
    r = lib.tb_ctx_create(0, 0, ctypes.byref(ctx))
    if torch.cuda.is_available():
        assert r == api.TB_OK
        lib.tb_ctx_destroy(ctx)
    else:
        assert r == -2
        assert lib.tb_last_error()


def test_simulator_raises_without_library(tmp_path):
    with pytest.raises(FileNotFoundError):
        api.load_library(tmp_path / "missing.so")
