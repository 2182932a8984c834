"""tb_run_static, the entry point that allocates no device memory, against tb_run.

Callers whose device memory belongs to someone else (a framework's caching pool, a process
under a hard memory cap, code that must not allocate while it runs) use tb_run_static: one
world's device state is carved from the library's fixed area. Its results must be bit-exact
with the ordinary entry point's (the tolerance of every parity test here: none), call after
call, since every call reuses the same area. This file is collected last on purpose.
"""
import numpy as np
import pytest

from twins_b200 import api, workloads

pytestmark = pytest.mark.gpu


def test_static_run_equals_tb_run_twice(native_lib):
    w = workloads.c1()[0]
    est, done, _, _ = api.run_world(w.topo, w.flows, w.params)
    assert (done >= 0).all()
    for _ in range(2):  # the area keeps the previous call's contents: each call must clear it
        s_est, s_done, status = api.run_world_static(w.topo, w.flows, w.params)
        assert status == api.TB_OK
        assert np.array_equal(s_est, est)
        assert np.array_equal(s_done, done)


def test_static_run_allocates_nothing(native_lib):
    """Once a first call has loaded the library's module (and its fixed area) on the device, a
    further call leaves the device's free memory as it was: nothing is allocated for the world."""
    import torch
    w = workloads.c1()[0]
    api.run_world_static(w.topo, w.flows, w.params)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    s_est, s_done, status = api.run_world_static(w.topo, w.flows, w.params)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert status == api.TB_OK and (s_done >= 0).all()
    assert free0 - free1 <= 2 << 20, f"free device memory dropped by {free0 - free1} bytes"


def test_static_run_rejects_a_world_too_large(native_lib):
    w = workloads.c2_small()[1]  # a FatTree k=8 world needs more than the fixed area
    with pytest.raises(api.TwinsError) as e:
        api.run_world_static(w.topo, w.flows, w.params)
    assert e.value.code == -3
    assert "fixed area" in str(e.value)
