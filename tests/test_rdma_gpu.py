"""The RDMA model on a B200 through the C ABI (tb_world_add_rdma, tb_run, tb_rdma_results,
tb_counters): every fixture world of tests/golden/rdma/ (the flow completion times and counters the
reference's twins-rdma gives for them: FatTree k=4 and k=8 and a leaf-spine under DCQCN, HPCC and
DCTCP, incasts with ECN marks, PFC pauses with small buffers, flows that start together) must be
identical, flow for flow, and so must its counters line; worlds batched in one launch must equal
their runs alone."""
import json

import numpy as np
import pytest

from conftest import GOLDEN
from twins_b200 import api

pytestmark = pytest.mark.gpu

RDMA = GOLDEN / "rdma"
CASES = json.loads((RDMA / "manifest.json").read_text())


def inputs(name):
    topo = (RDMA / f"{name}.topo").read_text()
    hosts = int(topo.split()[1])
    return (RDMA / f"{name}.cfg").read_text(), topo, api.Flows.load(RDMA / f"{name}.csv", hosts)


def want(name, n):
    out = np.full(n, -1, dtype=np.int64)
    for line in (RDMA / f"{name}.fct").read_text().splitlines():
        if line.strip():
            i, _, f = (int(x) for x in line.split())
            out[i] = f
    return out


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_rdma_world_equals_reference(native_lib, case):
    cfg, topo, flows = inputs(case["name"])
    start, fct, ev, stats, status = api.run_rdma_world(cfg, topo, flows)
    w = want(case["name"], len(flows))
    bad = np.nonzero(fct != w)[0]
    assert len(bad) == 0, f"{len(bad)} of {len(w)} flows differ, first {bad[0]}: {fct[bad[0]]} vs {w[bad[0]]}"
    assert (start == flows.start_ns).all()
    assert api.rdma_counters_line(ev) == case["counters"]
    assert status == api.TB_OK
    assert stats["packet_events"] > 0 and stats["switch_events"] > 0


def test_rdma_batch_equals_alone(native_lib):
    """All fixture worlds (different topologies, sizes and congestion controls) in one launch."""
    with api.Simulator() as sim:
        ids = [sim.add_rdma_world(*inputs(c["name"])) for c in CASES]
        assert sim.run() == api.TB_OK
        for c, i in zip(CASES, ids):
            _, fct = sim.rdma_results(i)
            assert (fct == want(c["name"], len(fct))).all(), c["name"]


def test_rdma_refusals(native_lib):
    """A context holds TCP or RDMA worlds, not both; the reference's refusals come back as errors."""
    cfg, topo, flows = inputs("ft4_incast15_hpcc")
    with api.Simulator() as sim:
        sim.add_rdma_world(cfg, topo, flows)
        with pytest.raises(api.TwinsError):
            sim.add_world(api.Topology.fattree(4), flows, api.TcpParams())
    with api.Simulator() as sim:
        with pytest.raises(api.TwinsError) as e:
            sim.add_rdma_world(cfg.replace("CC_MODE 3", "CC_MODE 2"), topo, flows)
        assert "CC_MODE" in str(e.value)
