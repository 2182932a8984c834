"""Serving (continuous batching) on a B200: requests join a running batch between launches, and
every request's results and counters equal its standalone run.

The server's capacities are small on purpose, so that requests wait for room, join while others
are in the middle of their runs (at launch slots > 0), and reuse the entities and world slots of
finished ones.
"""
import numpy as np
import pytest

from conftest import GOLDEN
from twins_b200 import api, workloads

pytestmark = pytest.mark.gpu


def requests():
    rng = np.random.default_rng(11)
    out = []
    # FatTree k=4, DCTCP and Cubic
    for tcp, n in [("dctcp", 120), ("cubic", 80)]:
        flows = workloads.leafspine_flows(rng, 16, n, 0.4)
        flows.size = np.minimum(flows.size, 200_000)
        out.append((api.Topology.fattree(4), flows, api.TcpParams(tcp, 30, 200)))
    # leaf-spine, NewReno, FIN and spraying
    flows = workloads.leafspine_flows(rng, 64, 150, 0.5)
    flows.size = np.minimum(flows.size, 300_000)
    out.append((api.Topology.leafspine(4, 2, 16), flows,
                api.TcpParams("newreno", 20, 100, fin=True, spray=True, rng_seed=3, rng_run=2)))
    # a Jellyfish topology file with link failures and recoveries
    topo = api.Topology.from_file(GOLDEN / "topo" / "jf32.txt", "150000:s2:s10,300000:s15:s29,450000:s2:s10:up")
    flows = workloads.leafspine_flows(rng, topo.hosts, 100, 0.4)
    flows.size = np.minimum(flows.size, 250_000)
    out.append((topo, flows, api.TcpParams("dctcp", 40, 200, spray=True)))
    # FatTree k=8 with persistent connections
    flows = workloads.c2_flows(seed=5, n_msgs=200)
    flows.size = np.minimum(flows.size, 150_000)
    out.append((api.Topology.fattree(8), flows, api.TcpParams("dctcp", 30, 200, fin=True)))
    return out


def small_server():
    # room for about two of the requests at once
    return api.Server(worlds=2, hosts=200, switches=100, ports=900, connections=400, messages=400, sent_list_entries=1 << 20,
                      ooo_blocks=1 << 18, slots_per_launch=64)


def check(srv, reqs, ids):
    alone = [api.run_world(*r) for r in reqs]
    for (est, done, ctr, _), i in zip(alone, ids):
        e2, d2, c2 = srv.results(i)
        assert (est == e2).all() and (done == d2).all()
        assert (done >= 0).all()
        assert c2 == ctr


def test_serve_equals_standalone(native_lib):
    reqs = requests()
    with small_server() as srv:
        ids = [srv.submit(*r) for r in reqs[:2]]
        for _ in range(3):
            srv.step()
        ids += [srv.submit(*r) for r in reqs[2:]]
        while srv.step() or srv.stats()["queued"]:
            pass
        infos = [srv.info(i) for i in ids]
        assert all(x["state"] == 2 for x in infos)
        assert sum(x["slot0"] > 0 for x in infos) >= 3  # joined a batch that was running
        st = srv.stats()
        assert st["admitted"] == st["retired"] == len(reqs) and st["running"] == 0
        check(srv, reqs, ids)


def test_serve_background_loop(native_lib):
    """The server's own thread runs the rounds while requests arrive."""
    reqs = requests()
    with small_server() as srv:
        srv.start()
        ids = []
        for r in reqs:
            ids.append(srv.submit(*r))
        for i in ids:
            srv.wait(i, timeout_s=600)
        check(srv, reqs, ids)
        for i in ids:
            srv.release(i)
        assert srv.stats()["running"] == 0


def test_serve_rejects_what_never_fits(native_lib):
    with small_server() as srv:
        topo = api.Topology.fattree(16)
        flows = api.Flows.from_arrays([0], [1], [1000], [0])
        with pytest.raises(api.TwinsError):
            srv.submit(topo, flows, api.TcpParams("dctcp", 30, 200))
