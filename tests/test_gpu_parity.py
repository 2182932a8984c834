"""Parity of the CUDA path (through the C ABI) on a B200.

- every golden case: each flow's established / completed time bit-exact with sequential ns-3
  (the stored outputs the reference and the oracle equal);
- batching: many golden worlds of different topologies and TCPs in one launch, each equal to
  its standalone result;
- seeded synthetic workloads of the benchmark shapes (FatTree k=4 C1; a reduced k=8 C2 with
  FIN, spraying and persistent connections, per TCP) against the CPU oracle, bit-exact;
- run statistics: the packet-event count equals the oracle's.
"""
import csv
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, manifest
from twins_b200 import api, workloads

pytestmark = pytest.mark.gpu

CASES = manifest()


def ns3(case):
    with open(GOLDEN / case["ns3"]) as f:
        rows = list(csv.reader(f))[1:]
    return np.array([int(r[4]) for r in rows]), np.array([int(r[5]) for r in rows])


def world_of(case):
    topo = api.Topology.from_args(case["args"], base=GOLDEN)
    flows = api.Flows.load(GOLDEN / case["flows"], topo.hosts)
    return topo, flows, api.TcpParams.from_args(case["args"], case["tcp"])


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_golden_case_bit_exact(native_lib, case):
    topo, flows, params = world_of(case)
    est, done, ctr, stats = api.run_world(topo, flows, params)
    want_est, want_done = ns3(case)
    bad = np.nonzero((est != want_est) | (done != want_done))[0]
    assert len(bad) == 0, f"{len(bad)} of {len(flows)} flows differ, first row {bad[0]}"
    assert ctr["ovf_active"] + ctr["ovf_due"] + ctr["ovf_ring"] + ctr["ovf_ooo"] + ctr["ovf_tx"] == 0
    assert stats["packet_events"] > 0


def test_batch_equals_standalone(native_lib):
    """Worlds of different topologies (FatTree, leaf-spine, Jellyfish with failures, Dragonfly)
    and TCPs in one batch: each equal to ns-3 (as standalone)."""
    picks = [c for c in CASES if c["workload"] not in ("k8_a2a50s", "k16_a2a30")][::3]
    with api.Simulator() as sim:
        ids = [sim.add_world(*world_of(c)) for c in picks]
        sim.run()
        for c, w in zip(picks, ids):
            est, done = sim.results(w)
            want_est, want_done = ns3(c)
            assert (est == want_est).all() and (done == want_done).all(), c["name"]


def oracle_run(oracle_bin, tmp_path, w, extra=()):
    path = tmp_path / f"{w.name}.csv"
    w.flows.write_csv(path)
    out = tmp_path / f"{w.name}.out.csv"
    topo = [f"--k={w.topo.k}"] if w.topo.kind == api.TOPO_FATTREE else \
        [f"--topo=leafspine", f"--leaves={w.topo.leaves}", f"--spines={w.topo.spines}", f"--hpl={w.topo.hpl}"]
    p = w.params
    cmd = [str(oracle_bin), *topo, f"--flows={path}", f"--out={out}", f"--tcp={p.tcp}", f"--ecnK={p.ecn_k}", f"--queue={p.queue}",
           f"--fin={int(p.fin)}", f"--spray={int(p.spray)}", f"--RngSeed={p.rng_seed}", f"--RngRun={p.rng_run}", *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, check=True)
    with open(out) as f:
        rows = list(csv.reader(f))[1:]
    events = int(r.stdout.split(" events ")[1].split()[0])
    return np.array([int(x[4]) for x in rows]), np.array([int(x[5]) for x in rows]), events


def test_c1_equals_oracle(native_lib, oracle_bin, tmp_path):
    w = workloads.c1()[0]
    want_est, want_done, events = oracle_run(oracle_bin, tmp_path, w)
    est, done, ctr, stats = api.run_world(w.topo, w.flows, w.params)
    assert (est == want_est).all() and (done == want_done).all()
    assert (done >= 0).all()
    assert stats["packet_events"] == events
    assert stats["graph_launches"] >= 1  # (the steady launches replay a captured CUDA graph)


@pytest.mark.parametrize("tcp", ["newreno", "dctcp", "cubic"])
def test_c2_reduced_equals_oracle(native_lib, oracle_bin, tmp_path, tcp):
    """The C2 shape (k=8, web-search-like sizes, persistent connections, FIN, spraying) at 1,500
    messages, per TCP."""
    flows = workloads.c2_flows(seed=3, n_msgs=1500)
    w = workloads.World(f"c2r_{tcp}", api.Topology.fattree(8), flows,
                        api.TcpParams(tcp, 30, 200, fin=True, spray=True, rng_seed=1, rng_run=1))
    want_est, want_done, events = oracle_run(oracle_bin, tmp_path, w)
    est, done, ctr, stats = api.run_world(w.topo, w.flows, w.params)
    assert (est == want_est).all() and (done == want_done).all()
    assert stats["packet_events"] == events


def test_repeated_runs_identical(native_lib):
    """tb_reset restores the initial state: a second run gives the same results and counts."""
    case = next(c for c in CASES if c["name"] == "k8_a2a30_cubic_spray")
    with api.Simulator() as sim:
        w = sim.add_world(*world_of(case))
        sim.run()
        a = sim.results(w)
        ea = sim.stats()["packet_events"]
        sim.run()
        b = sim.results(w)
        assert (a[0] == b[0]).all() and (a[1] == b[1]).all()
        assert sim.stats()["packet_events"] == ea


def test_max_slots_stops_early(native_lib):
    """max_slots ends the run at that simulated time; unfinished flows read -1."""
    w = workloads.c1()[0]
    with api.Simulator() as sim:
        i = sim.add_world(w.topo, w.flows, w.params)
        sim.run(max_slots=300)
        est, done = sim.results(i)
        st = sim.stats()
        assert st["slots"] <= 300
        assert (done == -1).any()


@pytest.mark.parametrize("name", ["k8_a2a30_dctcp_spray", "k8_r30_cubic_sprayfin", "jf32f_a2a50_newreno_spray"])
def test_launch_shapes_identical(native_lib, name):
    """Every launch shape (hosts per warp, frames staged per warp: 8 leaves most slots unstaged;
    switch egress with or without the ports' slot copies) gives the same results and event counts
    as ns-3 and as each other."""
    case = next(c for c in CASES if c["name"] == name)
    want_est, want_done = ns3(case)
    events = set()
    for lanes, stage, pl in [(1, 192, 0), (1, 8, 0), (1, 96, 0), (1, 384, 0), (4, 96, 0), (32, 192, 0), (7, 64, 0), (1, 384, 1),
                             (1, 8, 1), (32, 96, 1)]:
        est, done, ctr, stats = api.run_world(*world_of(case), host_lanes=lanes, stage_frames=stage, port_local=bool(pl))
        assert (est == want_est).all() and (done == want_done).all(), (lanes, stage, pl)
        assert stats["host_lanes"] == lanes and stats["stage_frames"] == stage and not stats["autotuned"]
        assert stats["port_local"] == (pl and lanes == 1)  # (several hosts per warp: the plain egress)
        events.add(stats["packet_events"])
    assert len(events) == 1


def test_batch_worlds_finish_apart(native_lib):
    """Leaf-spine worlds of different sizes, TCPs and lengths in one batch (the batched-sweep
    shape, small): each world stops when its last message is done, so its results and all its
    counters equal its standalone run."""
    rng = np.random.default_rng(7)
    worlds = []
    for i, (leaves, tcp, n) in enumerate([(4, "dctcp", 300), (6, "cubic", 60), (4, "newreno", 900), (8, "dctcp", 150)]):
        topo = api.Topology.leafspine(leaves, leaves // 2, 16)
        flows = workloads.leafspine_flows(rng, topo.hosts, n, 0.4)
        flows.size = np.minimum(flows.size, 300_000)
        worlds.append((topo, flows, api.TcpParams(tcp, [10, 20, 40, 80][i], [100, 200, 400, 100][i])))
    alone = [api.run_world(*w) for w in worlds]
    with api.Simulator() as sim:
        ids = [sim.add_world(*w) for w in worlds]
        sim.run()
        for (est, done, ctr, _), i in zip(alone, ids):
            e2, d2 = sim.results(i)
            assert (est == e2).all() and (done == d2).all()
            assert (done >= 0).all()
            assert sim.counters(i) == ctr


@pytest.mark.parametrize("lanes,port_local", [(None, False), (1, False), (1, True), (32, False)])
def test_free_batches_equal_lockstep(native_lib, lanes, port_local):
    """A batch whose worlds each run on a barrier of their own (the default) gives what one
    grid-wide barrier per slot gives: every world's results and counters, the batch's last slot;
    autotuned and for each fixed launch shape; and a run cut at 2,000 slots cuts every world
    there."""
    rng = np.random.default_rng(11)
    worlds = []
    for i, (leaves, tcp, n) in enumerate([(4, "cubic", 200), (8, "dctcp", 120), (4, "newreno", 500), (6, "dctcp", 40), (4, "dctcp", 0)]):
        topo = api.Topology.leafspine(leaves, leaves // 2, 16)
        flows = workloads.leafspine_flows(rng, topo.hosts, n, 0.5) if n else api.Flows.from_arrays([], [], [], [])
        if n:
            flows.size = np.minimum(flows.size, 200_000)
        worlds.append((topo, flows, api.TcpParams(tcp, [20, 40, 10, 80, 20][i], [200, 100, 400, 200, 100][i])))
    for max_slots in (0, 2000):
        got = {}
        for free in (True, False):
            kw = {} if lanes is None else {"host_lanes": lanes, "port_local": port_local}
            with api.Simulator(free_batches=free, **kw) as sim:
                ids = [sim.add_world(*w) for w in worlds]
                sim.run(max_slots)
                got[free] = ([sim.results(i) for i in ids], [sim.counters(i) for i in ids], sim.stats()["slots"])
        (ra, ca, sa), (rb, cb, sb) = got[True], got[False]
        assert all((x[0] == y[0]).all() and (x[1] == y[1]).all() for x, y in zip(ra, rb))
        assert ca == cb
        assert sa == sb
        if max_slots:
            assert sa == max_slots and any((x[1] < 0).any() for x in ra)


@pytest.mark.parametrize("name", ["k8_a2a30_cubic_spray", "k8_r30_dctcp_sprayfin", "df4x9_a2a30_newreno_spray"])
def test_chain_runs_25(native_lib, name):
    """The 25-run event-chain build (the reference's twins128, 128-byte frames) gives the same
    results as ns-3 and decides every tie."""
    case = next(c for c in CASES if c["name"] == name)
    est, done, ctr, stats = api.run_world(*world_of(case), chain_runs=25)
    want_est, want_done = ns3(case)
    assert (est == want_est).all() and (done == want_done).all()
    assert ctr["undecided_ties"] == 0


def test_edge_worlds(native_lib, oracle_bin, tmp_path):
    """Edge cases in one batch and alone: a world without flows, a single flow that starts 5 ms
    in (the idle skip jumps there), a one-byte flow, and a normal small world. Each equals its
    standalone run; the single flows equal the oracle."""
    empty = api.Flows.from_arrays([], [], [], [])
    late = api.Flows.from_arrays([3], [12], [150_000], [5_000_000])
    tiny = api.Flows.from_arrays([0, 5], [9, 0], [1, 2], [1_000, 1_000])
    small = workloads.c1()[0].flows
    topo = api.Topology.fattree(4)
    p = api.TcpParams("dctcp", 30, 200)
    worlds = [(topo, empty, p), (topo, late, p), (topo, tiny, api.TcpParams("cubic", 30, 200, fin=True)), (topo, small, p)]
    alone = [api.run_world(*w) for w in worlds]
    assert len(alone[0][0]) == 0
    for i in (1, 2):
        w = workloads.World(f"edge{i}", topo, worlds[i][1], worlds[i][2])
        want_est, want_done, _ = oracle_run(oracle_bin, tmp_path, w)
        assert (alone[i][0] == want_est).all() and (alone[i][1] == want_done).all()
        assert (alone[i][1] >= 0).all()
    with api.Simulator() as sim:
        ids = [sim.add_world(*w) for w in worlds]
        sim.run()
        for (est, done, ctr, _), i in zip(alone, ids):
            e2, d2 = sim.results(i)
            assert (est == e2).all() and (done == d2).all()
