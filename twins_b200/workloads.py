"""Seeded synthetic workloads of the benchmark configurations (numpy PCG64, explicit seeds).

    c1()  FatTree k=4, DCTCP (ecnK 30, queue 200), per-flow ECMP, one flow per connection, no FIN:
          all 240 ordered host pairs, sizes log-uniform in [1 KB, 1 MB] (whole bytes), starts per
          source host from Poisson arrivals at 30% offered load (about 1 ms).
    c2()  FatTree k=8, 10,000 flows between uniform random distinct pairs, sizes from a heavy-tailed
          web-search-like CDF (50% < 100 KB, mean ~1.6 MB, max 30 MB), Poisson starts at 50% load,
          25% of the connections carrying 4 messages (the conn column), FIN, per-packet spraying
          (RngSeed 1, RngRun 1); once per TCP (NewReno, DCTCP, Cubic).
    c4()  256 leaf-spine worlds (4..32 leaves, spines = leaves / 2, 16 hosts per leaf), each with a
          TCP, ecnK and queue limit from the sweep grid and 1,000..20,000 flows at 30..70% load.

The web-search-like CDF below is this project's own piecewise-linear distribution with the
stated shape; flow-size offsets are the gen.py conventions of the reference (sizes in bytes,
starts in ns, load = offered bytes / 100 Gbps host links).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .api import Flows, TcpParams, Topology

LINK_BYTES_PER_NS = 12.5  # 100 Gbps

# (bytes, cumulative probability): 50% below 100 KB, mean 1.62 MB, maximum 30 MB
WEB_CDF = [(1e3, 0.0), (1e4, 0.15), (2e4, 0.22), (5e4, 0.38), (1e5, 0.50), (3e5, 0.62), (1e6, 0.73),
           (3e6, 0.86), (1e7, 0.975), (3e7, 1.0)]


def web_sizes(rng: np.random.Generator, n: int) -> np.ndarray:
    """n sizes by inverse-CDF sampling with linear interpolation, whole bytes (>= 1)."""
    s = np.array([p[0] for p in WEB_CDF])
    c = np.array([p[1] for p in WEB_CDF])
    u = rng.random(n)
    return np.maximum(1, np.interp(u, c, s).astype(np.int64))


def web_mean() -> float:
    return sum((WEB_CDF[i][1] - WEB_CDF[i - 1][1]) * (WEB_CDF[i][0] + WEB_CDF[i - 1][0]) / 2 for i in range(1, len(WEB_CDF)))


@dataclass
class World:
    name: str
    topo: Topology
    flows: Flows
    params: TcpParams


def c1(seed: int = 1) -> list[World]:
    rng = np.random.default_rng(seed)
    topo = Topology.fattree(4)
    H = topo.hosts
    lo, hi = np.log(1e3), np.log(1e6)
    mean_size = (1e6 - 1e3) / (hi - lo)
    gap = mean_size / (0.3 * LINK_BYTES_PER_NS)  # ns between a host's starts at 30% load
    src, dst, size, start = [], [], [], []
    for s in range(H):
        others = [d for d in range(H) if d != s]
        rng.shuffle(others)
        t = 0.0
        for d in others:
            t += rng.exponential(gap)
            src.append(s)
            dst.append(d)
            size.append(int(np.floor(np.exp(rng.uniform(lo, hi)))))
            start.append(int(t))
    return [World("c1_k4_dctcp", topo, Flows.from_arrays(src, dst, size, start), TcpParams("dctcp", 30, 200))]


def c2_flows(seed: int = 1, n_msgs: int = 10000, k: int = 8, load: float = 0.5, reuse_share: float = 0.25,
             msgs_per_reuse: int = 4) -> Flows:
    rng = np.random.default_rng(seed)
    H = k ** 3 // 4
    # connections: a share carry msgs_per_reuse messages, the others one
    n_conn = int(round(n_msgs / (1 - reuse_share + reuse_share * msgs_per_reuse)))
    multi = rng.random(n_conn) < reuse_share
    counts = np.where(multi, msgs_per_reuse, 1)
    # trim / pad to exactly n_msgs messages
    while counts.sum() > n_msgs:
        i = int(rng.integers(n_conn))
        if counts[i] > 1:
            counts[i] -= 1
    while counts.sum() < n_msgs:
        counts = np.append(counts, 1)
    n_conn = len(counts)
    src = rng.integers(0, H, n_conn)
    dst = (src + rng.integers(1, H, n_conn)) % H  # distinct
    size = web_sizes(rng, n_msgs)
    rate = load * H * LINK_BYTES_PER_NS / web_mean()  # flows per ns, all hosts
    starts = np.cumsum(rng.exponential(1.0 / rate, n_msgs)).astype(np.int64)
    # the sorted arrival times go to connection slots in random order; a connection's messages
    # take their times in order
    owner = np.repeat(np.arange(n_conn), counts)
    rng.shuffle(owner)
    rows = sorted(range(n_msgs), key=lambda i: (starts[i], i))
    conn = owner[rows]
    return Flows.from_arrays(src[conn], dst[conn], size, starts[rows], conn)


def c2(seed: int = 1, tcps=("newreno", "dctcp", "cubic")) -> list[World]:
    topo = Topology.fattree(8)
    flows = c2_flows(seed)
    return [World(f"c2_k8_{t}", topo, flows, TcpParams(t, 30, 200, fin=True, spray=True, rng_seed=1, rng_run=1)) for t in tcps]


def leafspine_flows(rng: np.random.Generator, hosts: int, n: int, load: float) -> Flows:
    src = rng.integers(0, hosts, n)
    dst = (src + rng.integers(1, hosts, n)) % hosts
    size = web_sizes(rng, n)
    rate = load * hosts * LINK_BYTES_PER_NS / web_mean()
    start = np.cumsum(rng.exponential(1.0 / rate, n)).astype(np.int64)
    return Flows.from_arrays(src, dst, size, start)


def c4(seed: int = 1, n_worlds: int = 256, min_flows: int = 1000, max_flows: int = 20000) -> list[World]:
    rng = np.random.default_rng(seed)
    worlds = []
    for w in range(n_worlds):
        leaves = int(rng.choice(np.arange(4, 33, 2)))
        topo = Topology.leafspine(leaves, leaves // 2, 16)
        tcp = str(rng.choice(["newreno", "dctcp", "cubic"]))
        ecn_k = int(rng.choice([10, 20, 40, 80]))
        queue = int(rng.choice([100, 200, 400]))
        n = int(rng.integers(min_flows, max_flows + 1))
        load = float(rng.uniform(0.3, 0.7))
        flows = leafspine_flows(rng, topo.hosts, n, load)
        worlds.append(World(f"c4_{w:03d}_ls{leaves}_{tcp}_K{ecn_k}_q{queue}", topo, flows, TcpParams(tcp, ecn_k, queue)))
    return worlds


def c2_small(seed: int = 1, tcps=("newreno", "dctcp", "cubic")) -> list[World]:
    """The C2 shape at 1,500 messages (profiling and quick checks)."""
    topo = Topology.fattree(8)
    flows = c2_flows(seed, n_msgs=1500)
    return [World(f"c2s_k8_{t}", topo, flows, TcpParams(t, 30, 200, fin=True, spray=True, rng_seed=1, rng_run=1)) for t in tcps]


WORKLOADS = {"c1": c1, "c2": c2, "c2s": c2_small, "c4": c4}
