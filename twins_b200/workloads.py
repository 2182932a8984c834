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

from .api import TOPO_GRAPH, Flows, TcpParams, Topology

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


def c4_small(seed: int = 1) -> list[World]:
    """C4's shape at a profiler's size: 32 leaf-spine worlds of 500-3,000 flows."""
    return c4(seed, n_worlds=32, min_flows=500, max_flows=3000)


WORKLOADS = {"c1": c1, "c2": c2, "c2s": c2_small, "c4": c4, "c4s": c4_small}


# ------------------------------------------------------------------ served stream (C5 shape)
def jellyfish(n_sw: int = 64, degree: int = 8, hosts_per_sw: int = 4, seed: int = 1) -> Topology:
    """A seeded random regular graph of switches (each with `degree` switch links) and
    `hosts_per_sw` hosts on every switch, as a topology file's links (host h: h, switch j: -1-j).
    Jellyfish's construction: link random pairs of switches that have free ports and no link yet;
    when only switches that are already linked keep free ports, a switch with two free ports
    takes the place of a random link (x, y) it is not next to: (x, y) becomes (s, x) and (s, y)."""
    rng = np.random.default_rng(seed)
    free = [degree] * n_sw
    adj = set()
    while True:
        cand = [i for i in range(n_sw) if free[i] > 0]
        pairs = [(a, b) for ia, a in enumerate(cand) for b in cand[ia + 1:] if (a, b) not in adj]
        if pairs:
            a, b = pairs[int(rng.integers(len(pairs)))]
            adj.add((a, b))
            free[a] -= 1
            free[b] -= 1
            continue
        stuck = [i for i in cand if free[i] >= 2]
        if not stuck:
            break
        s_ = stuck[0]
        near = lambda x: (min(s_, x), max(s_, x)) in adj
        options = sorted((x, y) for x, y in adj if s_ not in (x, y) and not near(x) and not near(y))
        x, y = options[int(rng.integers(len(options)))]
        adj.discard((x, y))
        adj.add((min(s_, x), max(s_, x)))
        adj.add((min(s_, y), max(s_, y)))
        free[s_] -= 2
    links = [(h, -1 - h // hosts_per_sw) for h in range(n_sw * hosts_per_sw)]
    links += [(-1 - a, -1 - b) for a, b in sorted(adj)]
    return Topology(kind=TOPO_GRAPH, n_hosts=n_sw * hosts_per_sw, n_switches=n_sw, links=links)


def dragonfly(groups: int = 9, a: int = 4, h: int = 2, p: int = 4) -> Topology:
    """Dragonfly: `groups` groups of `a` switches, each group a full mesh, every switch with `h`
    global links and `p` hosts; with groups = a*h + 1 every pair of groups has one global link
    (switch j's global links go to groups g + 1 + j*h + i, i < h, in the consecutive arrangement)."""
    if groups != a * h + 1:
        raise ValueError("groups must be a*h + 1")
    n_sw = groups * a
    links = [(x, -1 - x // p) for x in range(n_sw * p)]
    for g in range(groups):
        for i in range(a):
            for j in range(i + 1, a):
                links.append((-1 - (g * a + i), -1 - (g * a + j)))
    seen = set()
    for g in range(groups):
        for j in range(a):
            for i in range(h):
                d = (g + 1 + j * h + i) % groups
                # the switch of group d that holds the link back to g
                off = (g - d - 1) % groups
                k = off // h
                e = (min(g * a + j, d * a + k), max(g * a + j, d * a + k))
                if e not in seen:
                    seen.add(e)
                    links.append((-1 - e[0], -1 - e[1]))
    return Topology(kind=TOPO_GRAPH, n_hosts=n_sw * p, n_switches=n_sw, links=links)


@dataclass
class Request:
    name: str
    arrival_s: float
    topo: Topology
    flows: Flows
    params: TcpParams


def served_stream(seed: int = 1, n: int = 200, rate_per_s: float = 40.0, size_cap: int = 1_000_000) -> list[Request]:
    """Seeded Poisson arrivals of TCP simulation requests: 40% FatTree k=4, 30% k=8, 10% k=16,
    10% Jellyfish (64 switches, degree 8, 4 hosts per switch), 10% Dragonfly (9 groups of 4
    switches, 2 global links and 4 hosts per switch). Each request draws its TCP, ecnK and queue
    from the sweep grid, flows from the web-search-like CDF (capped at `size_cap` bytes) at 30-60%
    load over about 0.5 ms of arrivals. A tenth of the graph requests carry one switch-switch link
    failure between 100 and 500 us, recovered 400 us later."""
    rng = np.random.default_rng(seed)
    jf = jellyfish(seed=seed)
    df = dragonfly()
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate_per_s)
        kind = rng.choice(["k4", "k8", "k16", "jf", "df"], p=[0.4, 0.3, 0.1, 0.1, 0.1])
        topo = {"k4": Topology.fattree(4), "k8": Topology.fattree(8), "k16": Topology.fattree(16), "jf": jf, "df": df}[kind]
        if kind in ("jf", "df") and rng.random() < 0.5:  # (a tenth of all requests: half of the graph ones)
            sw = [(a, b) for a, b in topo.links if a < 0 and b < 0]
            a, b = sw[int(rng.integers(len(sw)))]
            tf = int(rng.integers(100_000, 500_001))
            topo = Topology(kind=topo.kind, n_hosts=topo.n_hosts, n_switches=topo.n_switches, links=topo.links,
                            fails=[(tf, -1 - a, -1 - b, 0), (tf + 400_000, -1 - a, -1 - b, 1)])
        H = topo.hosts
        load = float(rng.uniform(0.3, 0.6))
        n_flows = int(max(8, round(load * H * LINK_BYTES_PER_NS * 500_000 / min(web_mean(), size_cap / 2))))
        n_flows = min(n_flows, 4000)
        flows = leafspine_flows(rng, H, n_flows, load)
        flows.size = np.minimum(flows.size, size_cap)
        params = TcpParams(str(rng.choice(["newreno", "dctcp", "cubic"])), int(rng.choice([10, 20, 40, 80])),
                           int(rng.choice([100, 200, 400])), spray=bool(kind in ("jf", "df")))
        out.append(Request(f"c5_{i:04d}_{kind}", t, topo, flows, params))
    return out


# ------------------------------------------------------------------ RDMA worlds (C3 shape)
# The HPCC fork's parameters as its example configuration sets them (the reference runs its RDMA
# validation with these: validation/hpcc/hpcc.cfg), in its "KEY VALUE" input format.
HPCC_CONFIG = {
    "ENABLE_QCN": "1", "USE_DYNAMIC_PFC_THRESHOLD": "1", "PACKET_PAYLOAD_SIZE": "1000", "SIMULATOR_STOP_TIME": "4.00",
    "CC_MODE": "3", "ALPHA_RESUME_INTERVAL": "1", "RATE_DECREASE_INTERVAL": "4", "CLAMP_TARGET_RATE": "0", "RP_TIMER": "900",
    "EWMA_GAIN": "0.00390625", "FAST_RECOVERY_TIMES": "1", "RATE_AI": "50Mb/s", "RATE_HAI": "100Mb/s", "MIN_RATE": "100Mb/s",
    "DCTCP_RATE_AI": "1000Mb/s", "ERROR_RATE_PER_LINK": "0.0000", "L2_CHUNK_SIZE": "4000", "L2_ACK_INTERVAL": "1",
    "L2_BACK_TO_ZERO": "0", "HAS_WIN": "1", "GLOBAL_T": "1", "VAR_WIN": "1", "FAST_REACT": "1", "U_TARGET": "0.95", "MI_THRESH": "0",
    "INT_MULTI": "1", "MULTI_RATE": "0", "SAMPLE_FEEDBACK": "0", "PINT_LOG_BASE": "1.05", "PINT_PROB": "1.0", "RATE_BOUND": "1",
    "ACK_HIGH_PRIO": "0", "LINK_DOWN": "0 0 0", "ENABLE_TRACE": "0",
    "KMAX_MAP": "3 25000000000 400 50000000000 800 100000000000 1600",
    "KMIN_MAP": "3 25000000000 100 50000000000 200 100000000000 400",
    "PMAX_MAP": "3 25000000000 0.2 50000000000 0.2 100000000000 0.2", "BUFFER_SIZE": "32",
}
RDMA_CC = {"dcqcn": 1, "hpcc": 3, "dctcp": 8}


def rdma_config(cc: str, **over) -> str:
    cfg = {**HPCC_CONFIG, "CC_MODE": str(RDMA_CC[cc]), **{k: str(v) for k, v in over.items()}}
    return "".join(f"{k} {v}\n" for k, v in cfg.items())


def fattree_text(k: int) -> str:
    """A FatTree k in TwiNS's topology format: hosts, then edge, aggregation and core switches."""
    h, e = k ** 3 // 4, k * k // 2
    links = [(f"h{x * (k // 2) + j}", f"s{x}") for x in range(e) for j in range(k // 2)]
    links += [(f"s{pod * (k // 2) + b}", f"s{e + pod * (k // 2) + a}") for pod in range(k) for a in range(k // 2) for b in range(k // 2)]
    links += [(f"s{e + pod * (k // 2) + a}", f"s{2 * e + a * (k // 2) + c}") for pod in range(k) for a in range(k // 2) for c in range(k // 2)]
    return f"hosts {h}\nswitches {e + e + (k // 2) ** 2}\n" + "".join(f"link {a} {b}\n" for a, b in links)


@dataclass
class RdmaWorld:
    name: str
    config: str
    topology: str
    flows: Flows


def c3_flows(seed: int = 1, k: int = 16, n: int = 50_000, load: float = 0.4, incasts: int = 16, fanin: int = 64,
             incast_bytes: int = 262_144) -> Flows:
    """All-to-all flows between seeded uniform distinct host pairs, web-search-like sizes, Poisson
    arrivals at `load` of the hosts' 100 Gb/s; plus `incasts` bursts of `fanin` senders to one
    seeded receiver, incast_bytes each, at seeded times within the arrivals' span."""
    rng = np.random.default_rng(seed)
    H = k ** 3 // 4
    src = rng.integers(0, H, n)
    dst = (src + rng.integers(1, H, n)) % H
    size = web_sizes(rng, n)
    rate = load * H * LINK_BYTES_PER_NS / web_mean()
    start = np.cumsum(rng.exponential(1.0 / rate, n)).astype(np.int64) + 1000
    span = int(start[-1])
    s2, d2, z2, t2 = [src], [dst], [size], [start]
    for _ in range(incasts):
        r = int(rng.integers(H))
        others = np.array([h for h in range(H) if h != r])
        snd = rng.choice(others, fanin, replace=False)
        t = int(rng.integers(1000, span))
        s2.append(snd)
        d2.append(np.full(fanin, r))
        z2.append(np.full(fanin, incast_bytes))
        t2.append(np.full(fanin, t))
    src, dst, size, start = (np.concatenate(x) for x in (s2, d2, z2, t2))
    order = np.argsort(start, kind="stable")
    return Flows.from_arrays(src[order], dst[order], size[order], start[order])


def c3(seed: int = 1, ccs=("dcqcn", "hpcc"), **kw) -> list[RdmaWorld]:
    """C3: FatTree k=16 (1,024 hosts, 320 switches, 100 Gb/s, 1 us), 50,000 flows plus 16 incasts of
    64 senders x 256 KB, once per congestion control."""
    flows = c3_flows(seed, **kw)
    topo = fattree_text(kw.get("k", 16))
    return [RdmaWorld(f"c3_k16_{cc}", rdma_config(cc), topo, flows) for cc in ccs]


def write_rdma(w: RdmaWorld, d) -> tuple:
    """The world's files for the reference's twins-rdma: config, topology, flows."""
    from pathlib import Path
    d = Path(d)
    cfg, topo, fl = d / f"{w.name}.cfg", d / f"{w.name}.topo", d / f"{w.name}.csv"
    cfg.write_text(w.config)
    topo.write_text(w.topology)
    with open(fl, "w") as f:
        f.write("src,dst,flow_size,start_ns\n")
        for i in range(len(w.flows)):
            f.write(f"{w.flows.src[i]},{w.flows.dst[i]},{w.flows.size[i]},{w.flows.start_ns[i]}\n")
    return cfg, topo, fl


def rdma_sweep_k8(golden_dir) -> list[RdmaWorld]:
    """The reference's RDMA k=8 parameter sweep (its validation/hpcc/sweep_k8.txt): FatTree k=8
    (its data/topo/fattree8.txt), flows k8_a2a30 and k8_a2a50s, DCQCN and HPCC, buffers of 2 and
    32 MB, and ECN thresholds Kmin/Kmax of 20/80, 50/200, 100/400 and 400/1600 KB at 100 Gb/s:
    32 worlds."""
    from pathlib import Path
    g = Path(golden_dir)
    topo = (g / "topo" / "fattree8.txt").read_text()
    out = []
    for wl in ("k8_a2a30", "k8_a2a50s"):
        flows = Flows.load(g / "flows" / f"{wl}.csv", 128)
        for cc in ("dcqcn", "hpcc"):
            for buf in (2, 32):
                for kmin in (20, 50, 100, 400):
                    cfg = rdma_config(cc, BUFFER_SIZE=buf, KMIN_MAP=f"1 100000000000 {kmin}", KMAX_MAP=f"1 100000000000 {4 * kmin}")
                    out.append(RdmaWorld(f"sw_{wl}_cc{RDMA_CC[cc]}_b{buf}_k{kmin}", cfg, topo, flows))
    return out
