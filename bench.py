#!/usr/bin/env python3
"""Benchmark: packet-events/s (and worlds/s) of the batched slot kernels on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c1|c4|c5] [--impl ours|reference]

A step simulates every world of the workload to completion (all flows done). The default
workload is C2: FatTree k=8, 10,000 flows (web-search-like sizes, Poisson at 50% load, 25% of
connections carrying 4 messages), FIN and per-packet spraying, run with NewReno, DCTCP and Cubic
as three worlds batched in one persistent launch. Inputs are seeded synthetic data.

ours:       `value`  = packet-events per second of device time (CUDA events on the launching
                       stream), state resident in HBM (restored by a device-to-device copy before
                       each step, outside the timed region; L2 flushed between steps);
            `e2e`    = the same metric through the C ABI from host buffers: world set-up, upload,
                       run and the download of every flow's result inside the timed region;
            `parity` = every flow of the step against the oracle run on the whole workload (and
                       against the reference's own CUDA build's fct.csv);
            `c4`, `c5`, `sweep_k8` (default run, one GPU): the batched sweep of 256 worlds against
                       the plain path, the served stream with p50/p99 latency against the requests
                       run alone, and the reference's k=8 golden sweep (138 worlds) as one batch,
                       each result compared.
reference:  the reference's CPU path for this model, the oracle port (the reference TwiNS has no
            CPU build of its TCP model), on the host cores, one process per world, each step the
            whole workload.
Multi-GPU (torchrun): every rank runs its own copy of the workload (seeded by rank), no
collective on the data path; time is the max over ranks ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import tempfile
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
# algorithmic bytes per packet-event, from the reference's record sizes: a switch event moves a
# 64-byte frame in and out; a host event reads its frame, writes the frames it emits, and reads
# and writes the connection record (368-byte sender record, 160-byte receiver record)
FRAME_B, SND_REC_B, RCV_REC_B = 64, 368, 160
METRIC = "packet-events/s"


def algorithmic_bytes(st: dict) -> int:
    rcv = st["host_events"] - st["host_sender_events"]
    return (2 * FRAME_B * st["switch_events"] + FRAME_B * st["host_events"] + FRAME_B * st["host_frames"]
            + 2 * SND_REC_B * st["host_sender_events"] + 2 * RCV_REC_B * rcv)


def hbm_peak():
    try:
        p = json.loads(PEAKS.read_text())
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            v = [x.strip() for x in line.split(",")]
            if len(v) < 9:
                continue
            try:
                sm.append(float(v[1]))
                mx = float(v[2])
            except ValueError:
                continue
            for n, x in zip(names, v[5:9]):
                if x.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def load_worlds(name: str, rank: int):
    from twins_b200 import workloads
    if name == "c5":  # (the served stream's requests as worlds: the reference arm's sample)
        return [workloads.World(r.name, r.topo, r.flows, r.params) for r in workloads.served_stream(1 + rank, n=200)]
    return workloads.WORKLOADS[name](1 + rank)


def topo_flags(topo):
    from twins_b200 import api
    if topo.kind == api.TOPO_FATTREE:
        return [f"--k={topo.k}"]
    if topo.kind == api.TOPO_LEAFSPINE:
        return ["--topo=leafspine", f"--leaves={topo.leaves}", f"--spines={topo.spines}", f"--hpl={topo.hpl}"]
    # a topology file (hosts / switches / link lines) in the temp directory, and its failures
    name = lambda x: f"h{x}" if x >= 0 else f"s{-1 - x}"
    text = f"hosts {topo.n_hosts}\nswitches {topo.n_switches}\n" + "".join(f"link {name(a)} {name(b)}\n" for a, b in topo.links)
    path = Path(tempfile.gettempdir()) / f"twins_topo_{abs(hash(text)) % 10 ** 12}.txt"
    if not path.exists():
        path.write_text(text)
    flags = ["--topo=graph", f"--topofile={path}"]
    if topo.fails:
        flags.append("--fail=" + ",".join(f"{t}:s{a}:s{b}" + (":up" if up else "") for t, a, b, up in topo.fails))
    return flags


def world_flags(w):
    p = w.params
    return [*topo_flags(w.topo), f"--tcp={p.tcp}", f"--ecnK={p.ecn_k}", f"--queue={p.queue}", f"--fin={int(p.fin)}",
            f"--spray={int(p.spray)}", f"--RngSeed={p.rng_seed}", f"--RngRun={p.rng_run}"]


def oracle_bin() -> Path:
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    return ROOT / "oracle" / "_build" / "twins_oracle"


def run_oracle(binary: Path, w, flows_path: Path, out_dir: Path, max_slots: int):
    cmd = [str(binary), *world_flags(w), f"--flows={flows_path}", f"--out={out_dir / (w.name + '.out.csv')}", f"--max_slots={max_slots}"]
    t0 = time.perf_counter()
    r = subprocess.run(cmd, capture_output=True, text=True, check=True)
    wall = time.perf_counter() - t0
    line = r.stdout.strip().splitlines()[-1]
    f = line.split()
    ev = int(f[f.index("events") + 1])
    sec = float(f[f.index("seconds") + 1])
    return ev, sec, wall


def write_flows(worlds, d: Path):
    paths = []
    for w in worlds:
        p = d / f"{w.name}.csv"
        if not p.exists():
            w.flows.write_csv(p)
        paths.append(p)
    return paths


def cpu_sample(worlds, slots: int, threads: int):
    """The oracle on the first `slots` slots of every world, one world per process."""
    binary = oracle_bin()
    d = Path(tempfile.gettempdir()) / "twins_bench_flows"
    d.mkdir(parents=True, exist_ok=True)
    paths = write_flows(worlds, d)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=max(1, min(threads, len(worlds)))) as ex:
        res = list(ex.map(lambda a: run_oracle(binary, a[0], a[1], d, slots), zip(worlds, paths)))
    wall = time.perf_counter() - t0
    return sum(r[0] for r in res), wall, res


def read_fct(path: Path):
    """Columns 5-6 (established_ns, completed_ns) of an fct.csv as int64 arrays."""
    rows = path.read_text().splitlines()[1:]
    est = np.array([int(r.split(",")[4]) for r in rows], dtype=np.int64)
    done = np.array([int(r.split(",")[5]) for r in rows], dtype=np.int64)
    return est, done


def reference_gpu(worlds, d: Path, ours=None):
    """The reference's own CUDA build (oracle/_ref/twins, built for sm_100a from its sources) on
    the worlds, batched as it batches them: worlds that share a topology and the global flags run
    as one --worlds file (its src/main.cu:267-325), timed by its "Simulation Duration" line. With
    `ours` (name -> (est, done)), every world's fct.csv is compared with this build's results."""
    binary = ROOT / "oracle" / "_ref" / "twins"
    if not binary.exists():
        return None
    paths = write_flows(worlds, d)
    groups = {}
    for w, p in zip(worlds, paths):
        flags = tuple(f for f in world_flags(w) if not f.startswith(("--tcp=", "--ecnK=", "--queue=", "--fin=")))
        groups.setdefault(flags, []).append((w, p))
    total, equal, flows = 0.0, 0, 0
    for flags, members in groups.items():
        wf = d / f"worlds_{abs(hash(flags)) % 10 ** 9}.txt"
        wf.write_text("".join(f"flows={p},tcp={w.params.tcp},ecnK={w.params.ecn_k},queue={w.params.queue},fin={int(w.params.fin)},"
                              f"out={d / (w.name + '.ref.csv')}\n" for w, p in members))
        r = subprocess.run([str(binary), *flags, f"--worlds={wf}"], capture_output=True, text=True, timeout=1200)
        if r.returncode != 0:
            return {"error": r.stderr.strip()[-200:]}
        for line in r.stdout.splitlines():
            if line.startswith("Simulation Duration:"):
                total += float(line.split(":")[1].strip().rstrip("s"))
        if ours is not None:
            for w, _ in members:
                est, done = read_fct(d / (w.name + ".ref.csv"))
                a = ours[w.name]
                equal += int(((est == a[0]) & (done == a[1])).sum())
                flows += len(est)
    out = {"seconds_per_step": total, "batches": len(groups),
           "binary": "oracle/_ref/twins (reference src/main.cu, nvcc sm_100a), same-topology worlds batched with --worlds"}
    if ours is not None:
        out["flows_equal"] = f"{equal}/{flows}"
    return out


class OracleRuns:
    """The oracle (CPU restatement, test infrastructure) on whole worlds, one process per world,
    started in the background: the parity check of every flow and the CPU baseline."""

    def __init__(self, worlds, d: Path):
        binary = oracle_bin()
        self.worlds = worlds
        self.d = d
        paths = write_flows(worlds, d)
        self.t0 = time.perf_counter()
        self.procs = [subprocess.Popen([str(binary), *world_flags(w), f"--flows={p}", f"--out={d / (w.name + '.oracle.csv')}"],
                                       stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for w, p in zip(worlds, paths)]

    def collect(self):
        events, secs, res = 0, [], {}
        for w, p in zip(self.worlds, self.procs):
            out, err = p.communicate()
            if p.returncode != 0:
                raise RuntimeError(f"oracle failed on {w.name}: {err[-200:]}")
            f = out.strip().splitlines()[-1].split()
            events += int(f[f.index("events") + 1])
            secs.append(float(f[f.index("seconds") + 1]))
            res[w.name] = read_fct(self.d / (w.name + ".oracle.csv"))
        return events, secs, res


def compare_all(worlds, ours, want):
    """Flows whose established and completed times are identical, over all worlds."""
    equal = total = 0
    for w in worlds:
        a, b = ours[w.name], want[w.name]
        equal += int(((a[0] == b[0]) & (a[1] == b[1])).sum())
        total += len(a[0])
    return equal, total


def plain_sample(worlds, n, device, batched_wps, batched=None):
    """The plain path: worlds run one at a time on the same GPU (each its own context and run),
    on every (len / n)-th world; worlds/s = sample size / summed device time of the sample. With
    `batched` (world index -> (est, done) from the batch), each sampled world's plain result is
    compared with its batched one."""
    from twins_b200 import api
    step = max(1, len(worlds) // max(1, n))
    idx = list(range(0, len(worlds), step))[:n]
    ms, events, equal = [], 0, 0
    for i in idx:
        w = worlds[i]
        with api.Simulator(device=device) as sim:
            sim.add_world(w.topo, w.flows, w.params)
            sim.run()
            st = sim.stats()
            est, done = sim.results(0)
        if batched is not None:
            equal += int((est == batched[i][0]).all() and (done == batched[i][1]).all())
        ms.append(st["kernel_ms"])
        events += st["packet_events"]
    wps = len(idx) / (sum(ms) / 1000.0)
    out = {"worlds_per_s": wps, "events_per_s": events / (sum(ms) / 1000.0), "sample_worlds": idx,
           "sample": f"{len(idx)} of {len(worlds)} worlds (every {step}th), each alone, device time summed",
           "batched_over_plain_worlds_per_s": batched_wps / wps}
    if batched is not None:
        out["batched_equal_plain"] = f"{equal}/{len(idx)}"
    return out


def c4_leg(device: int, plain_n: int, warmup: int, warmup_slots: int):
    """C4: 256 leaf-spine worlds of uneven size in one batch (one step, device time), against the
    plain path on a sample of the same worlds, each sampled world's results compared."""
    import torch
    from twins_b200 import api, workloads
    worlds = workloads.c4(1)
    sim = api.Simulator(device=device)
    for w in worlds:
        sim.add_world(w.topo, w.flows, w.params)
    sim.prepare()
    for _ in range(warmup):
        sim.run(warmup_slots)
    sim.reset()
    torch.cuda.synchronize()
    sim.run()
    torch.cuda.synchronize()
    st = sim.stats()
    res = {i: sim.results(i) for i in range(len(worlds))}
    unfinished = int(sum((res[i][1] < 0).sum() for i in res))
    sim.close()
    wps = len(worlds) / (st["kernel_ms"] / 1000.0)
    plain = plain_sample(worlds, plain_n, device, wps, batched=res)
    return {"config": "256 leaf-spine worlds (4-32 leaves, spines = leaves / 2, 16 hosts per leaf), tcp x ecnK {10,20,40,80} x "
                      "queue {100,200,400}, 1k-20k web-search-like flows at 30-70% load, one batch",
            "worlds_per_s": wps, "seconds_per_step": st["kernel_ms"] / 1000.0, "packet_events_per_s": st["packet_events"] / (st["kernel_ms"] / 1000.0),
            "packet_events": st["packet_events"], "flows": int(sum(len(w.flows) for w in worlds)), "unfinished_flows": unfinished,
            "steps": 1, "warmup": f"{warmup} runs of {warmup_slots} slots", "plain": plain,
            "batched_over_plain": plain["batched_over_plain_worlds_per_s"]}


def sweep_leg(device: int, ref_gpu: bool = True):
    """The reference's k=8 parameter sweep (138 ecnK x queue x TCP configurations of FatTree k=8,
    its data/ns3/sweep_k8 golden set, fixtures under tests/golden/sweep) as one batch of worlds, as
    its bench/sweep.py runs it (worlds with undecided ties again on the 25-run chain build, time
    included); worlds/s over device time, and every configuration compared with ns-3."""
    import torch
    from twins_b200 import api
    g = ROOT / "tests" / "golden"
    index = json.loads((g / "sweep" / "index.json").read_text())["k8"]
    z = np.load(g / "sweep" / "k8.npz")
    topo = api.Topology.fattree(8)
    flows = {c["flows"]: api.Flows.load(g / c["flows"], topo.hosts) for c in index}

    def batch(cfgs, runs):
        with api.Simulator(device=device, chain_runs=runs) as sim:
            for c in cfgs:
                sim.add_world(topo, flows[c["flows"]], api.TcpParams(c["tcp"], c["ecn_k"], c["queue"]))
            sim.run()
            torch.cuda.synchronize()
            return [sim.results(i) for i in range(len(cfgs))], [sim.counters(i)["undecided_ties"] for i in range(len(cfgs))], sim.stats()

    batch(index[:4], 9)  # (warm-up: loads the module, small)
    res, ties, st = batch(index, 9)
    ms = st["kernel_ms"]
    redo = [i for i, t in enumerate(ties) if t]
    if redo:
        r2, _, st2 = batch([index[i] for i in redo], 25)
        ms += st2["kernel_ms"]
        for j, i in enumerate(redo):
            res[i] = r2[j]
    equal, at = 0, 0
    for c, (est, done) in zip(index, res):
        n = c["rows"]
        equal += int((est == z["est"][at:at + n]).all() and (done == z["done"][at:at + n]).all())
        at += n
    ref = None
    if ref_gpu:
        try:
            ref = sweep_reference_gpu(index, z, g)
        except Exception as e:
            ref = {"error": str(e)[:200]}
    return {"config": "FatTree k=8 sweep: 138 configurations (k8_a2a30, k8_a2a50w flows) in one batch",
            "worlds_per_s": len(index) / (ms / 1000.0), "seconds": ms / 1000.0, "rerun_25_runs": len(redo),
            "identical_to_ns3": f"{equal}/{len(index)}", "reference_gpu": ref,
            "published": {"rtx5090_1x138_worlds_per_s": 52.3, "rx9060xt_2x69_worlds_per_s": 22.3,
                          "source": "reference docs/nvidia.md:126, README.md:257"}}


def sweep_reference_gpu(index, z, g: Path):
    """The reference's CUDA build on the same 138 configurations as one --worlds batch, as its
    bench/sweep.py runs a batch (worlds with undecided ties again on its twins128 build, time
    included), timed by its "Simulation Duration" lines; every configuration compared with ns-3."""
    binary, long_binary = ROOT / "oracle" / "_ref" / "twins", ROOT / "oracle" / "_ref" / "twins128"
    if not binary.exists():
        return None
    d = Path(tempfile.mkdtemp(prefix="sweep_ref_"))
    lines = [f"flows={g / c['flows']},tcp={c['tcp']},queue={c['queue']},ecnK={c['ecn_k']},out={d / (c['name'] + '.csv')}" for c in index]

    def run(b, ls, name):
        wf = d / name
        wf.write_text("\n".join(ls) + "\n")
        r = subprocess.run([str(b), "--k=8", f"--worlds={wf}"], capture_output=True, text=True, timeout=1800)
        if r.returncode != 0:
            raise RuntimeError(r.stderr.strip()[-200:])
        secs = sum(float(l.split(":")[1].strip().rstrip("s")) for l in r.stdout.splitlines() if l.startswith("Simulation Duration:"))
        return r, secs

    r, secs = run(binary, lines, "worlds.txt")
    reruns = 0
    if "undecided" in r.stderr and long_binary.exists():
        m = re.search(r"undecided-ties by world:([ 0-9]*)", r.stdout)
        redo = [lines[int(w)] for w in m.group(1).split()] if m else lines
        reruns = len(redo)
        _, s2 = run(long_binary, redo, "worlds_long.txt")
        secs += s2
    equal, at = 0, 0
    for c in index:
        n = c["rows"]
        est, done = read_fct(d / (c["name"] + ".csv"))
        equal += int((est == z["est"][at:at + n]).all() and (done == z["done"][at:at + n]).all())
        at += n
    shutil.rmtree(d, ignore_errors=True)
    return {"seconds": secs, "worlds_per_s": len(index) / secs, "rerun_twins128": reruns, "identical_to_ns3": f"{equal}/{len(index)}",
            "binary": "oracle/_ref/twins --k=8 --worlds (reference src/main.cu, nvcc sm_100a), one batch of 138"}


def serve_leg(device: int, requests: int, rate: float, serve_worlds: int):
    """C5: a seeded Poisson stream of simulation requests served by continuous batching (requests
    join the running batch between launches), against the same requests run one at a time, each
    served result compared with its run alone. Latency = completion - submission on the server's
    clock; worlds/s = requests / (last completion - first submission)."""
    from twins_b200 import api, workloads
    reqs = workloads.served_stream(seed=1, n=requests + 3, rate_per_s=rate)
    warm, reqs = reqs[:3], reqs[3:]
    # capacities for about `serve_worlds` requests of the mix at once (500 hosts, 170 switches,
    # 1,700 ports and 2,500 connections per request on average, with room), within 160 GB
    n = serve_worlds
    caps = dict(worlds=n, hosts=500 * n, switches=170 * n, ports=1700 * n, connections=2500 * n, messages=2500 * n,
                sent_list_entries=min(1 << 30, 2_800_000 * n), ooo_blocks=min(1 << 28, 700_000 * n), slots_per_launch=128,
                hbm_budget_bytes=160 * 10 ** 9)
    with api.Server(device=device, **caps) as srv:
        srv.start()
        for r in warm:  # warm-up requests (untimed)
            srv.wait(srv.submit(r.topo, r.flows, r.params), timeout_s=600)
        st0 = srv.stats()
        ids = []
        with Clocks(device) as clocks:
            t0 = time.perf_counter()
            for r in reqs:
                delay = r.arrival_s - reqs[0].arrival_s - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                ids.append(srv.submit(r.topo, r.flows, r.params))
            for i in ids:
                srv.wait(i, timeout_s=900)
        infos = [srv.info(i) for i in ids]
        served = [srv.results(i)[:2] for i in ids]
        st = srv.stats()
    lat = np.array([x["t_done"] - x["t_submit"] for x in infos])
    span = max(x["t_done"] for x in infos) - min(x["t_submit"] for x in infos)
    served_wps = len(ids) / span
    events = st["packet_events"] - st0["packet_events"]
    # the plain path: every request alone, one after the other (device time)
    plain_ms, plain_events, equal = 0.0, 0, 0
    for r, (est_s, done_s) in zip(reqs, served):
        with api.Simulator(device=device) as sim:
            sim.add_world(r.topo, r.flows, r.params)
            sim.run()
            x = sim.stats()
            est, done = sim.results(0)
        equal += int((est == est_s).all() and (done == done_s).all())
        plain_ms += x["kernel_ms"]
        plain_events += x["packet_events"]
    plain_wps = len(reqs) / (plain_ms / 1000.0)
    mix = {}
    for r in reqs:
        k = r.name.split("_")[2]
        mix[k] = mix.get(k, 0) + 1
    return {"config": "served stream (C5 shape, TCP requests): Poisson arrivals, 40% FatTree k=4, 30% k=8, 10% k=16, "
                      "10% Jellyfish 64x8 (4 hosts/switch), 10% Dragonfly 9x4; a tenth with a link failure",
            "requests": len(reqs), "rate_per_s": rate, "mix": mix, "flows": int(sum(len(r.flows) for r in reqs)),
            "worlds_per_s": served_wps, "span_s": span, "warmup_requests": len(warm),
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "packet_events_per_s": events / span,
            "device_busy_frac": (st["kernel_ms"] - st0["kernel_ms"]) / 1000.0 / span,
            "plain": {"worlds_per_s": plain_wps, "events_per_s": plain_events / (plain_ms / 1000.0),
                      "sample": "every request alone, one after the other, device time summed"},
            "served_over_plain": served_wps / plain_wps,
            "served_equal_alone": f"{equal}/{len(reqs)}",
            "server": {k: st[k] for k in ("launches", "slots_run", "admitted", "retired", "hbm_bytes", "host_lanes", "stage_frames", "grid")},
            "capacities": caps, "clocks": clocks.summary()}


# algorithmic bytes per RDMA packet-event, from the reference's record sizes: a switch event moves a
# 176-byte LFrame in and out; a NIC event reads its frame, writes the frames it emits, and reads and
# writes the queue pair (208-byte SndQP for an ACK or NACK, 16-byte RcvQP for data)
LFRAME_B, SNDQP_B, RCVQP_B = 176, 208, 16


def rdma_algorithmic_bytes(st: dict) -> int:
    return (2 * LFRAME_B * st["switch_events"] + LFRAME_B * st["host_events"] + LFRAME_B * st["host_frames"]
            + 2 * SNDQP_B * st["host_sender_events"] + 2 * RCVQP_B * (st["host_events"] - st["host_sender_events"]))


def c3_leg(device: int, warmup: int = 3, ref: bool = True, q3cap: int = 1 << 16):
    """C3: the RDMA model on FatTree k=16 (1,024 hosts, 320 switches), 50,000 all-to-all flows at 40%
    load plus 16 incasts of 64 x 256 KB, once with DCQCN and once with HPCC-INT. Device time of the
    slot kernel (state resident), end to end through the C ABI, the roofline of the algorithmic bytes,
    and the reference's own twins-rdma (built for sm_100a) on the same files: its time and every FCT
    compared."""
    import torch
    from twins_b200 import api, workloads
    peak, _ = hbm_peak()
    d = Path(tempfile.mkdtemp(prefix="twins_c3_"))
    out = {"config": "FatTree k=16 (1,024 hosts, 320 switches, 100 Gb/s, 1 us), 50,000 web-search-like all-to-all flows at 40% load "
                     "+ 16 incasts of 64 x 256 KB; HPCC example configuration (32 MB buffers, PFC, ECN); port queues of "
                     f"{q3cap} frames (both builds)"}
    for w in workloads.c3():
        cc = w.name.split("_")[-1]
        with api.Simulator(device=device) as sim:
            sim.set_rdma_queue_cap(q3cap)
            i = sim.add_rdma_world(w.config, w.topology, w.flows)
            sim.prepare()
            for _ in range(warmup):
                sim.run(300)
            torch.cuda.synchronize()
            status = sim.run()
            st = sim.stats()
            _, fct = sim.rdma_results(i)
            ev = sim.rdma_counters(i)
        t0 = time.perf_counter()
        with api.Simulator(device=device) as s2:
            s2.set_rdma_queue_cap(q3cap)
            j = s2.add_rdma_world(w.config, w.topology, w.flows)
            s2.run()
            s2.rdma_results(j)
            st2 = s2.stats()
        e2e_s = time.perf_counter() - t0
        sec = st["kernel_ms"] / 1000.0
        alg = rdma_algorithmic_bytes(st)
        leg = {"packet_events_per_s": st["packet_events"] / sec, "seconds": sec, "packet_events": st["packet_events"],
               "slots": st["slots"], "slots_run": st["slots_run"], "launches": st["launches"], "grid": st["grid"],
               "flows": len(w.flows), "flows_done": int((fct >= 0).sum()), "status": status, "counters": api.rdma_counters_line(ev),
               "e2e": {"packet_events_per_s": st["packet_events"] / e2e_s, "seconds": e2e_s, "h2d_bytes": st2["bytes_h2d"],
                       "d2h_bytes": st2["bytes_d2h"]},
               "roofline": {"bound": "hbm", "achieved": alg / sec / 1e9, "peak": peak, "unit": "GB/s", "frac": alg / sec / 1e9 / peak,
                            "algorithmic_bytes": alg}}
        exe = ROOT / "oracle" / "_ref" / "twins-rdma"
        if ref and exe.exists():
            cfg, topo, fl = workloads.write_rdma(w, d)
            r = subprocess.run([str(exe), cfg.name, f"--topo={topo.name}", f"--flows={fl.name}", f"--out={w.name}.ref.fct",
                                f"--q3cap={q3cap}"], cwd=d,
                               capture_output=True, text=True, timeout=1200)
            line = next((x for x in r.stdout.splitlines() if x.startswith("flows done")), "")
            ref_wall = float(line.split(" in ")[1].split(" s wall")[0]) if line else None
            want = np.full(len(w.flows), -1, dtype=np.int64)
            for x in (d / f"{w.name}.ref.fct").read_text().splitlines() if (d / f"{w.name}.ref.fct").exists() else []:
                a, _, f = (int(v) for v in x.split())
                want[a] = f
            leg["reference_gpu"] = {"rc": r.returncode, "seconds": ref_wall,
                                    "packet_events_per_s": st["packet_events"] / ref_wall if ref_wall else None,
                                    "counters": next((x for x in r.stdout.splitlines() if x.startswith("drops ")), ""),
                                    "flows_equal": f"{int((want == fct).sum())}/{len(fct)}",
                                    "binary": "oracle/_ref/twins-rdma (reference src/rdma/rmain.cu, nvcc sm_100a)"}
        out[cc] = leg
    return out


def rdma_sweep_leg(device: int, ref: bool = True):
    """The reference's RDMA k=8 sweep (validation/hpcc/sweep_k8.txt: 32 worlds of FatTree k=8, two
    workloads x DCQCN/HPCC x two buffer sizes x four ECN thresholds) as one batch: worlds/s over
    device time, against the reference's own twins-rdma running the same job file as its --batch,
    every FCT compared. Published: 19.8 worlds/s on an RTX 5090 (its docs/nvidia.md:147)."""
    import torch
    from twins_b200 import api, workloads
    worlds = workloads.rdma_sweep_k8(ROOT / "tests" / "golden")
    with api.Simulator(device=device) as sim:
        ids = [sim.add_rdma_world(w.config, w.topology, w.flows) for w in worlds]
        sim.prepare()
        sim.run(300)  # (warm-up: a short run)
        torch.cuda.synchronize()
        status = sim.run()
        st = sim.stats()
        res = [sim.rdma_results(i)[1] for i in ids]
    sec = st["kernel_ms"] / 1000.0
    out = {"config": "32 worlds of the reference's k=8 RDMA sweep (FatTree k=8, k8_a2a30 / k8_a2a50s flows, DCQCN / HPCC, 2 / 32 MB "
                     "buffers, Kmin 20 / 50 / 100 / 400 KB) in one batch",
           "worlds_per_s": len(worlds) / sec, "seconds": sec, "packet_events": st["packet_events"], "status": status,
           "flows_done": int(sum((r >= 0).sum() for r in res)), "flows": int(sum(len(r) for r in res)),
           "published": {"rtx5090_worlds_per_s": 19.8, "rx9060xt_worlds_per_s": 10.0, "source": "reference docs/nvidia.md:147, README.md:286-289"}}
    exe = ROOT / "oracle" / "_ref" / "twins-rdma"
    if ref and exe.exists():
        d = Path(tempfile.mkdtemp(prefix="twins_rsweep_"))
        jobs = []
        for w in worlds:
            cfg, topo, fl = workloads.write_rdma(w, d)
            jobs.append(f"{w.name} {topo.name} {fl.name}")
        (d / "jobs.txt").write_text("\n".join(jobs) + "\n")
        (d / "out").mkdir()
        base = d / f"{worlds[0].name}.cfg"
        # (each world's own config: the job lines carry its keys as overrides of the first one's)
        lines = []
        for w in worlds:
            kv = dict(line.split(" ", 1) for line in w.config.strip().splitlines())
            over = " ".join(f"{k}={v.replace(' ', ',')}" for k, v in kv.items() if k in ("CC_MODE", "BUFFER_SIZE", "KMIN_MAP", "KMAX_MAP"))
            lines.append(f"{w.name} {w.name}.topo {w.name}.csv {over}")
        (d / "jobs.txt").write_text("\n".join(lines) + "\n")
        r = subprocess.run([str(exe), base.name, "--batch=jobs.txt", "--outdir=out"], cwd=d, capture_output=True, text=True, timeout=1200)
        line = next((x for x in r.stdout.splitlines() if x.startswith("flows done")), "")
        ref_wall = float(line.split(" in ")[1].split(" s wall")[0]) if line else None
        equal = 0
        for w, fct in zip(worlds, res):
            want = np.full(len(fct), -1, dtype=np.int64)
            f = d / "out" / f"{w.name}.fct"
            for x in f.read_text().splitlines() if f.exists() else []:
                a, _, v = (int(y) for y in x.split())
                want[a] = v
            equal += int((want == fct).all())
        out["reference_gpu"] = {"rc": r.returncode, "seconds": ref_wall, "worlds_per_s": len(worlds) / ref_wall if ref_wall else None,
                                "worlds_equal": f"{equal}/{len(worlds)}",
                                "binary": "oracle/_ref/twins-rdma --batch (reference src/rdma/rmain.cu, nvcc sm_100a)"}
    return out


def reference_arm(args, worlds, config):
    """The reference arm: the reference's CPU path for this model on the host cores, which is the
    oracle port (the reference has no CPU build of its TCP model): every world of the workload
    whole, one process per world, all worlds at once; warm-up steps run a short prefix."""
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(worlds, 300, threads)
    evs, walls = [], []
    slots = args.ref_slots if args.ref_slots > 0 else 10 ** 12
    for _ in range(args.steps):
        ev, wall, _ = cpu_sample(worlds, slots, threads)
        evs.append(ev)
        walls.append(wall)
    value = sum(evs) / sum(walls)
    what = "whole" if args.ref_slots <= 0 else f"the first {args.ref_slots} slots of each of"
    sample = f"{what} {len(worlds)} worlds per step ({sum(evs) // len(evs)} packet-events), one process (core) per world, all at once"
    cores = min(threads, len(worlds))
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.mean(walls),
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                      "data": "synthetic", "config": config,
                      "cpu_baseline": {"value": value, "unit": "events/s", "cores": cores, "nproc": threads, "kind": "port",
                                       "sample": sample},
                      "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c2s", "c3", "c4", "c4s", "c5"])
    ap.add_argument("--requests", type=int, default=200, help="C5: requests in the served stream")
    ap.add_argument("--rate", type=float, default=100.0, help="C5: request arrivals per second (Poisson)")
    ap.add_argument("--serve-worlds", type=int, default=256, help="C5: requests the server holds at once")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-slots", type=int, default=0, help="reference arm: slots of each world per step (0: whole worlds)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--host-lanes", type=int, default=None, help="fixed hosts per warp (default: autotuned launch shapes)")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="C2 alone: no C4, C5 or sweep legs")
    ap.add_argument("--no-parity", action="store_true", help="no oracle comparison of every flow")
    ap.add_argument("--warmup-slots", type=int, default=None,
                    help="slots of each warm-up run (default: C2 3000, C4 400; 0: whole runs)")
    ap.add_argument("--plain-sample", type=int, default=16,
                    help="C4: worlds of the plain path (one world at a time) timed, every (256 / n)-th world")
    args = ap.parse_args()
    if args.warmup_slots is None:
        args.warmup_slots = 400 if args.workload == "c4" else 3000
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    world_size = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.workload == "c3" and args.impl == "ours":
        if rank == 0:
            import torch
            torch.cuda.set_device(local_rank)
            print(json.dumps({"workload": "c3", **c3_leg(local_rank), "rdma_sweep_k8": rdma_sweep_leg(local_rank)}))
        return
    if args.workload == "c5" and args.impl == "ours":
        if rank == 0:  # (one server on one GPU; other ranks have nothing to add)
            import torch
            torch.cuda.set_device(local_rank)
            out = serve_leg(local_rank, args.requests, args.rate, args.serve_worlds)
            print(json.dumps({"metric": "worlds/s (served)", "value": out["worlds_per_s"], "unit": "worlds/s", "n_gpus": 1, "steps": 1,
                              "warmup": out["warmup_requests"], "ms_per_step": 1000 * out["span_s"], "higher_is_better": True,
                              "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
                              "config": {"workload": out["config"]}, **{k: v for k, v in out.items() if k != "config"}}))
        return
    worlds = load_worlds(args.workload, rank)
    config = {"workload": {"c1": "FatTree k=4, 240 flows, DCTCP (C1)",
                           "c2": "FatTree k=8, 10,000 flows x {NewReno, DCTCP, Cubic}, FIN, spraying (C2)",
                           "c2s": "FatTree k=8, 1,500 flows x {NewReno, DCTCP, Cubic}, FIN, spraying (C2 shape, small)",
                           "c4": "256 leaf-spine worlds, 1k-20k flows each (C4)",
                           "c4s": "32 leaf-spine worlds, 500-3,000 flows each (C4 shape, small)",
                           "c5": "200 served-stream requests (C5 shape, TCP) as worlds"}[args.workload],
              "worlds": len(worlds), "flows_per_step": int(sum(len(w.flows) for w in worlds)),
              "l2": "flushed between steps (256 MiB write); state restored device-to-device before each step",
              "seed": 1}

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, worlds, config)
        return

    import torch
    from twins_b200 import api
    torch.cuda.set_device(local_rank)
    dist = None
    if world_size > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    scratch = Path(tempfile.mkdtemp(prefix="twins_bench_"))
    sim = api.Simulator(device=local_rank, host_lanes=args.host_lanes)
    for w in worlds:
        sim.add_world(w.topo, w.flows, w.params)
    sim.prepare()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
    for _ in range(args.warmup):
        sim.reset()
        sim.run(args.warmup_slots)
    kernel_ms, launches, stats = [], 0, None
    with Clocks(local_rank) as clocks:
        for _ in range(args.steps):
            flush.fill_(1)
            sim.reset()
            torch.cuda.synchronize()
            barrier()
            sim.run()
            torch.cuda.synchronize()
            stats = sim.stats()
            kernel_ms.append(stats["kernel_ms"])
            launches += stats["launches"]
    events = stats["packet_events"]
    ours = {w.name: sim.results(i) for i, w in enumerate(worlds)}
    unfinished = int(sum((d < 0).sum() for _, d in ours.values()))
    ms = statistics.mean(kernel_ms)
    from twins_b200 import shard
    ms_max, events_all = shard.aggregate(ms, float(events), dist, device=f"cuda:{local_rank}")
    value = events_all / (ms_max / 1000.0)
    # every flow against the oracle: whole worlds on the host cores, one process per world, in the
    # background while the other legs run (rank 0)
    oracle = OracleRuns(worlds, scratch) if rank == 0 and not args.no_parity else None

    # end to end through the C ABI from host buffers
    e2e_ms, h2d, d2h = [], 0, 0
    for _ in range(args.e2e_steps):
        barrier()
        t0 = time.perf_counter()
        with api.Simulator(device=local_rank, host_lanes=args.host_lanes) as s2:
            for w in worlds:
                s2.add_world(w.topo, w.flows, w.params)
            s2.run()
            for i in range(len(worlds)):
                s2.results(i)
            st2 = s2.stats()
        e2e_ms.append(1000 * (time.perf_counter() - t0))
        h2d, d2h = st2["bytes_h2d"], st2["bytes_d2h"]
    e2e_step = statistics.mean(e2e_ms) if e2e_ms else float("nan")
    if dist is not None:
        t = torch.tensor([e2e_step], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_step = float(t[0])
    e2e_value = events_all / (e2e_step / 1000.0)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peak, peak_kind = hbm_peak()
    alg = algorithmic_bytes(stats)
    achieved = alg / (ms / 1000.0) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "free_kernel_traffic.json"
    if tfile.exists():
        try:
            tj = json.loads(tfile.read_text())
            # DRAM bytes per packet-event from the capture, scaled to this step's events
            traffic = tj["dram_bytes_per_event"] * events / max(1, stats["launches"])
        except Exception:
            traffic = None
    ref_gpu = None
    if not args.no_ref_gpu:
        try:
            ref_gpu = reference_gpu(worlds, scratch, ours)
            if ref_gpu and "seconds_per_step" in ref_gpu:
                ref_gpu["value"] = events / ref_gpu["seconds_per_step"]
                ref_gpu["unit"] = "events/s"
        except Exception as e:
            ref_gpu = {"error": str(e)[:200]}
    extras = {}
    if args.workload == "c2" and not args.no_extras and world_size == 1:
        extras["c4"] = c4_leg(local_rank, args.plain_sample, 3, 200)
        extras["c5"] = serve_leg(local_rank, args.requests, args.rate, args.serve_worlds)
        extras["sweep_k8"] = sweep_leg(local_rank, not args.no_ref_gpu)
        extras["c3"] = c3_leg(local_rank)
        extras["rdma_sweep_k8"] = rdma_sweep_leg(local_rank)
    elif args.workload == "c4":
        extras["plain"] = plain_sample(worlds, args.plain_sample, local_rank, len(worlds) / (ms_max / 1000.0),
                                       batched=dict(enumerate(ours[w.name] for w in worlds)))
    parity, cpu = {}, None
    if oracle is not None:
        ev_cpu, secs, want = oracle.collect()
        eq, n = compare_all(worlds, ours, want)
        parity = {"flows_equal_oracle": f"{eq}/{n}", "oracle_events": ev_cpu, "events_equal_oracle": ev_cpu == events}
        cpu = {"value": ev_cpu / max(secs), "unit": "events/s", "cores": len(worlds), "nproc": os.cpu_count(), "kind": "port",
               "sample": f"the oracle on the whole workload ({len(worlds)} worlds, one process per world at once, "
                         f"event loop {', '.join(f'{s:.1f}' for s in secs)} s)"}
    if ref_gpu and "flows_equal" in ref_gpu:
        parity["flows_equal_reference_gpu_build"] = ref_gpu["flows_equal"]
    out = {
        "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic", "config": config,
        "worlds_per_s": len(worlds) * world_size / (ms_max / 1000.0),
        "packet_events_per_step": events, "unfinished_flows": unfinished,
        "slots_per_step": stats["slots"], "slots_run_per_step": stats["slots_run"],
        "e2e": {"value": e2e_value, "unit": "events/s", "ms_per_step": e2e_step, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "algorithmic_bytes_per_step": alg},
        "cpu_baseline": cpu,
        "parity": parity,
        "clocks": clocks.summary(),
        "gpu_launches": launches,
        "graph_launches": stats["graph_launches"],
        "launch": {"grid": stats["grid"], "host_lanes": stats["host_lanes"], "warps_per_block": stats["warps_per_block"],
                   "stage_frames": stats["stage_frames"], "autotuned": bool(stats["autotuned"])},
    }
    if ref_gpu is not None:
        out["reference_gpu"] = ref_gpu
    out.update(extras)
    print(json.dumps(out))
    sim.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
