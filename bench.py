#!/usr/bin/env python3
"""Benchmark: packet-events/s (and worlds/s) of the batched slot kernels on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c1|c4] [--impl ours|reference]

A step simulates every world of the workload to completion (all flows done). The default
workload is C2: FatTree k=8, 10,000 flows (web-search-like sizes, Poisson at 50% load, 25% of
connections carrying 4 messages), FIN and per-packet spraying, run with NewReno, DCTCP and Cubic
as three worlds batched in one persistent launch. Inputs are seeded synthetic data.

ours:       `value`  = packet-events per second of device time (CUDA events on the launching
                       stream), state resident in HBM (restored by a device-to-device copy before
                       each step, outside the timed region; L2 flushed between steps);
            `e2e`    = the same metric through the C ABI from host buffers: world set-up, upload,
                       run and the download of every flow's result inside the timed region.
reference:  the reference's CPU path for this model, the oracle port (the reference TwiNS has no
            CPU build of its TCP model), on the host cores, one world per process, each step a
            bounded sample of the workload (the first --ref-slots slots of every world).
Multi-GPU (torchrun): every rank runs its own copy of the workload (seeded by rank), no
collective on the data path; time is the max over ranks ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
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


def reference_gpu(worlds, d: Path):
    """The reference's own CUDA build (oracle/_ref/twins, built for sm_100a from its sources) on
    each world, one at a time as it runs them: its event-loop time ("Simulation Duration")."""
    binary = ROOT / "oracle" / "_ref" / "twins"
    if not binary.exists():
        return None
    paths = write_flows(worlds, d)
    total = 0.0
    for w, p in zip(worlds, paths):
        r = subprocess.run([str(binary), *world_flags(w), f"--flows={p}", f"--out={d / (w.name + '.ref.csv')}"], capture_output=True,
                           text=True, timeout=600)
        if r.returncode != 0:
            return {"error": r.stderr.strip()[-200:]}
        for line in r.stdout.splitlines():
            if line.startswith("Simulation Duration:"):
                total += float(line.split(":")[1].strip().rstrip("s"))
    return {"seconds_per_step": total, "binary": "oracle/_ref/twins (reference src/main.cu, nvcc sm_100a)"}


def plain_sample(worlds, n, device, batched_wps):
    """The plain path: worlds run one at a time on the same GPU (each its own context and run),
    on every (len / n)-th world; worlds/s = sample size / summed device time of the sample."""
    from twins_b200 import api
    step = max(1, len(worlds) // max(1, n))
    idx = list(range(0, len(worlds), step))[:n]
    ms, events = [], 0
    for i in idx:
        w = worlds[i]
        with api.Simulator(device=device) as sim:
            sim.add_world(w.topo, w.flows, w.params)
            sim.run()
            st = sim.stats()
        ms.append(st["kernel_ms"])
        events += st["packet_events"]
    wps = len(idx) / (sum(ms) / 1000.0)
    return {"worlds_per_s": wps, "events_per_s": events / (sum(ms) / 1000.0), "sample_worlds": idx,
            "sample": f"{len(idx)} of {len(worlds)} worlds (every {step}th), each alone, device time summed",
            "batched_over_plain_worlds_per_s": batched_wps / wps}


def serve_bench(args):
    """C5: a seeded Poisson stream of simulation requests served by continuous batching (requests
    join the running batch between launches), against the same requests run one at a time.
    Latency = completion - submission on the server's clock; worlds/s = requests / (last
    completion - first submission). One GPU (each rank would serve its own stream)."""
    import torch
    from twins_b200 import api, workloads
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local_rank)
    reqs = workloads.served_stream(seed=1, n=args.requests + 3, rate_per_s=args.rate)
    warm, reqs = reqs[:3], reqs[3:]
    # capacities for about `--serve-worlds` requests of the mix at once (500 hosts, 170 switches,
    # 1,700 ports and 2,500 connections per request on average, with room), within 160 GB
    n = args.serve_worlds
    caps = dict(worlds=n, hosts=500 * n, switches=170 * n, ports=1700 * n, connections=2500 * n, messages=2500 * n,
                sent_list_entries=min(1 << 30, 2_800_000 * n), ooo_blocks=min(1 << 28, 700_000 * n), slots_per_launch=128,
                hbm_budget_bytes=160 * 10 ** 9)
    with api.Server(device=local_rank, **caps) as srv:
        srv.start()
        for r in warm:  # warm-up requests (untimed)
            srv.wait(srv.submit(r.topo, r.flows, r.params), timeout_s=600)
        st0 = srv.stats()
        ids = []
        with Clocks(local_rank) as clocks:
            t0 = time.perf_counter()
            for r in reqs:
                delay = r.arrival_s - reqs[0].arrival_s - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                ids.append(srv.submit(r.topo, r.flows, r.params))
            for i in ids:
                srv.wait(i, timeout_s=900)
        infos = [srv.info(i) for i in ids]
        st = srv.stats()
    lat = np.array([x["t_done"] - x["t_submit"] for x in infos])
    span = max(x["t_done"] for x in infos) - min(x["t_submit"] for x in infos)
    served_wps = len(ids) / span
    events = st["packet_events"] - st0["packet_events"]
    # the plain path: every request alone, one after the other (device time)
    plain_ms, plain_events = 0.0, 0
    for r in reqs:
        with api.Simulator(device=local_rank) as sim:
            sim.add_world(r.topo, r.flows, r.params)
            sim.run()
            x = sim.stats()
        plain_ms += x["kernel_ms"]
        plain_events += x["packet_events"]
    plain_wps = len(reqs) / (plain_ms / 1000.0)
    mix = {}
    for r in reqs:
        k = r.name.split("_")[2]
        mix[k] = mix.get(k, 0) + 1
    print(json.dumps({
        "metric": "worlds/s (served)", "value": served_wps, "unit": "worlds/s", "n_gpus": 1, "steps": 1, "warmup": len(warm),
        "ms_per_step": 1000 * span, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic",
        "config": {"workload": "served stream (C5 shape, TCP requests): Poisson arrivals, 40% FatTree k=4, 30% k=8, 10% k=16, "
                               "10% Jellyfish 64x8 (4 hosts/switch), 10% Dragonfly 9x4; a tenth with a link failure",
                   "requests": len(reqs), "rate_per_s": args.rate, "mix": mix, "flows": int(sum(len(r.flows) for r in reqs)),
                   "capacities": caps},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
        "packet_events_per_s": events / span,
        "device_busy_frac": (st["kernel_ms"] - st0["kernel_ms"]) / 1000.0 / span,
        "plain": {"worlds_per_s": plain_wps, "events_per_s": plain_events / (plain_ms / 1000.0),
                  "sample": "every request alone, one after the other, device time summed"},
        "served_over_plain_worlds_per_s": served_wps / plain_wps,
        "server": {k: st[k] for k in ("launches", "slots_run", "admitted", "retired", "hbm_bytes", "host_lanes", "stage_frames", "grid")},
        "clocks": clocks.summary(),
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c2s", "c4", "c5"])
    ap.add_argument("--requests", type=int, default=200, help="C5: requests in the served stream")
    ap.add_argument("--rate", type=float, default=100.0, help="C5: request arrivals per second (Poisson)")
    ap.add_argument("--serve-worlds", type=int, default=256, help="C5: requests the server holds at once")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-slots", type=int, default=2500, help="reference arm: slots of each world per step")
    ap.add_argument("--cpu-slots", type=int, default=6000, help="cpu_baseline: slots of the sample world")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--host-lanes", type=int, default=None, help="fixed hosts per warp (default: autotuned launch shapes)")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--warmup-slots", type=int, default=None,
                    help="slots of each warm-up run (default: whole runs; C4: 400)")
    ap.add_argument("--plain-sample", type=int, default=16,
                    help="C4: worlds of the plain path (one world at a time) timed, every (256 / n)-th world")
    args = ap.parse_args()
    if args.warmup_slots is None:
        args.warmup_slots = 400 if args.workload == "c4" else 0
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    if args.workload == "c5" and args.impl == "ours":
        if rank == 0:  # (one server on one GPU; other ranks have nothing to add)
            serve_bench(args)
        return
    world_size = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    worlds = load_worlds(args.workload, rank)
    config = {"workload": {"c1": "FatTree k=4, 240 flows, DCTCP (C1)",
                           "c2": "FatTree k=8, 10,000 flows x {NewReno, DCTCP, Cubic}, FIN, spraying (C2)",
                           "c2s": "FatTree k=8, 1,500 flows x {NewReno, DCTCP, Cubic}, FIN, spraying (C2 shape, small)",
                           "c4": "256 leaf-spine worlds, 1k-20k flows each (C4)",
                           "c5": "200 served-stream requests (C5 shape, TCP) as worlds"}[args.workload],
              "worlds": len(worlds), "flows_per_step": int(sum(len(w.flows) for w in worlds)),
              "l2": "flushed between steps (256 MiB write); state restored device-to-device before each step",
              "seed": 1}

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        for _ in range(args.warmup):
            cpu_sample(worlds, min(args.ref_slots, 500), threads)
        evs, walls = [], []
        for _ in range(args.steps):
            ev, wall, _ = cpu_sample(worlds, args.ref_slots, threads)
            evs.append(ev)
            walls.append(wall)
        value = sum(evs) / sum(walls)
        sample = f"the first {args.ref_slots} slots ({args.ref_slots} us simulated) of each of the {len(worlds)} worlds, one process per world"
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.mean(walls),
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                          "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": value, "unit": "events/s", "cores": min(threads, len(worlds)), "kind": "port",
                                           "sample": sample},
                          "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
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

    sim = api.Simulator(device=local_rank, host_lanes=args.host_lanes)
    for w in worlds:
        sim.add_world(w.topo, w.flows, w.params)
    sim.prepare()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
    for _ in range(args.warmup):
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
    for w in range(len(worlds)):
        est, done = sim.results(w)
        if (done < 0).any():
            print(f"warning: world {worlds[w].name}: {(done < 0).sum()} flows unfinished", file=sys.stderr)
    ms = statistics.mean(kernel_ms)
    from twins_b200 import shard
    ms_max, events_all = shard.aggregate(ms, float(events), dist, device=f"cuda:{local_rank}")
    value = events_all / (ms_max / 1000.0)

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
        h2d = st2["bytes_h2d"]
        d2h = sum(len(w.flows) for w in worlds) * 32
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
    tfile = ROOT / "profiles" / "slot_kernel_traffic.json"
    if tfile.exists():
        try:
            tj = json.loads(tfile.read_text())
            # DRAM bytes per packet-event from the capture, scaled to this step's events
            traffic = tj["dram_bytes_per_event"] * events / max(1, stats["launches"])
        except Exception:
            traffic = None
    # CPU baseline: the oracle (one core) on a bounded sample of the DCTCP (or first) world
    sample_world = next((w for w in worlds if w.params.tcp == "dctcp"), worlds[0])
    ev_cpu, wall_cpu, res = cpu_sample([sample_world], args.cpu_slots, 1)
    cpu_value = ev_cpu / res[0][1]
    plain = None
    if args.workload == "c4":
        plain = plain_sample(worlds, args.plain_sample, local_rank, len(worlds) / (ms_max / 1000.0))
    ref_gpu = None
    if not args.no_ref_gpu and rank == 0:
        d = Path(tempfile.gettempdir()) / "twins_bench_ref"
        d.mkdir(exist_ok=True)
        try:
            # (C4: the plain path's sample of worlds, one at a time as the reference runs them)
            ref_worlds = [worlds[i] for i in plain["sample_worlds"]] if plain else worlds
            ref_gpu = reference_gpu(ref_worlds, d)
            if ref_gpu and "seconds_per_step" in ref_gpu:
                if plain:
                    ref_gpu["worlds_per_s"] = len(ref_worlds) / ref_gpu["seconds_per_step"]
                    ref_gpu["sample_worlds"] = plain["sample_worlds"]
                else:
                    ref_gpu["value"] = events / ref_gpu["seconds_per_step"]
                    ref_gpu["unit"] = "events/s"
        except Exception as e:
            ref_gpu = {"error": str(e)[:200]}
    out = {
        "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic", "config": config,
        "worlds_per_s": len(worlds) * world_size / (ms_max / 1000.0),
        "packet_events_per_step": events,
        "slots_per_step": stats["slots"], "slots_run_per_step": stats["slots_run"],
        "e2e": {"value": e2e_value, "unit": "events/s", "ms_per_step": e2e_step, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "algorithmic_bytes_per_step": alg},
        "cpu_baseline": {"value": cpu_value, "unit": "events/s", "cores": 1, "kind": "port",
                         "sample": f"oracle on the first {args.cpu_slots} slots of {sample_world.name}"},
        "clocks": clocks.summary(),
        "gpu_launches": launches,
        "graph_launches": stats["graph_launches"],
        "launch": {"grid": stats["grid"], "host_lanes": stats["host_lanes"], "warps_per_block": stats["warps_per_block"],
                   "stage_frames": stats["stage_frames"], "autotuned": bool(stats["autotuned"])},
    }
    if ref_gpu is not None:
        out["reference_gpu"] = ref_gpu
    if plain:
        out["plain"] = plain
    print(json.dumps(out))
    sim.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
