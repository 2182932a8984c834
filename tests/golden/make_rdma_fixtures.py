"""Writes tests/golden/rdma/: small RDMA worlds (our own topologies, flows and HPCC-style configs,
seeded) and their flow completion times as the reference's twins-rdma computes them, run on the
CPU (oracle/_ref/twins-rdma-cpu, which `make -C oracle ref-rdma-cpu` builds from the reference's
own src/rdma/rmain.cu). They pin the RDMA model where no GPU is at hand.

Each case: <name>.cfg (the reference's KEY VALUE config), <name>.topo, <name>.csv (flows:
src,dst,flow_size,start_ns), <name>.fct (the reference's output: id start_ns fct_ns), and a line
in manifest.json with the reference's counters line and, per field of the world the reference's
build_world makes of it (oracle/_ref/rdma_world_kat: parameters, wiring, ECMP routes, port
configurations), the SHA-256 of the field's JSON.

    TWINS_REFERENCE=/path/to/reference python tests/golden/make_rdma_fixtures.py
"""
import hashlib
import json
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
EXE = ROOT / "oracle" / "_ref" / "twins-rdma-cpu"
WORLD_KAT = ROOT / "oracle" / "_ref" / "rdma_world_kat"
OUT = Path(__file__).resolve().parent / "rdma"

# the HPCC fork's parameters, as its example configuration sets them (the file format is the
# reference's input format)
BASE_CFG = {
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


def fattree(k):
    """FatTree k: hosts, edge, aggregation and core switches, in that order."""
    h, e = k ** 3 // 4, k * k // 2
    links = []
    for x in range(e):  # edge x: hosts x*k/2 ..
        for j in range(k // 2):
            links.append((f"h{x * (k // 2) + j}", f"s{x}"))
    for pod in range(k):
        for a in range(k // 2):
            for b in range(k // 2):
                links.append((f"s{pod * (k // 2) + b}", f"s{e + pod * (k // 2) + a}"))
    for pod in range(k):
        for a in range(k // 2):
            for c in range(k // 2):
                links.append((f"s{e + pod * (k // 2) + a}", f"s{2 * e + a * (k // 2) + c}"))
    return h, e + e + (k // 2) ** 2, links


def leafspine(leaves, spines, hpl):
    links = [(f"h{l * hpl + j}", f"s{l}") for l in range(leaves) for j in range(hpl)]
    links += [(f"s{l}", f"s{leaves + s}") for l in range(leaves) for s in range(spines)]
    return leaves * hpl, leaves + spines, links


def topo_text(t):
    h, s, links = t
    return f"hosts {h}\nswitches {s}\n" + "".join(f"link {a} {b}\n" for a, b in links)


def incast(rng, hosts, n, size):
    dst = int(rng.integers(hosts))
    src = [x for x in rng.permutation(hosts).tolist() if x != dst][:n]
    return [(s, dst, size, 2000 + 37 * i) for i, s in enumerate(src)]


def uniform(rng, hosts, n, t_end):
    rows = []
    for _ in range(n):
        s, d = rng.choice(hosts, 2, replace=False).tolist()
        size = int(np.exp(rng.uniform(np.log(1e3), np.log(2e6))))
        rows.append((s, d, size, int(rng.uniform(1000, t_end))))
    return sorted(rows, key=lambda r: r[3])


def cases():
    rng = np.random.default_rng(2024)
    ft4, ls = fattree(4), leafspine(4, 2, 8)
    out = []
    for cc, name in [(1, "dcqcn"), (3, "hpcc"), (8, "dctcp")]:
        out.append((f"ft4_incast15_{name}", ft4, incast(rng, 16, 15, 400_000), {"CC_MODE": str(cc)}))
        out.append((f"ft4_uniform80_{name}", ft4, uniform(rng, 16, 80, 200_000), {"CC_MODE": str(cc)}))
        out.append((f"ls4x8_uniform120_{name}", ls, uniform(rng, 32, 120, 300_000), {"CC_MODE": str(cc)}))
    # PFC: a small buffer under an incast
    out.append(("ft4_incast15_hpcc_pfc", ft4, incast(rng, 16, 15, 300_000), {"CC_MODE": "3", "BUFFER_SIZE": "1"}))
    out.append(("ft4_incast15_dcqcn_pfc", ft4, incast(rng, 16, 15, 300_000), {"CC_MODE": "1", "BUFFER_SIZE": "1"}))
    # FatTree k=8 (128 hosts): 600 flows, and a 32-sender incast
    ft8 = fattree(8)
    for cc, name in [(1, "dcqcn"), (3, "hpcc"), (8, "dctcp")]:
        out.append((f"ft8_uniform600_{name}", ft8, uniform(rng, 128, 600, 400_000), {"CC_MODE": str(cc)}))
    out.append(("ft8_incast32_hpcc", ft8, incast(rng, 128, 32, 262_144), {"CC_MODE": "3"}))
    out.append(("ft8_incast32_dcqcn_pfc", ft8, incast(rng, 128, 32, 262_144), {"CC_MODE": "1", "BUFFER_SIZE": "2"}))
    # flows that start together (one ScheduleFlowInputs each time) and host pairs with several flows
    same = [(int(a), int(b), int(rng.integers(1000, 100_000)), int(1000 * rng.integers(1, 4)))
            for a, b in (rng.choice(16, 2, replace=False) for _ in range(60))]
    same += [(3, 7, 5000, 2000)] * 4
    out.append(("ft4_sametime64_dcqcn", ft4, same, {"CC_MODE": "1"}))
    return out


def world_digests(name):
    """The reference's world of a case, each field's JSON digested."""
    r = subprocess.run([str(WORLD_KAT), f"{name}.cfg", f"{name}.topo", f"{name}.csv"], cwd=OUT, capture_output=True, text=True, timeout=600,
                       check=True)
    return {k: hashlib.sha256(json.dumps(v, separators=(",", ":")).encode()).hexdigest() for k, v in json.loads(r.stdout).items()}


def main():
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref-rdma-cpu", "ref-rdma-world"], check=True)
    OUT.mkdir(exist_ok=True)
    manifest = []
    for name, topo, flows, over in cases():
        cfg = {**BASE_CFG, **over}
        (OUT / f"{name}.cfg").write_text("".join(f"{k} {v}\n" for k, v in cfg.items()))
        (OUT / f"{name}.topo").write_text(topo_text(topo))
        (OUT / f"{name}.csv").write_text("src,dst,flow_size,start_ns\n" + "".join(f"{s},{d},{z},{t}\n" for s, d, z, t in flows))
        r = subprocess.run([str(EXE), f"{name}.cfg", f"--topo={name}.topo", f"--flows={name}.csv", f"--out={name}.fct"], cwd=OUT,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, (name, r.returncode, r.stderr[-500:])
        counters = [x for x in (r.stdout + r.stderr).splitlines() if x.startswith("drops ")]
        manifest.append({"name": name, "flows": len(flows), "counters": counters[-1] if counters else "", "world": world_digests(name)})
        print(name, manifest[-1]["counters"])
    (OUT / "manifest.json").write_text(json.dumps(manifest, indent=1) + "\n")


if __name__ == "__main__":
    main()
