"""Copies the golden vectors the tests use out of the reference tree into tests/golden/.

The reference (TwiNS) stores sequential ns-3.46.1 outputs of its validation runs in
data/ns3/ref/<workload>_<Tcp>[_variant].csv (columns src,dst,flow_size,start_ns,
established_ns,completed_ns,hash_data,hash_ack), the flow files in data/flows/, the topology
arguments in data/flows/<workload>.csv.topo and topology files in data/topo/
(validation/check_exact.sh reads them the same way). This script copies a subset, unchanged,
and writes manifest.json listing each case: its flows, its ns-3 output, its topology and flags.

    TWINS_REFERENCE=/path/to/reference python tests/golden/make_fixtures.py

Run here (where the reference tree exists); the tests read only the copies.
"""
from __future__ import annotations

import json
import os
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
TCPS = {"dctcp": "TcpDctcp", "newreno": "TcpNewReno", "cubic": "TcpCubic"}

# (workload, variant, tcps): variant base | fin | spray | sprayfin | jit..jit4
CASES = [
    ("k8_paper", "base", "dctcp newreno cubic"),
    ("k8_paper", "spray", "dctcp newreno cubic"),
    ("k8_paper", "jit2", "dctcp"),
    ("k8_a2a30", "base", "dctcp newreno cubic"),
    ("k8_a2a30", "fin", "dctcp newreno cubic"),
    ("k8_a2a30", "spray", "dctcp newreno cubic"),
    ("k8_incast16", "base", "dctcp newreno cubic"),
    ("k8_fullsync", "base", "dctcp newreno cubic"),
    ("k8_fullexp", "base", "dctcp newreno cubic"),
    ("k8_a2a30b", "base", "dctcp newreno cubic"),
    ("k8_r30", "base", "dctcp newreno cubic"),
    ("k8_r30", "fin", "dctcp newreno cubic"),
    ("k8_r30", "sprayfin", "dctcp newreno cubic"),
    ("ls_paper", "base", "dctcp newreno cubic"),
    ("jf32_a2a30", "base", "dctcp newreno cubic"),
    ("jf32f_a2a50", "spray", "dctcp newreno cubic"),
    ("torus6f_a2a30", "base", "dctcp newreno cubic"),
    ("df4x9_a2a30", "spray", "dctcp newreno cubic"),
    ("k8_a2a50s", "base", "dctcp"),
    ("k16_a2a30", "base", "dctcp newreno"),
]


def topo_args(ref: Path, w: str) -> list[str]:
    t = ref / "data" / "flows" / f"{w}.csv.topo"
    if t.exists():
        for line in t.read_text().splitlines():
            if line.startswith("# twins "):
                return line[len("# twins "):].split()
    return [f"--k={w.split('_')[0][1:]}"]


def main(ref: Path) -> None:
    flows_dir = HERE / "flows"
    ns3_dir = HERE / "ns3"
    topo_dir = HERE / "topo"
    for d in (flows_dir, ns3_dir, topo_dir):
        d.mkdir(exist_ok=True)
    cases = []
    for w, variant, tcps in CASES:
        args = topo_args(ref, w)
        fixed = []
        for a in args:
            if a.startswith("--topofile=data/topo/"):
                name = a.split("/")[-1]
                shutil.copyfile(ref / "data" / "topo" / name, topo_dir / name)
                fixed.append(f"--topofile=topo/{name}")
            else:
                fixed.append(a)
        flow_name = f"{w}.csv" if variant in ("base", "fin", "spray", "sprayfin") else f"{w}_{variant}.csv"
        shutil.copyfile(ref / "data" / "flows" / flow_name, flows_dir / flow_name)
        for t in tcps.split():
            suffix = "" if variant == "base" else f"_{variant}"
            ref_name = f"{w}_{TCPS[t]}{suffix}.csv"
            shutil.copyfile(ref / "data" / "ns3" / "ref" / ref_name, ns3_dir / ref_name)
            extra = {"base": [], "fin": ["--fin=1"], "spray": ["--spray=1"], "sprayfin": ["--spray=1", "--fin=1"]}.get(variant, [])
            cases.append({"name": f"{w}_{t}_{variant}", "workload": w, "variant": variant, "tcp": t,
                          "flows": f"flows/{flow_name}", "ns3": f"ns3/{ref_name}", "args": fixed + extra})
    (HERE / "manifest.json").write_text(json.dumps(cases, indent=1) + "\n")
    print(f"{len(cases)} cases")


if __name__ == "__main__":
    root = os.environ.get("TWINS_REFERENCE") or (sys.argv[1] if len(sys.argv) > 1 else "")
    if not root:
        sys.exit("set TWINS_REFERENCE (or pass the reference tree's path)")
    main(Path(root))
