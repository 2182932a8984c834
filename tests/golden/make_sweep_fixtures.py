"""Copies the reference's stored ns-3 outputs of its two parameter sweeps into tests/golden/sweep/.

The reference (TwiNS) keeps sequential ns-3.46.1 outputs of an ecnK x queue x TCP sweep over two
FatTree workloads: data/ns3/sweep_k8/ (138 configurations of k=8: flows data/flows/k8_a2a30.csv and
k8_a2a50w.csv) and data/ns3/sweep_k16/ (48 of k=16: k16_a2a30.csv and k16_a2a50w.csv). Its
validation/check_sweeps.sh runs each sweep as batches of worlds (bench/sweep.py) and compares
columns 1-6 with those files. This script keeps what that comparison needs: the flow files
(copied unchanged into tests/golden/flows/) and, per configuration, columns 5-6 (established_ns,
completed_ns) in one compressed array file per sweep, after checking that columns 1-4 of every
output equal its flow file. It also copies the topology of the reference's RDMA k=8 sweep
(data/topo/fattree8.txt, for validation/hpcc/sweep_k8.txt).

    TWINS_REFERENCE=/path/to/reference python tests/golden/make_sweep_fixtures.py

Run where the reference tree exists; the tests read only the copies.
"""
from __future__ import annotations

import csv
import json
import os
import re
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
TCPS = {"TcpDctcp": "dctcp", "TcpNewReno": "newreno", "TcpCubic": "cubic"}
NAME = re.compile(r"(k\d+)_(\w+?)_(Tcp\w+)_q(\d+)_K(\d+)\.csv")


def main(ref: Path) -> None:
    out = HERE / "sweep"
    out.mkdir(exist_ok=True)
    index = {}
    for sweep in ("k8", "k16"):
        src = ref / "data" / "ns3" / f"sweep_{sweep}"
        configs, est, done = [], [], []
        flows_seen = {}
        for path in sorted(src.glob("*.csv")):
            m = NAME.fullmatch(path.name)
            assert m, path.name
            topo, wl, tcp, q, k = m.groups()
            flow_name = f"{topo}_{wl}.csv"
            if flow_name not in flows_seen:
                shutil.copyfile(ref / "data" / "flows" / flow_name, HERE / "flows" / flow_name)
                with open(HERE / "flows" / flow_name) as f:
                    flows_seen[flow_name] = [r[:4] for r in list(csv.reader(f))[1:]]
            with open(path) as f:
                rows = list(csv.reader(f))[1:]
            assert [r[:4] for r in rows] == flows_seen[flow_name], path.name
            configs.append({"name": path.stem, "k": int(topo[1:]), "flows": f"flows/{flow_name}", "tcp": TCPS[tcp],
                            "queue": int(q), "ecn_k": int(k), "rows": len(rows)})
            est.append(np.array([int(r[4]) for r in rows], dtype=np.int64))
            done.append(np.array([int(r[5]) for r in rows], dtype=np.int64))
        np.savez_compressed(out / f"{sweep}.npz", est=np.concatenate(est), done=np.concatenate(done))
        index[sweep] = configs
        print(f"{sweep}: {len(configs)} configurations")
    (out / "index.json").write_text(json.dumps(index, indent=1) + "\n")
    # the RDMA k=8 sweep's topology (the reference's validation/hpcc/sweep_k8.txt runs its worlds on
    # data/topo/fattree8.txt with the flows data/flows/k8_a2a30.csv and k8_a2a50s.csv)
    shutil.copyfile(ref / "data" / "topo" / "fattree8.txt", HERE / "topo" / "fattree8.txt")
    for f in ("k8_a2a30.csv", "k8_a2a50s.csv"):
        shutil.copyfile(ref / "data" / "flows" / f, HERE / "flows" / f)


if __name__ == "__main__":
    root = os.environ.get("TWINS_REFERENCE") or (sys.argv[1] if len(sys.argv) > 1 else "")
    if not root:
        sys.exit("set TWINS_REFERENCE (or pass the reference tree's path)")
    main(Path(root))
