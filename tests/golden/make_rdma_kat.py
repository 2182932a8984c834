"""Writes tests/golden/rdma_kat.json.gz: known answers of the reference's RDMA arithmetic (time and tx
times, node addresses, ECMP hashes, INT hop words, HPCC's per-hop utilisation, and event sequences
of DCQCN, DCTCP and HPCC on one queue pair), printed by oracle/_ref/rdma_kat, which
`make -C oracle ref-rdma-kat` builds from the reference's own src/rdma/rstep.cuh for the CPU.

The fixture groups the harness's lines by function: {fn: {"keys": [...], "rows": [[...], ...]}},
nested objects flattened to dotted keys ("a.rate": the rate before the event, "b.rate" after).
Doubles stay as the hex strings of their bits.

    TWINS_REFERENCE=/path/to/reference python tests/golden/make_rdma_kat.py
"""
import gzip
import json
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
EXE = ROOT / "oracle" / "_ref" / "rdma_kat"
OUT = Path(__file__).resolve().parent / "rdma_kat.json.gz"


def flat(d, pre=""):
    out = {}
    for k, v in d.items():
        if isinstance(v, dict):
            out.update(flat(v, pre + k + "."))
        else:
            out[pre + k] = v
    return out


def main():
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref-rdma-kat"], check=True)
    lines = subprocess.run([str(EXE)], check=True, capture_output=True, text=True).stdout.splitlines()
    out = {}
    for line in lines:
        d = flat(json.loads(line))
        fn = d.pop("fn")
        g = out.setdefault(fn, {"keys": list(d), "rows": []})
        assert list(d) == g["keys"], fn
        g["rows"].append([d[k] for k in g["keys"]])
    # (mtime 0: the same answers give the same bytes)
    OUT.write_bytes(gzip.compress((json.dumps(out, separators=(",", ":")) + "\n").encode(), mtime=0))
    print(OUT, {k: len(v["rows"]) for k, v in out.items()}, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
