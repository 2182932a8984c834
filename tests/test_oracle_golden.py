"""The oracle (a CPU restatement of the reference's TCP model) against the golden vectors: the
stored sequential ns-3 outputs the reference validates against (data/ns3/ref, copied to
tests/golden/ by make_fixtures.py). Every flow's establishment and completion time and the
ECMP hashes must be identical. This pins the oracle before it checks the CUDA path."""
import csv
import json
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, manifest

CASES = manifest()
# the largest cases run in the GPU suite's oracle comparisons only when asked
SLOW = {"k8_a2a50s", "k16_a2a30"}


def read_ref(path):
    with open(path) as f:
        rows = list(csv.reader(f))[1:]
    return [(int(r[4]), int(r[5])) for r in rows], [(int(r[6]), int(r[7])) for r in rows]


def run_oracle(oracle_bin, case, tmp_path):
    out = tmp_path / f"{case['name']}.csv"
    hashes = tmp_path / f"{case['name']}.hash.csv"
    cmd = [str(oracle_bin), *case["args"], f"--flows={GOLDEN / case['flows']}", f"--out={out}", f"--tcp={case['tcp']}",
           f"--hash_out={hashes}"]
    r = subprocess.run(cmd, cwd=GOLDEN, capture_output=True, text=True, check=True)
    with open(out) as f:
        got = [(int(x[4]), int(x[5])) for x in list(csv.reader(f))[1:]]
    with open(hashes) as f:
        hs = [(int(x[0]), int(x[1])) for x in list(csv.reader(f))[1:]]
    return got, hs, r.stdout


@pytest.mark.parametrize("case", [c for c in CASES if c["workload"] not in SLOW], ids=lambda c: c["name"])
def test_oracle_equals_ns3(oracle_bin, case, tmp_path):
    want, want_hash = read_ref(GOLDEN / case["ns3"])
    got, hs, _ = run_oracle(oracle_bin, case, tmp_path)
    assert len(got) == len(want)
    bad = [i for i, (a, b) in enumerate(zip(got, want)) if a != b]
    assert not bad, f"{len(bad)} flows differ from ns-3, first row {bad[0]}: {got[bad[0]]} vs {want[bad[0]]}"
    # the hash KAT (reference validation/check_hashes.sh): ns-3's hash columns per connection
    assert hs == want_hash


@pytest.mark.parametrize("case", [c for c in CASES if c["workload"] in SLOW], ids=lambda c: c["name"])
def test_oracle_equals_ns3_large(oracle_bin, case, tmp_path):
    want, _ = read_ref(GOLDEN / case["ns3"])
    got, _, _ = run_oracle(oracle_bin, case, tmp_path)
    assert got == want


def test_oracle_planted_error_is_caught(oracle_bin, tmp_path):
    """A mistake planted in the oracle's input (one flow's size off by one byte) changes the
    result: the comparison is sensitive at the single-flow level."""
    case = next(c for c in CASES if c["name"] == "k8_paper_dctcp_base")
    flows = (GOLDEN / case["flows"]).read_text().splitlines()
    head, first = flows[0], flows[1].split(",")
    first[1] = str(int(first[1]) + 1)
    planted = tmp_path / "planted.csv"
    planted.write_text("\n".join([head, ",".join(first)] + flows[2:]) + "\n")
    out = tmp_path / "o.csv"
    subprocess.run([str(oracle_bin), *case["args"], f"--flows={planted}", f"--out={out}", "--tcp=dctcp"], check=True,
                   capture_output=True)
    want, _ = read_ref(GOLDEN / case["ns3"])
    with open(out) as f:
        got = [(int(x[4]), int(x[5])) for x in list(csv.reader(f))[1:]]
    assert got != want


SWEEP = json.loads((GOLDEN / "sweep" / "index.json").read_text())


def sweep_want(sweep, i):
    z = np.load(GOLDEN / "sweep" / f"{sweep}.npz")
    at = sum(c["rows"] for c in SWEEP[sweep][:i])
    n = SWEEP[sweep][i]["rows"]
    return list(zip(z["est"][at:at + n].tolist(), z["done"][at:at + n].tolist()))


@pytest.mark.parametrize("sweep,i", [("k8", 0), ("k8", 70), ("k8", 137), ("k16", 5)])
def test_oracle_equals_ns3_sweep(oracle_bin, sweep, i, tmp_path):
    """Sample configurations of the reference's ecnK x queue x TCP sweeps (the golden set of its
    batching path): the oracle equals the stored ns-3 output, which pins the sweep fixtures."""
    c = SWEEP[sweep][i]
    out = tmp_path / "out.csv"
    subprocess.run([str(oracle_bin), f"--k={c['k']}", f"--flows={GOLDEN / c['flows']}", f"--out={out}", f"--tcp={c['tcp']}",
                    f"--ecnK={c['ecn_k']}", f"--queue={c['queue']}"], capture_output=True, text=True, check=True)
    with open(out) as f:
        got = [(int(x[4]), int(x[5])) for x in list(csv.reader(f))[1:]]
    assert got == sweep_want(sweep, i)
