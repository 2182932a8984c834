"""The RDMA oracle's fixtures (tests/golden/rdma/: FatTree k=4 and k=8 and leaf-spine worlds under
DCQCN, HPCC and DCTCP, with
ECN marks and PFC pauses, and the flow completion times that the reference's twins-rdma gives
for them, run on the CPU): every flow completes, each output line matches its flow, and, where
the CPU build of the reference is here (`make -C oracle ref-rdma-cpu`), it reproduces every
fixture exactly."""
import json
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT

RDMA = GOLDEN / "rdma"
EXE = ROOT / "oracle" / "_ref" / "twins-rdma-cpu"


def cases():
    return json.loads((RDMA / "manifest.json").read_text())


def flows(name):
    lines = (RDMA / f"{name}.csv").read_text().splitlines()[1:]
    return [tuple(int(x) for x in l.split(",")) for l in lines]


def fct(path):
    return [tuple(int(x) for x in l.split()) for l in path.read_text().splitlines() if l.strip()]


@pytest.mark.parametrize("case", cases(), ids=lambda c: c["name"])
def test_fixture_consistent(case):
    fl, out = flows(case["name"]), fct(RDMA / f"{case['name']}.fct")
    assert len(fl) == len(out) == case["flows"]
    for i, ((src, dst, size, start), (fid, start_ns, fct_ns)) in enumerate(zip(fl, out)):
        assert fid == i and start_ns == start and fct_ns > 0
    assert "overflows: tx 0 queue 0 ackq 0 qps 0 due 0" in case["counters"]


def test_coverage():
    cs = cases()
    counters = " ".join(c["counters"] for c in cs)
    assert {"dcqcn", "hpcc", "dctcp"} <= {n for c in cs for n in c["name"].split("_")}
    assert any(" pauses 0 " not in c["counters"] for c in cs) and any(" marks 0 " not in c["counters"] for c in cs), counters


@pytest.mark.skipif(not EXE.exists(), reason="the CPU build of the reference's twins-rdma (make -C oracle ref-rdma-cpu) is not here")
@pytest.mark.parametrize("case", cases(), ids=lambda c: c["name"])
def test_oracle_reproduces(case, tmp_path):
    name = case["name"]
    for ext in ("cfg", "topo", "csv"):
        shutil.copy(RDMA / f"{name}.{ext}", tmp_path)
    r = subprocess.run([str(EXE), f"{name}.cfg", f"--topo={name}.topo", f"--flows={name}.csv", f"--out={name}.fct"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    assert fct(tmp_path / f"{name}.fct") == fct(RDMA / f"{name}.fct")


@pytest.mark.skipif(not EXE.exists(), reason="the CPU build of the reference's twins-rdma (make -C oracle ref-rdma-cpu) is not here")
def test_oracle_refuses_wide_switches(tmp_path):
    """Switches of more than 32 ports run in the GPU's wide blocks: the CPU build refuses them."""
    hpl = 40
    links = [f"link h{l * hpl + j} s{l}\n" for l in range(2) for j in range(hpl)] + [f"link s{l} s{2 + s}\n" for l in range(2) for s in range(2)]
    (tmp_path / "w.topo").write_text(f"hosts {2 * hpl}\nswitches 4\n" + "".join(links))
    (tmp_path / "w.csv").write_text("src,dst,flow_size,start_ns\n0,79,10000,1000\n")
    shutil.copy(RDMA / "ft4_incast15_hpcc.cfg", tmp_path / "w.cfg")
    r = subprocess.run([str(EXE), "w.cfg", "--topo=w.topo", "--flows=w.csv", "--out=w.fct"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 3 and "wide switches" in r.stderr
