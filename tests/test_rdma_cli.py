"""The twins-rdma front-end (the reference's RDMA command line over the C ABI) and the RDMA oracle's
pin on a B200.

- The reference's own twins-rdma built for sm_100a from its sources (oracle/_ref/twins-rdma) gives
  every fixture of tests/golden/rdma/ exactly (the fixtures come from its CPU build): the oracle's
  two builds agree.
- This build's twins-rdma, with the reference's arguments (config file, --topo/--flows/--out,
  KEY=VALUE overrides, --batch job files with --outdir and --path), writes the same "id start_ns
  fct_ns" files, the same counters line, and exits as the reference does: 0 when every flow is
  done, 2 when some are unfinished at the stop time.
"""
import json
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

RDMA = GOLDEN / "rdma"
CASES = json.loads((RDMA / "manifest.json").read_text())
CLI = ROOT / "twins_b200" / "lib" / "twins-rdma"
REF_GPU = ROOT / "oracle" / "_ref" / "twins-rdma"


def fct(path):
    return [tuple(int(x) for x in l.split()) for l in path.read_text().splitlines() if l.strip()]


def counters(out):
    return [x for x in out.splitlines() if x.startswith("drops ")][-1]


def stage(tmp_path, name):
    for ext in ("cfg", "topo", "csv"):
        shutil.copy(RDMA / f"{name}.{ext}", tmp_path)


@pytest.mark.skipif(not REF_GPU.exists(), reason="the reference's GPU build (make -C oracle ref-rdma) is not here")
@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_reference_gpu_build_equals_fixture(case, tmp_path):
    name = case["name"]
    stage(tmp_path, name)
    r = subprocess.run([str(REF_GPU), f"{name}.cfg", f"--topo={name}.topo", f"--flows={name}.csv", f"--out={name}.fct"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    assert fct(tmp_path / f"{name}.fct") == fct(RDMA / f"{name}.fct")
    assert counters(r.stdout + r.stderr) == case["counters"]


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_cli_equals_fixture(native_lib, case, tmp_path):
    name = case["name"]
    stage(tmp_path, name)
    r = subprocess.run([str(CLI), f"{name}.cfg", f"--topo={name}.topo", f"--flows={name}.csv", f"--out={name}.fct"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    assert fct(tmp_path / f"{name}.fct") == fct(RDMA / f"{name}.fct")
    assert counters(r.stdout) == case["counters"]
    assert r.stdout.startswith(f"flows done {case['flows']} of {case['flows']}; simulated ")


def test_cli_batch_and_overrides(native_lib, tmp_path):
    """A job file of worlds with per-world KEY=VALUE overrides, files found through --path: every
    world's DIR/name.fct equals its fixture (the override restates the fixture's own setting)."""
    names = [c["name"] for c in CASES if c["name"].startswith("ft4_")][:5]
    data = tmp_path / "data"
    data.mkdir()
    for n in names:
        stage(data, n)
    jobs = "".join(f"{n} {n}.topo {n}.csv CC_MODE={(RDMA / f'{n}.cfg').read_text().split('CC_MODE ')[1].split()[0]}\n" for n in names)
    (tmp_path / "jobs.txt").write_text("# name topo flows overrides\n" + jobs)
    out = tmp_path / "out"
    out.mkdir()
    base = data / f"{names[0]}.cfg"
    r = subprocess.run([str(CLI), str(base), "--batch=jobs.txt", f"--outdir={out}", f"--path={data}"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    for n in names:
        cfg_pfc = (RDMA / f"{n}.cfg").read_text()
        if "BUFFER_SIZE 32" not in cfg_pfc:
            continue  # (the base config's buffer differs from a PFC fixture's)
        assert fct(out / f"{n}.fct") == fct(RDMA / f"{n}.fct"), n


def test_cli_stop_time_exit_2(native_lib, tmp_path):
    """SIMULATOR_STOP_TIME=0.0001 (100 us) stops the run with flows unfinished: exit status 2 and
    only the completed flows in the output."""
    name = "ft4_uniform80_dcqcn"
    stage(tmp_path, name)
    r = subprocess.run([str(CLI), f"{name}.cfg", f"--topo={name}.topo", f"--flows={name}.csv", f"--out={name}.fct",
                        "SIMULATOR_STOP_TIME=0.0001"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 2, r.stderr[-500:]
    got = fct(tmp_path / f"{name}.fct")
    assert 0 < len(got) < case_flows(name)
    full = {i: (s, f) for i, s, f in fct(RDMA / f"{name}.fct")}
    assert all(full[i] == (s, f) and s + f < 100_000 for i, s, f in got)


@pytest.mark.skipif(not REF_GPU.exists(), reason="the reference's GPU build (make -C oracle ref-rdma) is not here")
@pytest.mark.parametrize("name,window", [("ft4_incast15_dcqcn_pfc", ""), ("ft4_uniform80_hpcc", ""), ("ls4x8_uniform120_dctcp", "200000:900000")])
def test_txtrace_equals_reference(native_lib, name, window, tmp_path):
    """--txtrace (with --from / --until) writes, line for line, the transmission trace the
    reference's twins-rdma writes for the same world: every frame put on a link with its start,
    node, device, kind, hosts, port, sequence, bytes and ECN bits (PFC frames included)."""
    stage(tmp_path, name)
    extra = []
    if window:
        a, b = window.split(":")
        extra = [f"--from={a}", f"--until={b}"]
    for binary, out in ((REF_GPU, "ref.tx"), (CLI, "ours.tx")):
        r = subprocess.run([str(binary), f"{name}.cfg", f"--topo={name}.topo", f"--flows={name}.csv", f"--out={out}.fct", f"--txtrace={out}"]
                           + extra, cwd=tmp_path, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-500:]
    ref = (tmp_path / "ref.tx").read_text().splitlines()
    ours = (tmp_path / "ours.tx").read_text().splitlines()
    assert len(ref) > 100 and ours == ref
    if window:
        assert all(200000 <= int(l.split()[0]) <= 900000 for l in ours)
    if name.endswith("_pfc"):
        assert any(l.split()[3] in "PR" for l in ours)


def test_txtrace_refuses_batch(native_lib, tmp_path):
    """As the reference: --txtrace traces one world, so a --batch run with it is refused."""
    name = "ft4_incast15_dcqcn"
    stage(tmp_path, name)
    (tmp_path / "jobs.txt").write_text(f"a {name}.topo {name}.csv\nb {name}.topo {name}.csv\n")
    r = subprocess.run([str(CLI), f"{name}.cfg", "--batch=jobs.txt", "--outdir=.", "--txtrace=t.tx"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 1 and "one world" in r.stderr


def case_flows(name):
    return next(c["flows"] for c in CASES if c["name"] == name)


@pytest.mark.skipif(not REF_GPU.exists(), reason="the reference's GPU build (make -C oracle ref-rdma) is not here")
def test_rdma_sweep_batch_equals_reference_batch(native_lib, tmp_path):
    """The reference's RDMA k=8 sweep (32 worlds: two workloads x DCQCN/HPCC x two buffer sizes x four
    ECN thresholds on its fattree8 topology) in one batch equals, world for world, the reference's
    own twins-rdma running the same worlds as its --batch."""
    from twins_b200 import api, workloads
    worlds = workloads.rdma_sweep_k8(GOLDEN)
    with api.Simulator() as sim:
        ids = [sim.add_rdma_world(w.config, w.topology, w.flows) for w in worlds]
        assert sim.run() == api.TB_OK
        got = [sim.rdma_results(i)[1] for i in ids]
    lines = []
    for w in worlds:
        workloads.write_rdma(w, tmp_path)
        kv = dict(line.split(" ", 1) for line in w.config.strip().splitlines())
        over = " ".join(f"{k}={v.replace(' ', ',')}" for k, v in kv.items() if k in ("CC_MODE", "BUFFER_SIZE", "KMIN_MAP", "KMAX_MAP"))
        lines.append(f"{w.name} {w.name}.topo {w.name}.csv {over}")
    (tmp_path / "jobs.txt").write_text("\n".join(lines) + "\n")
    (tmp_path / "out").mkdir()
    r = subprocess.run([str(REF_GPU), f"{worlds[0].name}.cfg", "--batch=jobs.txt", "--outdir=out"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-500:]
    for w, fct in zip(worlds, got):
        want = {i: f for i, _, f in fct_rows(tmp_path / "out" / f"{w.name}.fct")}
        assert len(want) == len(fct) and all(want[i] == fct[i] for i in range(len(fct))), w.name


def fct_rows(path):
    return [tuple(int(x) for x in l.split()) for l in path.read_text().splitlines() if l.strip()]
