"""The RDMA world set-up (twins_b200/csrc/tr_world.h) against the reference's build_world on every
RDMA fixture world (tests/golden/rdma/manifest.json holds, per world, the SHA-256 of each field of
the reference's world, printed by oracle/rdma_world_kat.cpp): the HPCC fork's parameters from the
config, the link wiring and port numbering, the switches' ECMP route tables, maxRtt / maxBdp,
every switch port's headroom, PFC threshold shift and ECN thresholds, and the flows (source ports,
start order, start chains) with the hosts' start lists."""
import ctypes as C
import hashlib
import json
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT

RDMA = GOLDEN / "rdma"
SHIM = ROOT / "tests" / "rdma_world.cpp"
CSRC = ROOT / "twins_b200" / "csrc"


@pytest.fixture(scope="module")
def rw(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not here")
    so = tmp_path_factory.mktemp("rw") / "librw.so"
    subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", f"-I{CSRC}", "-o", str(so), str(SHIM)], check=True)
    lib = C.CDLL(str(so))
    lib.rw_world.restype, lib.rw_world.argtypes = C.c_char_p, [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_char_p)]
    return lib


def world(rw, cfg, topo, flows="src,dst,flow_size,start_ns\n0,1,1000,1000\n"):
    err = C.c_char_p()
    out = rw.rw_world(cfg.encode(), topo.encode(), flows.encode(), C.byref(err))
    return (json.loads(out), None) if out is not None else (None, err.value.decode())


def cases():
    return json.loads((RDMA / "manifest.json").read_text())


@pytest.mark.parametrize("case", cases(), ids=lambda c: c["name"])
def test_world_equals_reference(rw, case):
    name = case["name"]
    w, err = world(rw, (RDMA / f"{name}.cfg").read_text(), (RDMA / f"{name}.topo").read_text(), (RDMA / f"{name}.csv").read_text())
    assert err is None, err
    got = {k: hashlib.sha256(json.dumps(v, separators=(",", ":")).encode()).hexdigest() for k, v in w.items()}
    assert got.keys() == case["world"].keys()
    assert [k for k in got if got[k] != case["world"][k]] == []


def test_world_refusals(rw):
    cfg = (RDMA / "ft4_incast15_hpcc.cfg").read_text()
    topo = (RDMA / "ft4_incast15_hpcc.topo").read_text()
    assert world(rw, cfg, topo)[1] is None
    assert "CC_MODE" in world(rw, cfg.replace("CC_MODE 3", "CC_MODE 2"), topo)[1]
    assert "L2_ACK_INTERVAL" in world(rw, cfg.replace("L2_ACK_INTERVAL 1", "L2_ACK_INTERVAL 0"), topo)[1]
    assert "one link" in world(rw, cfg, topo + "link h0 s1\n")[1]
    assert "not hosts" in world(rw, cfg, topo, "src,dst,flow_size,start_ns\n0,16,1000,1000\n")[1]
    # HPCC's INT header holds 5 hops: a chain of 7 switches between two hosts is refused
    chain = "hosts 2\nswitches 7\nlink h0 s0\n" + "".join(f"link s{i} s{i + 1}\n" for i in range(6)) + "link h1 s6\n"
    assert "5 switches" in world(rw, cfg, chain)[1]
    w, err = world(rw, cfg.replace("CC_MODE 3", "CC_MODE 1"), chain)
    assert err is None and w["params"][9] == 2 * 8 * 1000 + 8 * 80  # maxRtt: twice 8 links of 1 us, and 8 tx times of a 1000-byte frame at 100 Gb/s


def test_world_overrides_and_bad_ids(rw):
    """NVL_BASE_RTT and NVL_WIN replace maxRtt and maxBdp as the reference's build_world does
    (src/rdma/rmain.cu:687-690: NVL_WIN only with HAS_WIN); negative flow ids and links to nodes that
    do not exist are refused, not indexed."""
    cfg = (RDMA / "ft4_incast15_hpcc.cfg").read_text()
    topo = (RDMA / "ft4_incast15_hpcc.topo").read_text()
    base, _ = world(rw, cfg, topo)
    w, err = world(rw, cfg + "NVL_BASE_RTT 12345\nNVL_WIN 777\n", topo)
    assert err is None and w["params"][9] == 12345 and w["params"][8] == 777
    assert w["params"][:8] == base["params"][:8]
    w, err = world(rw, cfg.replace("HAS_WIN 1", "HAS_WIN 0") + "NVL_WIN 777\n", topo)
    assert err is None and w["params"][8] == 0
    assert "negative" in world(rw, cfg, topo, "src,dst,flow_size,start_ns\n-1,3,1000,1000\n")[1]
    assert "does not exist" in world(rw, cfg, topo + "link h0 s99\n")[1]
    assert "does not exist" in world(rw, cfg, "link h0 s0\n" + topo)[1]
