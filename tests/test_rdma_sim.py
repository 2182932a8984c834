"""The RDMA slot code itself (twins_b200/csrc/tr_sim.cuh over the layout of tr_layout.h), run on the
CPU by a harness of the tests (tests/rdma_sim.cpp), against the oracle's fixtures
(tests/golden/rdma/: the flow completion times and counters the reference's twins-rdma gives).
Every flow's completion time must be identical, and so must the counters line (drops, ECN marks,
PAUSE and RESUME frames, NACKs, undecided ties, overflows). The same functions run on the B200 in
the library's slot kernel (tests/test_rdma_gpu.py)."""
import ctypes as C
import json
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

RDMA = GOLDEN / "rdma"
CSRC = ROOT / "twins_b200" / "csrc"


def cases():
    return json.loads((RDMA / "manifest.json").read_text())


@pytest.fixture(scope="module")
def rs(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not here")
    so = tmp_path_factory.mktemp("rs") / "librs.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC", f"-I{CSRC}", "-o", str(so),
                    str(ROOT / "tests" / "rdma_sim.cpp")], check=True)
    lib = C.CDLL(str(so))
    lib.rs_error.restype = C.c_char_p
    lib.rs_run.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), C.POINTER(C.c_longlong),
                           C.POINTER(C.c_ulonglong), C.POINTER(C.c_longlong), C.c_int, C.c_int]
    return lib


def run(rs, names, tail_log2=20, serial_only=0):
    n = len(names)
    arr = lambda ext: (C.c_char_p * n)(*[(RDMA / f"{x}.{ext}").read_bytes() for x in names])
    nf = sum(len((RDMA / f"{x}.csv").read_text().splitlines()) - 1 for x in names)
    fct = np.zeros(nf, dtype=np.int64)
    ev = np.zeros(40, dtype=np.uint64)
    slots = C.c_longlong()
    r = rs.rs_run(n, arr("cfg"), arr("topo"), arr("csv"), fct.ctypes.data_as(C.POINTER(C.c_longlong)),
                  ev.ctypes.data_as(C.POINTER(C.c_ulonglong)), C.byref(slots), tail_log2, serial_only)
    assert r == 0, rs.rs_error().decode()
    return fct, ev


def want(name):
    rows = [tuple(int(x) for x in l.split()) for l in (RDMA / f"{name}.fct").read_text().splitlines() if l.strip()]
    n = len((RDMA / f"{name}.csv").read_text().splitlines()) - 1
    out = np.full(n, -1, dtype=np.int64)
    for i, _, f in rows:
        out[i] = f
    return out


def counters_line(ev):
    return (f"drops {ev[0]} marks {ev[1]} pauses {ev[2]} resumes {ev[3]} nacks {ev[11]} | undecided ties {ev[8]}, on lost tails {ev[9]} | "
            f"overflows: tx {ev[4]} queue {ev[5]} ackq {ev[6]} qps {ev[7]} due {ev[12]} | acks for done QPs {ev[10]}")


@pytest.mark.parametrize("serial_only", [0, 1], ids=["safe_slots", "serial"])
@pytest.mark.parametrize("case", cases(), ids=lambda c: c["name"])
def test_slot_code_equals_reference(rs, case, serial_only):
    """Both switch paths: safe slots where they apply (egress ports apart), and every slot in one
    order."""
    fct, ev = run(rs, [case["name"]], serial_only=serial_only)
    w = want(case["name"])
    bad = np.nonzero(fct != w)[0]
    assert len(bad) == 0, f"{len(bad)} of {len(w)} flows differ, first {bad[0]}: {fct[bad[0]]} vs {w[bad[0]]}"
    assert counters_line(ev) == case["counters"]


def test_batch_equals_alone(rs):
    """Worlds of different topologies and congestion controls side by side: each equals its fixture."""
    names = [c["name"] for c in cases() if c["name"].startswith(("ft4_", "ls4x8"))][::2]
    fct, _ = run(rs, names)
    at = 0
    for x in names:
        w = want(x)
        assert (fct[at:at + len(w)] == w).all(), x
        at += len(w)
