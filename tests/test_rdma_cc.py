"""The RDMA model's arithmetic (twins_b200/csrc/tr_cc.cuh) against the reference's own answers
(tests/golden/rdma_kat.json.gz, printed by the reference's src/rdma/rstep.cuh built for the CPU:
tests/golden/make_rdma_kat.py), bit for bit: ns-3.17 time and tx times (and ns-3.36's), node
addresses, ECMP hashes, INT hop words and HPCC's per-hop utilisation, and event sequences on one
queue pair for DCQCN (CNPs, alpha / decrease / increase timers), DCTCP-RDMA and HPCC (fast react,
sample feedback, pacing after a rate change). Every check runs twice: on the CPU (the header built
with g++) and, marked gpu, on a B200 (the same header built with nvcc for sm_100a, each function run
in a kernel)."""
import ctypes as C
import gzip
import json
import shutil
import struct
import subprocess

import pytest

from conftest import GOLDEN, ROOT

SHIM = ROOT / "tests" / "rdma_cc.cpp"
SHIM_GPU = ROOT / "tests" / "rdma_cc_gpu.cu"
CSRC = ROOT / "twins_b200" / "csrc"
U64, U32, U8 = C.c_uint64, C.c_uint32, C.c_uint8


class QpRate(C.Structure):
    _fields_ = [("rate", U64), ("max_rate", U64), ("target", U64), ("snd_nxt", U64), ("base_rtt", U64), ("win", U32),
                ("alpha_cnp", U8), ("dec_cnp", U8), ("first_cnp", U8), ("rp_stage", U32), ("alpha", C.c_double),
                ("last_update_seq", U32), ("inc_stage", C.c_int32), ("cur_rate", U64), ("u", C.c_double), ("hop", U64 * 5),
                ("high_seq", U32), ("ecn_cnt", U32), ("batch", U32), ("ca_state", U32)]


class CcParams(C.Structure):
    _fields_ = [("g", C.c_double), ("rate_first_cnp", C.c_double), ("clamp", C.c_int), ("rpg_threshold", U32), ("rai", U64),
                ("rhai", U64), ("min_rate", U64), ("dctcp_rai", U64), ("u_target", C.c_double), ("mi_thresh", U32),
                ("sample_feedback", C.c_int), ("int_multi", U32), ("mtu", U32)]


def dbl(h):
    return struct.unpack("<d", struct.pack("<Q", int(h, 16)))[0]


def bits(x):
    return "0x%016x" % struct.unpack("<Q", struct.pack("<d", x))[0]


@pytest.fixture(scope="module", params=["cpu", pytest.param("gpu", marks=pytest.mark.gpu)])
def rc(request, tmp_path_factory):
    so = tmp_path_factory.mktemp("rc") / f"librc_{request.param}.so"
    if request.param == "cpu":
        if shutil.which("g++") is None:
            pytest.skip("g++ is not here")
        cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC", f"-I{CSRC}", "-o", str(so), str(SHIM)]
    else:
        cmd = ["nvcc", "-std=c++17", "-O2", "--fmad=false", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
               f"-I{CSRC}", "-o", str(so), str(SHIM_GPU)]
    subprocess.run(cmd, check=True)
    lib = C.CDLL(str(so))
    ull, qp, pp = C.c_ulonglong, C.POINTER(QpRate), C.POINTER(CcParams)
    sig = {
        "rc_failed": (C.c_int, []),
        "rc_sizes": (None, [C.POINTER(C.c_int)]),
        "rc_ns_seconds": (C.c_longlong, [C.c_double]),
        "rc_tx": (C.c_longlong, [ull, C.c_uint, C.c_int]),
        "rc_node_ip": (C.c_uint, [C.c_int]),
        "rc_ecmp": (C.c_uint, [C.c_uint] * 4),
        "rc_hop_make": (ull, [ull, ull, C.c_uint, ull, C.c_uint]),
        "rc_hop_time_delta": (ull, [ull, ull]),
        "rc_hop_bytes_delta": (ull, [ull, ull, C.c_uint]),
        "rc_hop_u": (C.c_double, [ull, ull, C.c_uint, ull, C.c_uint, C.POINTER(ull)]),
        "rc_dcqcn": (C.c_uint, [qp, pp, C.c_int]),
        "rc_dctcp": (None, [qp, pp, C.c_uint, C.c_int]),
        "rc_hpcc": (C.c_int, [qp, pp, C.POINTER(ull), C.c_int, C.c_int]),
        "rc_paced": (C.c_longlong, [C.c_longlong, C.c_int, ull, ull, C.c_uint]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    sizes = (C.c_int * 2)()
    lib.rc_sizes(sizes)
    assert (sizes[0], sizes[1]) == (C.sizeof(QpRate), C.sizeof(CcParams))
    yield lib
    assert lib.rc_failed() == 0  # (a CUDA call of the device shim failed)


@pytest.fixture(scope="module")
def kat():
    raw = json.loads(gzip.decompress((GOLDEN / "rdma_kat.json.gz").read_bytes()))
    return {fn: [dict(zip(g["keys"], r)) for r in g["rows"]] for fn, g in raw.items()}


def test_time_and_tx(rc, kat):
    assert len(kat["ns_seconds"]) >= 200
    for r in kat["ns_seconds"]:
        assert rc.rc_ns_seconds(dbl(r["x"])) == r["ns"], r
    for r in kat["tx"]:
        assert rc.rc_tx(r["bps"], r["bytes"], 0) == r["ns17"], r
        assert rc.rc_tx(r["bps"], r["bytes"], 1) == r["ns36"], r


def test_addresses_and_ecmp(rc, kat):
    for r in kat["ecmp"]:
        assert rc.rc_node_ip(r["id"]) == r["ip"]
        assert rc.rc_ecmp(*r["w"], r["seed"]) == r["h"], r


def test_int_hops(rc, kat):
    for r in kat["hop"]:
        h = [rc.rc_hop_make(r["t"][i], r["b"][i], r["q"][i], r["rate"], r["multi"]) for i in range(2)]
        assert h == r["h"], r
        assert rc.rc_hop_time_delta(h[1], h[0]) == r["dtime"]
        assert rc.rc_hop_bytes_delta(h[1], h[0], r["multi"]) == r["dbytes"]
        tau = C.c_ulonglong()
        u = rc.rc_hop_u(h[1], h[0], r["multi"], r["max_rate"], r["win"], C.byref(tau))
        # (the path's U is the largest hop's, from 0: a hop of utilisation 0 leaves U = 0, dt = 0)
        U, dt = (u, tau.value) if u > 0 else (0.0, 0)
        assert bits(U) == r["U"] and dt == r["dt"], r


def params(row):
    P = CcParams()
    for k in ("rpg_threshold", "rai", "rhai", "min_rate", "dctcp_rai", "mi_thresh", "sample_feedback", "int_multi", "mtu", "clamp"):
        setattr(P, k, row[k])
    for k in ("g", "rate_first_cnp", "u_target"):
        setattr(P, k, dbl(row[k]))
    return P


def sub(row, pre):
    return {k[len(pre):]: v for k, v in row.items() if k.startswith(pre)}


def state(d):
    """A queue pair's rate state from the fixture's fields (before or after an event)."""
    q = QpRate()
    for k in ("rate", "max_rate", "target", "snd_nxt", "base_rtt", "win", "alpha_cnp", "dec_cnp", "first_cnp", "rp_stage", "cur_rate",
              "high_seq", "ecn_cnt", "batch", "ca_state"):
        if k in d:
            setattr(q, k, d[k])
    q.alpha = dbl(d["alpha"])
    if "u" in d:
        q.u = dbl(d["u"])
    q.last_update_seq, q.inc_stage = d["lus"], d["inc"]
    q.hop[:] = d["hop"]
    return q


def same(q, d):
    """The fields of q that the fixture's state holds, against it."""
    want = dict(d)
    got = {k: getattr(q, k) for k in want if hasattr(q, k) and k not in ("alpha", "u", "hop")}
    got.update(alpha=bits(q.alpha), lus=q.last_update_seq, inc=q.inc_stage, hop=list(q.hop))
    if "u" in want:
        got["u"] = bits(q.u)
    for k in ("next_avail", "last_pkt"):
        got[k] = want[k]  # (pacing: checked by the caller)
    return got == want


def test_single_events(rc, kat):
    """One event on a queue pair in a random state (random gains, thresholds, stages, flags)."""
    for r in kat["dcqcn1"]:
        P, q = params(sub(r, "P.")), state(sub(r, "a."))
        started = rc.rc_dcqcn(C.byref(q), C.byref(P), r["ev"])
        assert started == r["started"] and same(q, sub(r, "b.")), r
    for r in kat["dctcp1"]:
        P, q = params(sub(r, "P.")), state(sub(r, "a."))
        rc.rc_dctcp(C.byref(q), C.byref(P), r["ack"], r["cnp"])
        assert same(q, sub(r, "b.")), r
    n_set = 0
    for r in kat["hpcc1"]:
        P, a = params(sub(r, "P.")), sub(r, "a.")
        q = state(a)
        old = q.rate
        s = rc.rc_hpcc(C.byref(q), C.byref(P), (C.c_ulonglong * 5)(*r["hops"]), r["nhop"], r["fast"])
        b = sub(r, "b.")
        assert s == r["set"] and same(q, b), r
        na = rc.rc_paced(a["next_avail"], 0, old, q.rate, a["last_pkt"]) if s else a["next_avail"]
        assert na == b["next_avail"], r
        n_set += s
    assert len(kat["dcqcn1"]) >= 300 and n_set > 50


def sequences(kat, name):
    ps = {r["seq"]: r for r in kat[name + "_params"]}
    qs = {r["seq"]: r for r in kat[name + "_qp"]}
    steps = {}
    for r in kat[name]:
        steps.setdefault(r["seq"], []).append(r)
    assert len(steps) >= 24
    return [(params(ps[s]), qs[s], steps[s]) for s in sorted(steps)]


def test_dcqcn_sequences(rc, kat):
    for P, q0, steps in sequences(kat, "dcqcn"):
        # a new queue pair: the line rate, target = rate, alpha 1, before its first CNP
        q = QpRate(rate=q0["rate"], max_rate=q0["max_rate"], target=q0["max_rate"], first_cnp=1, alpha=1.0)
        for r in steps:
            started = rc.rc_dcqcn(C.byref(q), C.byref(P), r["ev"])
            got = (q.rate, q.target, bits(q.alpha), q.rp_stage, q.alpha_cnp, q.dec_cnp, q.first_cnp, started)
            want = (r["rate"], r["target"], r["alpha"], r["rp_stage"], r["alpha_cnp"], r["dec_cnp"], r["first_cnp"], r["started"])
            assert got == want, (r["seq"], r["step"])


def test_dctcp_sequences(rc, kat):
    for P, q0, steps in sequences(kat, "dctcp"):
        q = QpRate(rate=q0["rate"], max_rate=q0["max_rate"], snd_nxt=q0["snd_nxt"])
        for r in steps:
            q.snd_nxt = r["snd_nxt"]
            rc.rc_dctcp(C.byref(q), C.byref(P), r["ack"], r["cnp"])
            got = (q.rate, bits(q.alpha), q.last_update_seq, q.batch, q.ecn_cnt, q.ca_state, q.high_seq)
            want = (r["rate"], r["alpha"], r["lus"], r["batch"], r["ecn_cnt"], r["ca_state"], r["high_seq"])
            assert got == want, (r["seq"], r["step"])


def test_hpcc_sequences(rc, kat):
    acks = {(r["seq"], r["step"]): r for r in kat["hpcc_ack"]}
    n_set = n_fast = 0
    for P, q0, steps in sequences(kat, "hpcc"):
        q = QpRate(rate=q0["rate"], max_rate=q0["max_rate"], cur_rate=q0["max_rate"], base_rtt=q0["base_rtt"], win=q0["win"], u=1.0)
        next_avail = q0["next_avail"]
        for r in steps:
            a = acks[(r["seq"], r["step"])]
            q.snd_nxt = a["snd_nxt"]
            old = q.rate
            hops = (C.c_ulonglong * 5)(*a["hops"])
            s = rc.rc_hpcc(C.byref(q), C.byref(P), hops, a["nhop"], a["fast"])
            if s:
                next_avail = rc.rc_paced(next_avail, 0, old, q.rate, q0["last_pkt"])
            n_set += s
            n_fast += a["fast"]
            got = (q.rate, q.cur_rate, q.inc_stage, bits(q.u), q.last_update_seq, list(q.hop), s, next_avail)
            want = (r["rate"], r["cur_rate"], r["inc"], r["u"], r["lus"], r["hop"], r["set"], r["next_avail"])
            assert got == want, (r["seq"], r["step"])
    assert n_set > 100 and n_fast > 100
