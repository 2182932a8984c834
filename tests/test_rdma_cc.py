"""The RDMA model's arithmetic (twins_b200/csrc/tr_cc.cuh) against the reference's own answers
(tests/golden/rdma_kat.json.gz, printed by the reference's src/rdma/rstep.cuh built for the CPU:
tests/golden/make_rdma_kat.py), bit for bit: ns-3.17 time and tx times (and ns-3.36's), node
addresses, ECMP hashes, INT hop words and HPCC's per-hop utilisation, and event sequences on one
queue pair for DCQCN (CNPs, alpha / decrease / increase timers), DCTCP-RDMA and HPCC (fast react,
sample feedback, pacing after a rate change). Every check runs twice: on the CPU (the header built
with g++) and, marked gpu, on a B200 (the same header built with nvcc for sm_100a, each function run
in a kernel)."""
import ctypes as C

import pytest

import rdma_shim
from rdma_shim import QpRate, bits, dbl, params, same, state, sub


@pytest.fixture(scope="module", params=["cpu", pytest.param("gpu", marks=pytest.mark.gpu)])
def rc(request, tmp_path_factory):
    lib = request.getfixturevalue("rdma_lib") if request.param == "cpu" else rdma_shim.build(tmp_path_factory.mktemp("rc_gpu"), gpu=True)
    yield lib
    assert lib.rc_failed() == 0  # (a CUDA call of the device shim failed)


@pytest.fixture(scope="module")
def kat(rdma_kat):
    return rdma_kat


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
