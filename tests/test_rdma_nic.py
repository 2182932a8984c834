"""The RDMA model's NIC rules (twins_b200/csrc/tr_nic.cuh) against the reference's own answers
(tests/golden/rdma_kat.json.gz, printed by the reference's src/rdma/rstep.cuh built for the CPU),
bit for bit: frame sizes, the queue pairs' round robin with the window and pacing (and the removal
of finished queue pairs), a queue pair's start, the dequeue's next data frame and pacing or the
NIC's next send, the receiver's go-back-N check with the ACK or NACK it queues, and the sender's
handling of an ACK or NACK with DCQCN, HPCC and DCTCP. The rules run on the CPU here (g++); that
the same headers build for sm_100a is checked with nvcc."""
import ctypes as C
import shutil
import subprocess

import pytest

from conftest import ROOT
from rdma_shim import CSRC, NicParams, QpRate, QpSend, RxQp, bits, params, same, state, sub

RC_NIC = ROOT / "tests" / "rdma_nic_compile.cu"


@pytest.fixture(scope="module")
def nic(rdma_lib):
    return rdma_lib


@pytest.fixture(scope="module")
def kat(rdma_kat):
    return rdma_kat


def test_frame_sizes(nic, kat):
    for r in kat["sizes"]:
        P = NicParams(seq_extra=r["seq_extra"], int_size=r["int_size"])
        out = (C.c_uint * 2)()
        nic.rc_frame_sizes(C.byref(P), r["payload"], out)
        assert list(out) == [r["data"], r["ack"]], r


def test_round_robin(nic, kat):
    picks = set()
    for r in kat["rr"]:
        P = NicParams(var_win=r["var_win"], ack_high_prio=r["ack_high_prio"])
        k = len(r["qps"])
        rates, sends = (QpRate * k)(), (QpSend * k)()
        for i, (size, nxt, una, rate, max_rate, win, na) in enumerate(r["qps"]):
            rates[i].snd_nxt, rates[i].rate, rates[i].max_rate, rates[i].win = nxt, rate, max_rate, win
            sends[i].size, sends[i].snd_una, sends[i].next_avail = size, una, na
        lst = (C.c_int * k)(*(r["list"] + [0] * (k - r["n"])))
        n = C.c_int(r["n"])
        pick = nic.rc_next_qindex(C.byref(P), r["paused"], r["ackq_n"], lst, C.byref(n), r["rr"], r["now"], rates, sends)
        assert (pick, n.value, list(lst[:n.value])) == (r["pick"], r["n_after"], r["list_after"]), r
        picks.add(pick if pick < 0 else 0)
    assert picks == {-1, -1024, 0}


def test_receiver_check(nic, kat):
    seen = set()
    for r in kat["rx"]:
        P = NicParams(seq_extra=r["seq_extra"], int_size=r["int_size"], ack_interval=r["ack_interval"], chunk=r["chunk"],
                      nack_interval=r["nack_interval"])
        rx = RxQp(r["expected"], r["last_nack"], r["nack_timer"])
        x = nic.rc_rx_check(C.byref(P), C.byref(rx), r["seq"], r["payload"], r["now"])
        seen.add(x)
        assert (rx.expected, rx.last_nack, rx.nack_timer) == (r["expected_after"], r["last_nack_after"], r["nack_timer_after"]), r
        # an ACK (1) or a NACK (2) is queued, carrying the expected byte and the frame's ECN as a CNP
        assert r["queued"] == (x in (1, 2)), r
        if x in (1, 2):
            out = (C.c_uint * 2)()
            nic.rc_frame_sizes(C.byref(P), 0, out)
            assert (r["kind"], r["ack_seq"], r["cnp"], r["size"]) == (x, rx.expected, 1 if r["ecn"] else 0, out[1]), r
    assert seen == {1, 2, 3, 4, 5}


@pytest.mark.parametrize("fn", ["ack", "ack_hp"])
def test_ack_received(nic, kat, fn):
    n_done = 0
    for r in kat[fn]:
        P = NicParams(cc=r["cc"], fast_react=r["fast_react"])
        Cp, a = params(sub(r, "P.")), sub(r, "a.")
        q = state(a)
        s = QpSend(size=r["size"], snd_una=r["snd_una"], next_avail=a["next_avail"], last_pkt=a["last_pkt"])
        hops = (C.c_ulonglong * 5)(*r["hops"])
        out = nic.rc_ack_received(C.byref(P), C.byref(Cp), C.byref(q), C.byref(s), r["seq"], r["nack"], r["cnp"], hops, r["nhop"])
        b = sub(r, "b.")
        assert same(q, b), r
        assert s.next_avail == b["next_avail"] and s.snd_una == r["snd_una_after"] and s.done == r["done"], r
        # completion: the reference stamps the flow's completion time and stops the DCQCN timers
        assert bool(out & 1) == (r["fct"] >= 0) == bool(r["done"]), r
        started = 0 if out & 1 else out >> 4
        assert started == r["started"], r
        n_done += s.done
    assert n_done > 10


def test_dequeue(nic, kat):
    """The NIC's dequeue: the round robin's pick sends its next data frame (sequence number, size,
    snd_nxt, the pacing of its next send); with none ready, the next send is scheduled at the
    earliest queue pair's time (unless one is pending)."""
    sent = scheduled = 0
    for r in kat["dequeue"]:
        P = NicParams(mtu=r["mtu"], seq_extra=4 if r["simai"] else 0, int_size=r["int_size"], var_win=r["var_win"], ns336=r["simai"])
        k = len(r["qps"])
        rates, sends = (QpRate * k)(), (QpSend * k)()
        for i, (size, nxt, una, rate, max_rate, win, na) in enumerate(r["qps"]):
            rates[i].snd_nxt, rates[i].rate, rates[i].max_rate, rates[i].win = nxt, rate, max_rate, win
            sends[i].size, sends[i].snd_una, sends[i].next_avail = size, una, na
        lst = (C.c_int * k)(*range(k))
        n = C.c_int(r["n"])
        pick = nic.rc_next_qindex(C.byref(P), 0, 0, lst, C.byref(n), r["rr"], r["now"], rates, sends)
        assert n.value == r["n_after"], r
        if pick >= 0:
            f = lst[pick]
            seq = C.c_uint()
            size = nic.rc_next_data(C.byref(P), C.byref(rates[f]), C.byref(sends[f]), r["now"], r["rate_bound"], C.byref(seq))
            assert (r["sent"], r["flow"], r["seq"], r["size"], r["rr_after"]) == (1, f, seq.value, size, pick), r
            sent += 1
        else:
            assert not r["sent"] and r["rr_after"] == r["rr"], r
            t = nic.rc_next_send_at(C.byref(P), lst, n.value, r["now"], rates, sends)
            want = r["ns_at"] if r["ns_at"] >= 0 or t < 0 else t
            assert r["ns_at_after"] == want, r
            scheduled += r["ns_at"] < 0 and t >= 0
        assert [[rates[i].snd_nxt, sends[i].last_pkt, sends[i].next_avail] for i in range(k)] == r["after"], r
    assert sent > 100 and scheduled > 10, (sent, scheduled)


def test_qp_start(nic, kat):
    for r in kat["qp_start"]:
        P = NicParams(cc=r["cc"])
        q, s = QpRate(snd_nxt=77), QpSend()
        nic.rc_qp_start(C.byref(P), C.byref(q), C.byref(s), r["size"], r["bps"], r["win"], r["base_rtt"], r["now"])
        got = (q.rate, q.max_rate, q.target, q.win, q.base_rtt, bits(q.alpha), q.first_cnp, q.cur_rate, bits(q.u), s.next_avail, q.snd_nxt, s.size)
        want = (r["rate"], r["max_rate"], r["target"], r["q_win"], r["q_base_rtt"], r["alpha"], r["first_cnp"], r["cur_rate"], r["u"],
                r["next_avail"], r["snd_nxt"], r["size"])
        assert got == want, r


def test_nic_rules_build_for_sm100a(tmp_path):
    """The rules are host and device functions: the header builds for sm_100a."""
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc is not here")
    subprocess.run(["nvcc", "-std=c++17", "--fmad=false", "-gencode", "arch=compute_100a,code=sm_100a", "-c", f"-I{CSRC}", "-o",
                    str(tmp_path / "nic.o"), str(RC_NIC)], check=True)
