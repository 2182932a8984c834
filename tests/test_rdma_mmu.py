"""The RDMA model's switch buffer rules and ECMP choice (twins_b200/csrc/tr_mmu.cuh) against the
reference's own answers (tests/golden/rdma_kat.json.gz: the reference's s_forward with the egress
busy, s_start_q3 sending onto its link, and s_route, built for the CPU), bit for bit: admission
through the reserve, the shared pool and the headroom, drops, PAUSE and RESUME, ECN marking at
dequeue with the port's random stream, the INT stamp of HPCC data, and the egress port of data
and ACKs. The rules run on the CPU here (g++); tests/test_rdma_nic.py builds them for sm_100a."""
import ctypes as C

import pytest

from rdma_shim import MmuPort, MmuSwitch, dbl


@pytest.fixture(scope="module")
def mmu(rdma_lib):
    return rdma_lib


@pytest.fixture(scope="module")
def kat(rdma_kat):
    return rdma_kat


def ports(r, key):
    ing, hdrm, egr, paused, tx_bytes, queue_bytes, q0_n = r[key]
    return MmuPort(ing, hdrm, egr, paused), tx_bytes, queue_bytes, q0_n


def counters(p):
    return [p.ing, p.hdrm, p.egr, p.paused]


def test_admission(mmu, kat):
    seen = {0: 0, 1: 0, 2: 0}
    for r in kat["admit"]:
        sw = MmuSwitch(*r["sw"])
        cfg = r["cfg"][r["in"]]
        pin, _, qin, q0_in = ports(r, "pin")
        pout, _, qout, _ = ports(r, "pout")
        res = mmu.rc_mmu_admit(r["buffer"], C.byref(sw), C.byref(pin), cfg[1], cfg[2], C.byref(pout), r["size"], r["nvs"])
        assert (res & 1, res >> 1 & 1) == (r["drop"], r["pause"]), r
        assert sw.shared_used == r["shared_after"], r
        assert counters(pin) == r["pin_after"][:4] and counters(pout) == r["pout_after"][:4], r
        # (the queues, the caller's: a PAUSE frame joins the ingress port's queue 0, an admitted
        # frame the egress port's data queue)
        assert r["pin_after"][6] == q0_in + r["pause"]
        assert r["pout_after"][5] == qout + (0 if r["drop"] else r["size"])
        seen[0 if res == 0 else res] += 1
    assert all(v > 20 for v in seen.values()), seen


def test_release(mmu, kat):
    n_mark = n_resume = n_stamp = 0
    for r in kat["release"]:
        sw = MmuSwitch(*r["sw"])
        cin, cout = r["cfg"][r["in"]], r["cfg"][r["out"]]
        pin, _, _, q0_in = ports(r, "pin")
        pout, tx_bytes, qout, _ = ports(r, "pout")
        drawn = C.c_int()
        res = mmu.rc_mmu_release(r["buffer"], C.byref(sw), C.byref(pin), cin[2], C.byref(pout), r["size"], r["ecn"], cout[3], cout[4],
                                 dbl(cout[5]), r["nvs"], dbl(r["u"]), C.byref(drawn))
        assert (res >> 2 & 1, res >> 3 & 1, drawn.value) == (r["mark"], r["resume"], r["drawn"]), r
        assert sw.shared_used == r["shared_after"], r
        assert counters(pin) == r["pin_after"][:4] and counters(pout) == r["pout_after"][:4], r
        assert r["pin_after"][6] == q0_in + r["resume"]  # (RESUME joins the ingress port's queue 0)
        assert r["sent_ecn"] == (3 if res & 4 else 0)
        # the INT stamp of an HPCC data frame (not on an NVSwitch)
        hops = (C.c_ulonglong * 5)(*r["hops"])
        nhop = C.c_ushort(r["nhop"])
        if r["kind"] == 0 and r["cc"] == 3 and not r["nvs"]:
            mmu.rc_int_stamp(hops, C.byref(nhop), r["now"], tx_bytes, qout, cout[0], r["multi"])
            n_stamp += nhop.value != r["nhop"]
        assert (list(hops), nhop.value) == (r["sent_hops"], r["sent_nhop"]), r
        assert r["pout_after"][4] == tx_bytes + r["size"]
        n_mark += r["mark"]
        n_resume += r["resume"]
    assert n_mark > 20 and n_resume > 20 and n_stamp > 20


def test_ecmp_choice(mmu, kat):
    for r in kat["route"]:
        want_q = 0 if (r["ack_high_prio"] and not r["data"]) else 3
        assert r["q"] == want_q
        if r["n"] == 0:
            assert r["port"] == -1
            continue
        k = mmu.rc_ecmp_choice(r["src"], r["dst"], r["sport"], r["data"], r["seed"], r["n"])
        assert r["ports"][k] == r["port"], r
