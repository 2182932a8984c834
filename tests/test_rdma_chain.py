"""The RDMA model's event order (twins_b200/csrc/tr_chain.cuh) against the reference's own answers
(tests/golden/rdma_kat.json.gz: chains grown with the reference's cpush from flows' start chains,
spilling into its shared tail ring past 6 runs, compared by its ccmp with its memo, with and
without a virtual push on either side, lineages in lockstep and siblings at two depths included),
and the chains' hashes against a fold of chain_hash over the events after their flows' starts.
The rules run on the CPU here (g++); tests/test_rdma_nic.py builds them for sm_100a."""
import collections
import ctypes as C

import pytest


@pytest.fixture(scope="module")
def ch(rdma_lib):
    return rdma_lib


@pytest.fixture(scope="module")
def kat(rdma_kat):
    return rdma_kat


def flat_runs(runs):
    return (C.c_uint * max(1, 2 * len(runs)))(*[x for r in runs for x in r])


def test_event_codes(ch):
    for lead, ord_, want in [(0, 0, (1 << 5) | 31), (999, 2, (1000 << 5) | 29), (5, 40, (6 << 5) | 0), (1 << 40, 0, (((1 << 27) - 2) << 5) | 31)]:
        assert ch.rc_event_code(lead, ord_) == want


def test_chain_order(ch, kat):
    ranks = {r["world"]: r["rank"] for r in kat["chain_rank"]}
    orders = collections.Counter()
    ties = memo_only = 0
    for r in kat["chain"]:
        assert not r["inexact"]
        rank = (C.c_uint * len(ranks[r["world"]]))(*ranks[r["world"]])
        (ra, rb), (ha, hb) = (r["a"], r["b"]), [int(h, 16) for h in r["hash"]]
        # the hash folds every lead after the flow's start (its start chain: 3 events, hash 0),
        # oldest first
        for runs, h in ((ra, ha), (rb, hb)):
            codes = [code for code, cnt in reversed(runs) for _ in range(cnt)][3:]
            x = 0
            for code in codes:
                x = ch.rc_chain_hash(x, code)
            assert x == h, r
        got = ch.rc_chain_order(flat_runs(ra), len(ra), r["root"][0], ha, flat_runs(rb), len(rb), r["root"][1], hb, rank)
        assert got == r["walk"], r
        if r["order"] != r["walk"]:
            # the reference's memo keys a decision by the two chains' ancestors' hashes, which are
            # 0 for every chain just after a flow's start: an event compared with an identical chain
            # (one that no other event has: siblings differ in their ordinals) can get an unrelated
            # cached decision there
            assert ra == rb and r["root"][0] == r["root"][1] and ha == hb, r
            memo_only += 1
            continue
        orders[got] += 1
        ties += r["root"][0] != r["root"][1] and ha == hb
    assert min(orders.values()) > 100 and ties > 10 and memo_only < 20, (orders, ties, memo_only)
