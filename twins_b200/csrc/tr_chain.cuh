// twins-b200: the RDMA model's event order (the reference's unbounded event chains): which of two
// events at the same time ns-3 runs first, from the chains of scheduling leads back to their flows'
// starts. Host and device functions over run lists (newest run first); how a kernel stores the
// runs is its own. Bit-exact with the reference's ccmp (src/rdma/rstep.cuh:380-560), which the
// oracle's known-answer vectors pin.
//
// An event's code is (lead + 1) << 5 | (31 - ordinal): its lead (the delay with which its parent
// scheduled it) and its ordinal among its parent's scheduled events. A chain is the run-length list
// of codes from the event back through its ancestors to a root (a flow's start); its hash folds
// every lead, oldest first.
#pragma once
#include "tr_cc.cuh"

namespace tr
{

constexpr int CODE_ORD_BITS = 5;
constexpr uint32_t CODE_ORD_MAX = (1u << CODE_ORD_BITS) - 1;
constexpr uint64_t CODE_LEAD_MAX = (1ull << (32 - CODE_ORD_BITS)) - 2;

struct ChainRun
{
    uint32_t code, cnt;
};

// an event's code (leads past CODE_LEAD_MAX - 1 and ordinals past 31 saturate) (reference:
// src/rdma/rstep.cuh:155-161)
TR_HD uint32_t event_code(int64_t lead, int ord)
{
    uint64_t l = (uint64_t)lead + 1;
    if (l > CODE_LEAD_MAX)
        l = CODE_LEAD_MAX;
    return (uint32_t)(l << CODE_ORD_BITS | (CODE_ORD_MAX - (uint32_t)(ord < (int)CODE_ORD_MAX ? ord : (int)CODE_ORD_MAX)));
}

// a chain's hash after one more event: splitmix64's finalizer over the event's lead (ordinals
// never enter it) (reference: src/rdma/rstep.cuh:223-231)
TR_HD uint64_t chain_hash(uint64_t h, uint32_t code)
{
    uint64_t z = h + 0x9e3779b97f4a7c15ull * ((code >> CODE_ORD_BITS) + 1ull);
    z = (z ^ z >> 30) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ z >> 27) * 0x94d049bb133111ebull;
    return z ^ z >> 31;
}

// a chain as the comparison reads it: its runs (newest first), root (1 + the flow's index in
// start order; 0: none) and hash
struct ChainView
{
    const ChainRun *runs;
    int n;
    uint32_t root;
    uint64_t hash;
};

// < 0: a's event runs first, > 0: b's, 0: the chains do not tell (reference: ccmp, ccmp_walk,
// src/rdma/rstep.cuh:409-560). Chains of distinct roots with equal hashes (their leads are equal
// all the way: lineages in lockstep) follow the order of their roots' start chains, root_rank.
// Otherwise, going back from the events: the first differing lead decides (the larger lead is
// the earlier ancestor); a chain that ends first runs first; when both end together, distinct
// roots decide by start order, else the deepest differing ordinal (the sibling scheduled first).
TR_HD int chain_order(const ChainView &a, const ChainView &b, const uint32_t *root_rank)
{
    if (a.root && b.root && a.root != b.root && a.hash == b.hash)
        return root_rank[a.root - 1] < root_rank[b.root - 1] ? -1 : 1;
    int ord = 0, ia = 0, ib = 0;
    uint32_t la = a.n ? a.runs[0].cnt : 0, lb = b.n ? b.runs[0].cnt : 0;
    for (;;)
    {
        const uint32_t ca = ia < a.n ? a.runs[ia].code : 0, cb = ib < b.n ? b.runs[ib].code : 0;
        if (ca == 0 || cb == 0)
        {
            if (ca == 0 && cb == 0)
            {
                if (a.root && b.root && a.root != b.root)
                    return a.root < b.root ? -1 : 1;
                return ord;
            }
            return ca == 0 ? -1 : 1;
        }
        if (ca >> CODE_ORD_BITS != cb >> CODE_ORD_BITS)
            return ca > cb ? -1 : 1;
        if (ca != cb)
            ord = (ca & CODE_ORD_MAX) > (cb & CODE_ORD_MAX) ? -1 : 1;
        const uint32_t m = la < lb ? la : lb;
        la -= m;
        lb -= m;
        if (la == 0 && ++ia < a.n)
            la = a.runs[ia].cnt;
        if (lb == 0 && ++ib < b.n)
            lb = b.runs[ib].cnt;
    }
}

} // namespace tr
