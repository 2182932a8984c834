// twins-b200: the RDMA model's slot (the network of the HPCC fork of ns-3.17 that the reference's
// twins-rdma restates): the state of NICs, queue pairs, switch ports and links in HBM, the events of
// one NIC host or one switch in one slot in ns-3's order, and the slot's end (finish, exact idle
// skip). Host and device functions: the CUDA kernel (tr_kernel.cu) runs them a warp per entity, and
// a CPU harness of the tests runs the same code an entity at a time.
//
// The model (reference: src/rdma/rstep.cuh, src/rdma/rdma.h). Time runs in slots of D ns, the
// shortest link delay: a frame that starts in slot s arrives in slot s + 1 or later, so within a slot
// every NIC and every switch handles its own events alone. A link files its frames by the slot they
// arrive in (a ring of buckets, each tagged with its slot). Simultaneous events follow ns-3's order:
// their chains of scheduling leads back to the flows' starts (tr_chain.cuh), here with their oldest
// runs in a ring of immutable tail nodes shared by all chains.
//
// Exactness: integer and IEEE double arithmetic only, no contraction (built with --fmad=false and
// -ffp-contract=off; fma() where the reference's -march=native build fuses, in tr_cc.cuh).
#pragma once
#include "tb_common.cuh"
#include "tr_chain.cuh"
#include "tr_mmu.cuh"
#include "tr_nic.cuh"

#include <climits>
#include <cstddef>

namespace tr
{

// ------------------------------------------------------------------ records
constexpr int RUNS = 6;        // a chain's inline runs (newest first); older ones in tail nodes
constexpr int MAX_DUE = 64;    // DCQCN timers a NIC runs in one slot, at most
constexpr int PG = 3;          // the data priority's queue
constexpr uint32_t PFC_BYTES = 43;

enum : uint8_t
{
    K_DATA = 0,
    K_ACK,
    K_NACK,
    K_PAUSE,
    K_RESUME
};

// an event's chain: its runs newest first, the tail node holding the runs after r[RUNS - 1] (its
// position + 1; 0: none), the hash of the leads since its root (a flow's StartApplication; 1 + the
// flow's place in start order, over all worlds)
struct Chain
{
    ChainRun r[RUNS];
    uint64_t tail;
    uint64_t hash;
    uint32_t root, pad;
};
static_assert(sizeof(Chain) == 72, "Chain");

// a run spilled out of a chain: immutable once written; pos tells whether the ring has since
// reused its place
struct TailNode
{
    uint32_t code, cnt;
    uint64_t next, pos;
};

// an entity's reserved positions of the tail ring: next .. end - 1
struct TailChunk
{
    uint64_t next, end;
};

// a frame's contents (the reference's wire format: INT hop words, flow, sequence, size, ...; 16-byte
// aligned: it moves as 16-byte words, ld_pkt)
struct alignas(16) Pkt
{
    uint64_t hop[MAX_HOP];
    uint32_t flow;
    uint32_t seq;   // data: its first byte; ACK / NACK: the receiver's next expected byte
    uint16_t size;  // bytes on the wire
    uint16_t nhop;
    uint8_t kind;
    uint8_t ecn;    // 3: congestion experienced
    uint8_t cnp;    // ACK / NACK: the ECN echo
    uint8_t q;      // PFC: the paused queue
    uint8_t inport; // queued at a switch: its ingress port
    uint8_t ord;    // on a link: the arrival's ordinal among its sender's event's
    uint16_t sport;
    uint16_t src, dst; // hosts (numbered over all worlds)
};
static_assert(sizeof(Pkt) == 64 && alignof(Pkt) == 16, "Pkt");

// a frame on a link: its arrival time, the chain of the event that sent it, its contents (16-byte
// aligned: frames move as 16-byte words, ld_frame)
struct alignas(16) Frame
{
    int64_t ts;
    Chain c;
    Pkt p;
};
static_assert(sizeof(Frame) == 144 && alignof(Frame) == 16 && offsetof(Frame, p) % 16 == 0, "Frame");

// a NIC (QbbNetDevice + RdmaEgressQueue of a host with one link)
struct Nic
{
    int64_t tc_at;        // its TransmitComplete (-1: the device is ready)
    int64_t ns_at;        // its m_nextSend (-1: none)
    int64_t wake;         // the earliest time it must run without input
    int64_t due_min;      // at most its queue pairs' earliest DCQCN timer (INT64_MAX: none)
    long long ob_last;    // its out link's last bucket tag written (slot << 16 | frames)
    uint32_t paused;      // PFC-paused queues (bits)
    int ackq_head, ackq_n;
    int qp_n, rr;         // its queue-pair list's length; the last one served
    int next_start, start_end; // its flows, in start order, still to start
    TailChunk tail;       // its positions of the tail ring
};

// a sending queue pair: its rate state (tr_cc.cuh), its NIC view (tr_nic.cuh), its DCQCN timers
struct Qp
{
    QpRate r;
    QpSend q;
    int64_t t[3]; // alpha update, rate-decrease check, rate increase (-1: none)
    TxMemo tx;    // its last tx time computed
};
struct QpChains
{
    Chain c[3];
};

// a switch port: its transmission, PAUSE state, two queues (0: PFC frames; PG: data and ACKs),
// byte counters, buffer counters as ingress and egress, ECN random stream
struct Port
{
    int64_t tc_at;
    long long ob_last;
    uint64_t tx_bytes;
    uint32_t paused;
    int q0_head, q0_n, q3_head, q3_n;
    uint32_t bytes_total;
    MmuPort mmu;
    tb::Rng rng;
    TailChunk tail; // its positions of the tail ring
};

struct SwState
{
    MmuSwitch mmu;
    uint32_t max_shift; // its ports' largest PFC threshold shift (the lowest threshold)
};

// static set-up
struct RWorld
{
    NicParams nic;
    CcParams cc;
    int ecn, qbb, rate_bound;
    uint32_t buffer_size;
    int64_t alpha_int, dec_int, rp_int; // DCQCN timer intervals (ns)
    int first_flow, n_flows;             // the world's flows (global ids)
};
struct HostInfo
{
    int world, link_in, link_out;
};
struct SwInfo
{
    int world, deg, pbase, hbase; // its world, ports, first port, its world's first host
    uint32_t seed;                 // ECMP hash seed: its node id in its world
    uint32_t rt_off;               // its routes towards its world's hosts
};
struct PortInfo
{
    int link_in, link_out;
    uint64_t bps;                  // its out link's rate
    uint32_t hdrm_cap, shift, kmin, kmax;
    double pmax;
};
struct LinkInfo
{
    int64_t delay;
    uint64_t bps;
    uint64_t moff;   // its first frame slot in msg
    uint32_t coff;   // its first bucket tag in msg_cnt
    uint16_t nb, cap;
    uint32_t rc;     // its rate's class: its row of tx times (RSim::txt)
};
constexpr int TXT_N = 9216; // frames shorter than this many bytes take their tx time from a table
struct FlowInfo
{
    int src, dst;       // hosts over all worlds
    uint64_t size;
    int64_t start;
    uint32_t sport, win;
    uint64_t base_rtt;
    Chain start_chain;
};

// the run's control: the slot, its end, the counters of the slot barrier
struct RCtl
{
    int64_t slot;
    int64_t slots_run;
    unsigned long long next_wake;
    unsigned int flows_done;
    unsigned int activity;
    unsigned int arrive, gen;
    int finished, error;
    // (TR_PROFILE builds) this slot's longest NIC and switch (ns), the last release of the barrier
    unsigned long long prof_host_max, prof_sw_max, prof_release;
};

// counters (the reference's event counters, same indices)
enum
{
    EV_DROP = 0,
    EV_MARK = 1,
    EV_PAUSE = 2,
    EV_RESUME = 3,
    EV_OVF_TX = 4,
    EV_OVF_QUEUE = 5,
    EV_OVF_ACKQ = 6,
    EV_OVF_QPS = 7,
    EV_UNDECIDED = 8,
    EV_LOST_TAIL = 9,
    EV_ACK_DONE = 10,
    EV_NACK = 11,
    EV_OVF_DUE = 12,
    EV_LATE_DATA = 13,
    EV_HOST_ARRIVALS = 20,   // frames a NIC received (packet-events at hosts)
    EV_SWITCH_ARRIVALS = 21, // frames a switch received (packet-events at switches)
    EV_HOST_FRAMES = 22,     // frames NICs sent
    EV_HOST_ACKS = 23,       // of the NICs' arrivals: ACKs and NACKs
    EV_HOST_DATA = 24,       // of the NICs' arrivals: data
    EV_HOST_EVENTS = 25,     // every NIC event (arrivals, transmissions done, sends, timers, starts)
    EV_SWITCH_EVENTS = 26,   // every switch event (arrivals, transmissions done)
    EV_PROF_SW_PHASE = 14,   // (TR_PROFILE builds) 14..18: switch slots' phases on their lane 0, summed (cycles):
                             // ports loaded, arrivals staged, safe or not decided, events, ports stored
    EV_PROF_SW_BUSY = 19,    // (TR_PROFILE builds) switch slots with events
    EV_PROF_CMPS = 30,       // (TR_PROFILE builds) chain comparisons
    EV_PROF_TAIL_LOADS = 31, // (TR_PROFILE builds) tail nodes read by them
    EV_PROF_SAFE = 32,       // (TR_PROFILE builds) switch slots run as safe slots
    EV_PROF_SERIAL = 33,     // (TR_PROFILE builds) switch slots with events run in one order
    EV_PROF_HOST_NS = 34,    // (TR_PROFILE builds) the slots' longest NIC, summed (ns)
    EV_PROF_SW_NS = 35,      // (TR_PROFILE builds) the slots' longest switch, summed (ns)
    EV_PROF_SLOT_NS = 37,    // (TR_PROFILE builds) the slots' durations, barrier to barrier, summed (ns)
    EV_PROF_LANE_EV = 38,    // (TR_PROFILE builds) the slots' most events of one switch lane, summed
    EV_PROF_LANE_EV_SLOT = 39, // (TR_PROFILE builds) this slot's most events of one switch lane
    EV_TIMEOUT = 36,
    EV_N = 40
};

// every array of a run (device pointers in the kernel, host pointers in the CPU harness)
struct RSim
{
    int H, S, F, W, P; // hosts, switches, flows, worlds, switch ports
    int64_t D;         // the slot (ns)
    int64_t max_slots;
    const RWorld *world;
    const HostInfo *hinfo;
    Nic *nic;
    Chain *h_tc, *h_ns;
    Pkt *ackq;
    int ackq_cap;
    int *qps;
    int qps_cap;
    const SwInfo *sinfo;
    SwState *sw;
    const PortInfo *pinfo;
    Port *port;
    Chain *p_tc;
    Pkt *q0, *q3;
    int q0_cap, q3_cap;
    const uint32_t *rt; // per (switch, host): first port index in rtp, count
    const uint8_t *rtp;
    const FlowInfo *flow;
    const int *start_list;
    const uint32_t *root_rank;
    Qp *qp;
    QpChains *qc;
    RxQp *rx;
    int64_t *fct;
    const LinkInfo *link;
    const int32_t *txt; // [rate classes][TXT_N]: tx_ns(rate, bytes)
    Frame *msg;
    long long *msg_cnt;
    unsigned int *pend;
    int pend_n;
    TailNode *tail;
    unsigned long long *tail_cnt;
    uint64_t tail_mask;
    unsigned long long *ev;
    RCtl *ctl;
    int serial_only; // switches run every slot's events in one order (no safe slots)
    // the transmission trace (one world): a record per frame put on a link in [tx_from, tx_until]
    struct TxRec *tx;
    unsigned long long *tx_cnt, tx_cap;
    int64_t tx_from, tx_until;
};

// a transmission as the reference's --txtrace records it (src/rdma/rdma.h TxRec): its start (ns),
// the ns-3 node (hosts, then switches) and device (port + 1), the kind, the flow's source and
// destination hosts as the frame's sender sees them (data: src, dst; ACK / NACK: dst, src; PFC:
// the queue, 0), its port, sequence, bytes and ECN bits
struct TxRec
{
    int64_t ts;
    int32_t node, dev;
    uint32_t a, b, sport, seq;
    uint16_t size;
    uint8_t kind, ecn;
};

TR_HD void trace_tx(const RSim &s, int64_t now, int node, int port, const Pkt &p)
{
    if (!s.tx || now < s.tx_from || now > s.tx_until)
        return;
#ifdef __CUDA_ARCH__
    const unsigned long long i = atomicAdd(s.tx_cnt, 1ull);
#else
    const unsigned long long i = (*s.tx_cnt)++;
#endif
    if (i >= s.tx_cap)
        return;
    TxRec &r = s.tx[i];
    r.ts = now;
    r.node = node;
    r.dev = port + 1;
    r.kind = p.kind;
    r.size = p.size;
    r.ecn = p.ecn;
    const bool pfc = p.kind == K_PAUSE || p.kind == K_RESUME, data = p.kind == K_DATA;
    r.a = pfc ? p.q : data ? p.src : p.dst;
    r.b = pfc ? 0 : data ? p.dst : p.src;
    r.sport = pfc ? 0 : p.sport;
    r.seq = pfc ? 0 : p.seq;
}

// ------------------------------------------------------------------ memory shared between entities
// Frames, bucket tags and tail nodes are written by other entities (other SMs) in earlier slots:
// read from L2, never from a stale L1 line.
#ifdef __CUDA_ARCH__
__device__ __forceinline__ long long ld_tag(const long long *p) { return __ldcg(p); }
__device__ __forceinline__ unsigned ld_flag(const unsigned *p) { return __ldcg(p); }
__device__ __forceinline__ TailNode ld_tail(const TailNode *p)
{
    TailNode n;
    const uint2 a = __ldcg(reinterpret_cast<const uint2 *>(p));
    n.code = a.x;
    n.cnt = a.y;
    n.next = __ldcg(&p->next);
    n.pos = __ldcg(&p->pos);
    return n;
}
__device__ __forceinline__ void ld_frame(Frame &f, const Frame *src)
{
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    uint4 *d = reinterpret_cast<uint4 *>(&f);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(Frame) / 16); i++)
        d[i] = __ldcg(s + i);
}
__device__ __forceinline__ unsigned long long atom_add(unsigned long long *p, unsigned long long v) { return atomicAdd(p, v); }
__device__ __forceinline__ unsigned atom_add(unsigned *p, unsigned v) { return atomicAdd(p, v); }
__device__ __forceinline__ void atom_min(unsigned long long *p, unsigned long long v) { atomicMin(p, v); }
#else
inline long long ld_tag(const long long *p) { return *p; }
inline unsigned ld_flag(const unsigned *p) { return *p; }
inline TailNode ld_tail(const TailNode *p) { return *p; }
inline void ld_frame(Frame &f, const Frame *src) { f = *src; }
inline unsigned long long atom_add(unsigned long long *p, unsigned long long v)
{
    const unsigned long long o = *p;
    *p += v;
    return o;
}
inline unsigned atom_add(unsigned *p, unsigned v)
{
    const unsigned o = *p;
    *p += v;
    return o;
}
inline void atom_min(unsigned long long *p, unsigned long long v)
{
    if (v < *p)
        *p = v;
}
#endif
TR_HD void count(const RSim &s, int i, unsigned long long n = 1) { atom_add(&s.ev[i], n); }

// ------------------------------------------------------------------ event order
// the chain of an event that the event with chain `par` schedules with `code`; a run pushed out of
// the inline runs goes to a new tail node, at the next position of the caller's chunk of the ring
// (an entity takes TAIL_CHUNK positions at a time: one shared counter for every spill was the slot
// kernel's most contended address) (reference: cpush, src/rdma/rstep.cuh:233-290)
constexpr uint64_t TAIL_CHUNK = 64;
TR_HD void chain_push(const RSim &s, Chain &out, uint32_t code, const Chain &par, TailChunk &tc)
{
    Chain c;
    if (par.r[0].code == code)
    {
        c = par;
        if (c.r[0].cnt != 0xFFFFFFFFu)
            c.r[0].cnt++;
    }
    else
    {
        c.r[0].code = code;
        c.r[0].cnt = 1;
        for (int i = 1; i < RUNS; i++)
            c.r[i] = par.r[i - 1];
        c.root = par.root;
        c.tail = par.tail;
        c.pad = 0;
        if (par.r[RUNS - 1].code)
        {
            if (tc.next == tc.end)
            {
                tc.next = atom_add(s.tail_cnt, TAIL_CHUNK) + 1;
                tc.end = tc.next + TAIL_CHUNK;
            }
            const uint64_t pos = tc.next++;
            TailNode &n = s.tail[(pos - 1) & s.tail_mask];
            n.code = par.r[RUNS - 1].code;
            n.cnt = par.r[RUNS - 1].cnt;
            n.next = par.tail;
            n.pos = pos;
            c.tail = pos;
        }
    }
    c.hash = chain_hash(par.hash, code);
    out = c;
}

// a chain's runs, newest first, as a stream of (code, repetitions): a virtual first event `code0`
// (0: none) merged into the chain's first run when equal, the inline runs, then its tail nodes
struct RunWalk
{
    const Chain *c;
    int i;          // the inline run (RUNS: in the tail; -1: the virtual event)
    uint64_t node;  // the tail node's position
    uint64_t next;
    uint32_t code;  // 0: the end
    uint32_t left;
    bool lost;      // the ring reused a tail node this chain needs

    TR_HD void start(const RSim &s, const Chain &ch, uint32_t code0)
    {
        c = &ch;
        node = next = 0;
        lost = false;
        if (code0 && ch.r[0].code == code0)
        {
            i = 0;
            code = code0;
            left = ch.r[0].cnt == 0xFFFFFFFFu ? ch.r[0].cnt : ch.r[0].cnt + 1;
        }
        else if (code0)
        {
            i = -1;
            code = code0;
            left = 1;
        }
        else
        {
            i = 0;
            load(s);
        }
    }
    TR_HD void load(const RSim &s)
    {
        if (i < RUNS)
        {
            code = c->r[i].code;
            left = c->r[i].cnt;
            if (code)
                return;
            if (i < RUNS - 1 || c->tail == 0)
                return; // (the chain ends)
            i = RUNS;
            node = c->tail;
        }
        if (node == 0)
        {
            code = 0;
            return;
        }
        const TailNode n = ld_tail(&s.tail[(node - 1) & s.tail_mask]);
#ifdef TR_PROFILE
        count(s, EV_PROF_TAIL_LOADS);
#endif
        if (n.pos != node)
        {
            lost = true;
            code = 0;
            return;
        }
        code = n.code;
        left = n.cnt;
        next = n.next;
    }
    TR_HD void step(const RSim &s)
    {
        if (i < RUNS)
        {
            i++;
            if (i == RUNS)
                node = c->tail;
        }
        else
            node = next;
        load(s);
    }
};

// which of two simultaneous events ns-3 runs first: < 0 a (its chain cpush(pa, a); pa 0: a itself),
// > 0 b, 0 undecided; *inexact: the decision met a reused tail node. The order of tr_chain.cuh's
// chain_order, over chains whose older runs lie in tail nodes (reference: ccmp and ccmp_walk,
// src/rdma/rstep.cuh:409-560, without its memo of decisions)
TR_HD int chain_cmp(const RSim &s, uint32_t pa, const Chain &a, uint32_t pb, const Chain &b, bool *inexact)
{
    *inexact = false;
    const uint64_t ha = pa ? chain_hash(a.hash, pa) : a.hash, hb = pb ? chain_hash(b.hash, pb) : b.hash;
    if (a.root && b.root && a.root != b.root && ha == hb)
        return s.root_rank[a.root - 1] < s.root_rank[b.root - 1] ? -1 : 1;
    RunWalk A, B;
    A.start(s, a, pa);
    B.start(s, b, pb);
    int ord = 0;
    for (;;)
    {
        const uint32_t ca = A.code, cb = B.code;
        if (ca == 0 || cb == 0)
        {
            *inexact = (ca == 0 && A.lost) || (cb == 0 && B.lost);
            if (ca == 0 && cb == 0)
            {
                if (a.root && b.root && a.root != b.root)
                    return a.root < b.root ? -1 : 1;
                return ord;
            }
            if (ca == 0)
                return A.lost ? ord : -1;
            return B.lost ? ord : 1;
        }
        if (ca >> CODE_ORD_BITS != cb >> CODE_ORD_BITS)
            return ca > cb ? -1 : 1;
        if (ca != cb)
            ord = (ca & CODE_ORD_MAX) > (cb & CODE_ORD_MAX) ? -1 : 1;
        // one tail node, at one place in it: the rest is a common lineage
        if (A.i >= RUNS && B.i >= RUNS && A.node == B.node && A.left == B.left)
            return ord;
        const uint32_t m = A.left < B.left ? A.left : B.left;
        A.left -= m;
        B.left -= m;
        if (A.left == 0)
            A.step(s);
        if (B.left == 0)
            B.step(s);
    }
}

// does event a (time ta, chain cpush(pa, a)) run before event b? Undecided ties keep b, the
// earlier candidate; they and decisions on reused tail nodes are counted
TR_HD bool runs_before(const RSim &s, int64_t ta, uint32_t pa, const Chain &a, int64_t tb, uint32_t pb, const Chain &b)
{
    if (ta != tb)
        return ta < tb;
    bool inexact;
#ifdef TR_PROFILE
    count(s, EV_PROF_CMPS);
#endif
    const int c = chain_cmp(s, pa, a, pb, b, &inexact);
    if (inexact)
        count(s, EV_LOST_TAIL);
    if (c == 0)
        count(s, EV_UNDECIDED);
    return c < 0;
}

// ------------------------------------------------------------------ links
// a frame's transmission time on a link (from its rate's table below TXT_N bytes: the same values)
TR_HD int64_t link_tx_ns(const RSim &s, const LinkInfo &l, uint32_t bytes)
{
    if (bytes < (uint32_t)TXT_N)
    {
#ifdef __CUDA_ARCH__
        return __ldg(&s.txt[(size_t)l.rc * TXT_N + bytes]);
#else
        return s.txt[(size_t)l.rc * TXT_N + bytes];
#endif
    }
    return tx_ns(l.bps, bytes);
}

// a sender's place in its out link's ring: the bucket of the slot its frames arrive in
struct OutLink
{
    int link;
    LinkInfo li;
    int64_t lo, hi;      // the open bucket's times (hi 0: none open)
    uint64_t base;       // its first frame in msg
    uint32_t tag_at;     // its tag in msg_cnt
    uint32_t n;          // frames in it
    long long last;      // the last tag written (kept between slots)

    TR_HD void open(const RSim &s, int l, long long last_tag)
    {
        link = l;
        li = s.link[l];
        hi = 0;
        last = last_tag;
    }
    TR_HD void flush(const RSim &s)
    {
        if (hi == 0)
            return;
        last = (long long)(lo / s.D) << 16 | n;
        s.msg_cnt[tag_at] = last;
        hi = 0;
    }
    // room for a frame arriving at ts (null: the bucket is full, counted)
    TR_HD Frame *push(const RSim &s, int64_t ts)
    {
        if (ts >= hi)
        {
            flush(s);
            const int64_t a = ts / s.D;
            const int b = (int)(a % li.nb);
            tag_at = li.coff + (uint32_t)b;
            lo = a * s.D;
            hi = lo + s.D;
            base = li.moff + (uint64_t)b * li.cap;
            n = (last >> 16) == a ? (uint32_t)(last & 0xFFFF) : 0;
            s.pend[a % s.pend_n] = 1;
        }
        if (n >= li.cap)
        {
            count(s, EV_OVF_TX);
            return nullptr;
        }
        return s.msg + base + n++;
    }
};

// the frames of a link arriving in slot t: their count and first index in msg
TR_HD int bucket_of(const RSim &s, int link, int64_t t, uint64_t *base)
{
    const LinkInfo &l = s.link[link];
    const int b = (int)(t % l.nb);
    const long long tag = ld_tag(&s.msg_cnt[l.coff + b]);
    *base = l.moff + (uint64_t)b * l.cap;
    return (tag >> 16) == t ? (int)(tag & 0xFFFF) : 0;
}

// the code of a frame's arrival: lead its tx time + the link's delay, its ordinal
TR_HD uint32_t arrival_code(const RSim &s, const LinkInfo &l, const Frame &f) { return event_code(link_tx_ns(s, l, f.p.size) + l.delay, f.p.ord); }

// ------------------------------------------------------------------ a warp's lanes
// (lanes = 1 on the CPU: every lane's share runs in turn)
#ifdef __CUDA_ARCH__
__device__ __forceinline__ void lanes_sync() { __syncwarp(); }
// the lanes of a switch: a warp (32) or the whole block
__device__ __forceinline__ void group_sync(int lanes)
{
    if (lanes <= 32)
        __syncwarp();
    else
        __syncthreads();
}
__device__ __forceinline__ void sh_add(uint32_t *p, uint32_t v) { atomicAdd(p, v); }
__device__ __forceinline__ void sh_add(int *p, int v) { atomicAdd(p, v); }
__device__ __forceinline__ void sh_sub(uint32_t *p, uint32_t v) { atomicSub(p, v); }
__device__ __forceinline__ void ld_pkt(Pkt &p, const Pkt *src)
{
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    uint4 *d = reinterpret_cast<uint4 *>(&p);
#pragma unroll
    for (int i = 0; i < 4; i++)
        d[i] = __ldcg(s + i);
}
__device__ __forceinline__ void ld_chain(Chain &c, const Chain *src)
{
    const uint2 *s = reinterpret_cast<const uint2 *>(src);
    uint2 *d = reinterpret_cast<uint2 *>(&c);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(Chain) / 8); i++)
        d[i] = __ldcg(s + i);
}
// (own data: written only by this entity's lane, so an L1 line of it is never stale)
__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }
#else
inline void lanes_sync() {}
inline void group_sync(int) {}
inline void prefetch_l1(const void *) {}
inline void sh_add(uint32_t *p, uint32_t v) { *p += v; }
inline void sh_add(int *p, int v) { *p += v; }
inline void sh_sub(uint32_t *p, uint32_t v) { *p -= v; }
inline void ld_pkt(Pkt &p, const Pkt *src) { p = *src; }
inline void ld_chain(Chain &c, const Chain *src) { c = *src; }
#endif

// an arrival of the slot staged by the lanes: what the event order and the route need (the frame
// itself stays in its link's bucket, msg[frame])
struct SArr
{
    int64_t ts;
    uint32_t acode;
    uint32_t frame;
    uint32_t flow;
    int16_t out;      // egress port (-1: a PFC frame, or no route)
    uint8_t q, in;    // its queue; its ingress port
    uint16_t size;
    uint8_t kind;
    uint8_t pre;      // a NIC's HPCC ACK: its hops' U and tau were worked out by the lanes (HPre)
    uint16_t copy;    // its frame's copy in shared memory (SwWork::fr), or NO_COPY: read from its link
};
static_assert(sizeof(SArr) == 32, "SArr");
constexpr uint16_t NO_COPY = 0xFFFF;

// an HPCC ACK's hop utilisation U and its interval, worked out ahead (hpcc_hops_u)
struct HPre
{
    double U;
    uint64_t dt;
};

constexpr int HOST_STAGE = 128; // a NIC's arrivals of a slot staged; more are read one by one
constexpr int SW_STAGE = 512;   // a switch's arrivals of a slot staged; more run unstaged, serially
constexpr int SW_FRAMES = 192;  // of them, those whose frames are copied into shared memory
constexpr int SAFE_PORTS = 32;  // switches with more ports run every slot serially

TR_HD void stage_arrival(const RSim &s, SArr &a, uint32_t frame, const LinkInfo &lin, Pkt &p)
{
    const Frame *f = &s.msg[frame];
    a.ts = (int64_t)ld_tag((const long long *)&f->ts);
    ld_pkt(p, &f->p);
    a.acode = event_code(link_tx_ns(s, lin, p.size) + lin.delay, p.ord);
    a.frame = frame;
    a.flow = p.flow;
    a.size = p.size;
    a.kind = p.kind;
    a.pre = 0;
    a.copy = NO_COPY;
    a.out = -1;
    a.q = PG;
    a.in = 0;
}

// ------------------------------------------------------------------ a NIC host's slot
struct Due
{
    int64_t at;
    int flow, kind;
};

// a NIC's running event
struct HostEv
{
    const RSim *s;
    const RWorld *w;
    int h;
    Nic n;
    OutLink out;
    int64_t now;
    Chain cur;
    int ord;   // events the running event has scheduled
    int nout;  // frames sent this slot
};

TR_HD void h_transmit(HostEv &e, Pkt p)
{
    const RSim &s = *e.s;
    const int64_t tx = link_tx_ns(*e.s, e.out.li, p.size);
    e.n.tc_at = e.now + tx;
    chain_push(s, s.h_tc[e.h], event_code(tx, e.ord++), e.cur, e.n.tail);
    p.ord = (uint8_t)(e.ord < 255 ? e.ord : 255);
    e.ord++;
    e.nout++;
    const int64_t ts = e.now + tx + e.out.li.delay;
    Frame *f = e.out.push(s, ts);
    if (!f)
        return;
    f->ts = ts;
    f->c = e.cur;
    f->p = p;
    trace_tx(s, e.now, e.h, 0, p);
}

TR_HD void h_next_send(HostEv &e, int64_t at)
{
    e.n.ns_at = at;
    chain_push(*e.s, e.s->h_ns[e.h], event_code(at - e.now, e.ord++), e.cur, e.n.tail);
}

// QbbNetDevice::DequeueAndTransmit of a host: the ACK queue first, then the next queue pair in
// round robin that can send, else the NIC's next send time
TR_HD void h_dequeue(HostEv &e)
{
    const RSim &s = *e.s;
    if (e.n.tc_at >= 0)
        return;
    int *list = s.qps + (size_t)e.h * s.qps_cap;
    auto view = [&](int f) { return QpView{s.qp[f].r, s.qp[f].q}; };
    const int idx = next_qindex(e.w->nic, e.n.paused, e.n.ackq_n, list, &e.n.qp_n, e.n.rr, e.now, view);
    if (idx == -1)
    {
        const Pkt p = s.ackq[(size_t)e.h * s.ackq_cap + e.n.ackq_head];
        e.n.ackq_head = e.n.ackq_head + 1 == s.ackq_cap ? 0 : e.n.ackq_head + 1;
        e.n.ackq_n--;
        h_transmit(e, p);
        return;
    }
    if (idx >= 0)
    {
        const int f = list[idx];
        e.n.rr = idx;
        Qp &q = s.qp[f];
        const FlowInfo &fi = s.flow[f];
        // the frame's size and sequence number first; the queue pair's pacing after its start
        const uint64_t left = bytes_left(q.r, q.q);
        const uint32_t payload = left < e.w->nic.mtu ? (uint32_t)left : e.w->nic.mtu;
        Pkt p = {};
        p.kind = K_DATA;
        p.flow = (uint32_t)f;
        p.src = (uint16_t)fi.src;
        p.dst = (uint16_t)fi.dst;
        p.sport = (uint16_t)fi.sport;
        p.seq = (uint32_t)q.r.snd_nxt;
        p.size = (uint16_t)data_size(e.w->nic, payload);
        h_transmit(e, p);
        uint32_t seq;
        next_data(e.w->nic, q.r, q.q, e.now, e.w->rate_bound != 0, &seq, &q.tx);
        return;
    }
    const int64_t t = next_send_at(e.w->nic, list, e.n.qp_n, e.now, view);
    if (e.n.ns_at < 0 && t >= 0)
        h_next_send(e, t);
}

// a DCQCN timer of flow f set for t (its NIC's lower bound follows)
TR_HD void h_timer_set(HostEv &e, int f, int kind, int64_t lead)
{
    const RSim &s = *e.s;
    Qp &q = s.qp[f];
    q.t[kind] = e.now + lead;
    if (q.t[kind] < e.n.due_min)
        e.n.due_min = q.t[kind];
    chain_push(s, s.qc[f].c[kind], event_code(lead, e.ord++), e.cur, e.n.tail);
}

// RdmaHw::ReceiveAck
TR_HD void h_ack(HostEv &e, const Pkt &p, const double *pre_u = nullptr, uint64_t pre_dt = 0)
{
    const RSim &s = *e.s;
    const RWorld &w = *e.w;
    const int f = (int)p.flow;
    Qp &q = s.qp[f];
    if (q.q.done)
    {
        count(s, EV_ACK_DONE);
        return;
    }
    const unsigned r = ack_received(w.nic, w.cc, q.r, q.q, p.seq, p.kind == K_NACK, p.cnp != 0, p.hop, p.nhop, pre_u, pre_dt, &q.tx);
    if (r & ACK_COMPLETED)
    {
        q.t[0] = q.t[1] = q.t[2] = -1;
        s.fct[f] = e.now - s.flow[f].start;
        atom_add(&s.ctl->flows_done, 1u);
    }
    if (r & ACK_CNP)
    {
        // the first CNP: the alpha update and, a nanosecond after the decrease interval, its check
        if (r >> 4 & T_ALPHA)
            h_timer_set(e, f, 0, w.alpha_int);
        if (r >> 4 & T_DEC)
            h_timer_set(e, f, 1, w.dec_int + 1);
    }
    if ((r & ACK_RATE_SET) && e.n.ns_at >= 0 && q.q.next_avail < e.n.ns_at)
        h_next_send(e, q.q.next_avail < e.now ? e.now : q.q.next_avail);
    h_dequeue(e);
}

// RdmaHw::ReceiveUdp: the receiver's go-back-N check, an ACK or NACK into the ACK queue
TR_HD void h_data(HostEv &e, const Pkt &p)
{
    const RSim &s = *e.s;
    RxQp &r = s.rx[p.flow];
    const uint32_t payload = p.size - data_hdr(e.w->nic);
    if (r.expected >= s.flow[p.flow].size)
        count(s, EV_LATE_DATA);
    const int x = rx_check(e.w->nic, r, p.seq, payload, e.now);
    if (x != RX_ACK && x != RX_NACK)
        return;
    if (x == RX_NACK)
        count(s, EV_NACK);
    Pkt a = p;
    a.kind = x == RX_ACK ? K_ACK : K_NACK;
    a.seq = r.expected;
    a.cnp = p.ecn ? 1 : 0;
    a.ecn = 0;
    a.size = (uint16_t)ack_size(e.w->nic);
    if (e.n.ackq_n >= s.ackq_cap)
    {
        count(s, EV_OVF_ACKQ);
        return;
    }
    int at = e.n.ackq_head + e.n.ackq_n;
    if (at >= s.ackq_cap)
        at -= s.ackq_cap;
    s.ackq[(size_t)e.h * s.ackq_cap + at] = a;
    e.n.ackq_n++;
    h_dequeue(e);
}

// StartApplication -> AddQueuePair -> NewQp
TR_HD void h_start(HostEv &e, int f)
{
    const RSim &s = *e.s;
    const FlowInfo &fi = s.flow[f];
    Qp &q = s.qp[f];
    qp_start(e.w->nic, q.r, q.q, fi.size, e.out.li.bps, fi.win, fi.base_rtt, e.now);
    q.t[0] = q.t[1] = q.t[2] = -1;
    if (e.n.qp_n >= s.qps_cap)
    {
        count(s, EV_OVF_QPS);
        return;
    }
    s.qps[(size_t)e.h * s.qps_cap + e.n.qp_n++] = f;
    h_dequeue(e);
}

// a DCQCN timer fires (UpdateAlphaMlx, CheckRateDecreaseMlx, RateIncEventTimerMlx): it restarts,
// the decrease check may start the increase timer
TR_HD void h_dcqcn_timer(HostEv &e, int f, int kind)
{
    const RWorld &w = *e.w;
    Qp &q = e.s->qp[f];
    if (kind == 0)
    {
        dcqcn_alpha(q.r, w.cc);
        h_timer_set(e, f, 0, w.alpha_int);
    }
    else if (kind == 1)
    {
        h_timer_set(e, f, 1, w.dec_int);
        if (dcqcn_decrease(q.r, w.cc) & T_RP)
            h_timer_set(e, f, 2, w.rp_int);
    }
    else
    {
        h_timer_set(e, f, 2, w.rp_int);
        dcqcn_increase(q.r, w.cc);
    }
}

// the DCQCN timers of a NIC due before t1, in event order, into due[] (*n); the NIC's lower bound
// made exact
TR_HD void h_collect_due(const RSim &s, int h, Nic &n, int64_t t1, Due *due, int *ndue)
{
    *ndue = 0;
    if (n.due_min >= t1)
        return;
    const int *list = s.qps + (size_t)h * s.qps_cap;
    int64_t mn = INT64_MAX;
    for (int i = 0; i < n.qp_n; i++)
    {
        const int f = list[i];
        const Qp &q = s.qp[f];
        for (int k = 0; k < 3; k++)
            if (q.t[k] >= 0 && q.t[k] < mn)
                mn = q.t[k];
        for (int k = 0; k < 3; k++)
            if (q.t[k] >= 0 && q.t[k] < t1)
            {
                if (*ndue == MAX_DUE)
                {
                    count(s, EV_OVF_DUE);
                    continue;
                }
                const Due x = {q.t[k], f, k};
                int j = (*ndue)++;
                while (j > 0 && runs_before(s, x.at, 0, s.qc[f].c[k], due[j - 1].at, 0, s.qc[due[j - 1].flow].c[due[j - 1].kind]))
                {
                    due[j] = due[j - 1];
                    j--;
                }
                due[j] = x;
            }
    }
    n.due_min = mn;
}

// A NIC host's events of slot t in ns-3's order: arrivals on its in link, its TransmitComplete,
// its next send, its DCQCN timers and its flows' starts. The lanes stage the slot's arrivals; lane 0
// runs the events. Returns (on lane 0) whether it sent or holds frames; *wake: its earliest event
// without input (INT64_MAX: none). due: room for MAX_DUE timers; stage: for HOST_STAGE arrivals.
// (reference: host_step<1>, src/rdma/rstep.cuh:1649-2114)
TR_HD bool host_events(const RSim &s, int h, int64_t t, int64_t *wake, Due *due, const SArr *stage, const HPre *pre, int na, uint64_t abase);

TR_HD bool host_slot(const RSim &s, int h, int64_t t, int64_t *wake, Due *due, SArr *stage, HPre *pre, int lane, int lanes)
{
    const HostInfo hi = s.hinfo[h];
    const int64_t t1 = (t + 1) * s.D;
    uint64_t abase;
    const int na = bucket_of(s, hi.link_in, t, &abase);
    const int64_t wake0 = s.nic[h].wake;
    if (na == 0 && wake0 >= t1)
    {
        *wake = wake0;
        return false;
    }
    if (na <= HOST_STAGE)
    {
        const LinkInfo lin = s.link[hi.link_in];
        for (int j = lane; j < na; j += lanes)
        {
            Pkt p;
            stage_arrival(s, stage[j], (uint32_t)(abase + j), lin, p);
            // the queue pair its event will read (the NIC's own records: L1 holds no stale copy)
            if (p.kind == K_ACK || p.kind == K_NACK)
            {
                prefetch_l1(&s.qp[p.flow]);
                prefetch_l1(reinterpret_cast<const char *>(&s.qp[p.flow]) + 128);
            }
            else if (p.kind == K_DATA)
                prefetch_l1(&s.rx[p.flow]);
        }
        if (lane == 0)
        {
            prefetch_l1(&s.h_tc[h]);
            prefetch_l1(&s.h_ns[h]);
        }
        lanes_sync();
        // HPCC with fast react and no sampled feedback: an ACK's hop utilisations depend only on its
        // INT words and those its queue pair holds then, the previous ACK's of the slot (or the
        // stored ones): the lanes work them out ahead (reference: src/rdma/rstep.cuh:1729-1748)
        const RWorld &w = s.world[hi.world];
        if (w.nic.cc == 3 && w.nic.fast_react && !w.cc.sample_feedback)
        {
            for (int j = lane; j < na; j += lanes)
            {
                SArr &a = stage[j];
                if (a.kind != K_ACK && a.kind != K_NACK)
                    continue;
                Pkt p;
                ld_pkt(p, &s.msg[a.frame].p);
                if (p.nhop > MAX_HOP)
                    continue;
                int k = j - 1;
                while (k >= 0 && !(stage[k].flow == a.flow && (stage[k].kind == K_ACK || stage[k].kind == K_NACK)))
                    k--;
                const QpRate &r = s.qp[a.flow].r;
                uint64_t held[MAX_HOP];
                if (k >= 0)
                {
                    Pkt pk;
                    ld_pkt(pk, &s.msg[stage[k].frame].p);
                    for (int i = 0; i < MAX_HOP; i++)
                        held[i] = pk.hop[i];
                }
                else
                    for (int i = 0; i < MAX_HOP; i++)
                        held[i] = r.hop[i];
                hpcc_hops_u(p.hop, p.nhop, held, w.cc.int_multi, r.max_rate, r.win, &pre[j].U, &pre[j].dt);
                a.pre = 1;
            }
            lanes_sync();
        }
    }
    bool act = false;
    if (lane == 0)
        act = host_events(s, h, t, wake, due, stage, pre, na, abase);
    lanes_sync();
    return act;
}

// lane 0's share of host_slot: the events
TR_HD bool host_events(const RSim &s, int h, int64_t t, int64_t *wake, Due *due, const SArr *stage, const HPre *pre, int na, uint64_t abase)
{
    const HostInfo hi = s.hinfo[h];
    const int64_t t1 = (t + 1) * s.D;
    Nic &ng = s.nic[h];
    const LinkInfo lin = s.link[hi.link_in];
    const bool staged = na <= HOST_STAGE;
    HostEv e;
    e.s = &s;
    e.w = &s.world[hi.world];
    e.h = h;
    e.n = ng;
    e.out.open(s, hi.link_out, e.n.ob_last);
    e.nout = 0;
    int ndue = 0;
    if (e.w->nic.cc == 1)
        h_collect_due(s, h, e.n, t1, due, &ndue);
    int ai = 0, di = 0;
    SArr a{};           // the next arrival
    Chain ac;           // its chain (read when a tie or its event needs it)
    bool have_a = false, have_ac = false;
    int sf_at = -1, sf = -1;
    int64_t sf_t = INT64_MAX;
    unsigned long long n_ev = 0, n_arr = 0, n_ack = 0, n_data = 0;
    for (;;)
    {
        if (!have_a && ai < na)
        {
            if (staged)
                a = stage[ai];
            else
            {
                Pkt p;
                stage_arrival(s, a, (uint32_t)(abase + ai), lin, p);
            }
            have_a = true;
            have_ac = false;
        }
        while (di < ndue && s.qp[due[di].flow].t[due[di].kind] != due[di].at)
            di++; // (stopped or moved)
        if (sf_at != e.n.next_start)
        {
            sf_at = e.n.next_start;
            sf = sf_at < e.n.start_end ? s.start_list[sf_at] : -1;
            sf_t = sf >= 0 ? s.flow[sf].start : INT64_MAX;
        }
        // candidates in the reference's order: arrival, TransmitComplete, next send, timer, start
        int64_t ct[5];
        ct[0] = have_a ? a.ts : INT64_MAX;
        ct[1] = e.n.tc_at >= 0 && e.n.tc_at < t1 ? e.n.tc_at : INT64_MAX;
        ct[2] = e.n.ns_at >= 0 && e.n.ns_at < t1 ? e.n.ns_at : INT64_MAX;
        ct[3] = di < ndue ? due[di].at : INT64_MAX;
        ct[4] = sf_t < t1 ? sf_t : INT64_MAX;
        int64_t tmin = INT64_MAX;
        for (int k = 0; k < 5; k++)
            tmin = ct[k] < tmin ? ct[k] : tmin;
        if (tmin == INT64_MAX)
            break;
        if (ct[0] == tmin && !have_ac)
        {
            ld_chain(ac, &s.msg[a.frame].c);
            have_ac = true;
        }
        auto chain_of = [&](int k) -> const Chain & {
            return k == 0 ? ac : k == 1 ? s.h_tc[h] : k == 2 ? s.h_ns[h] : k == 3 ? s.qc[due[di].flow].c[due[di].kind] : s.flow[sf].start_chain;
        };
        int bk = -1;
        for (int k = 0; k < 5; k++)
        {
            if (ct[k] != tmin)
                continue;
            if (bk < 0 || runs_before(s, tmin, k == 0 ? a.acode : 0, chain_of(k), tmin, bk == 0 ? a.acode : 0, chain_of(bk)))
                bk = k;
        }
        e.now = tmin;
        if (bk == 0)
            chain_push(s, e.cur, a.acode, ac, e.n.tail);
        else
            e.cur = chain_of(bk);
        e.ord = 0;
        n_ev++;
        if (bk == 0)
        {
            have_a = false;
            ai++;
            n_arr++;
            Pkt p;
            ld_pkt(p, &s.msg[a.frame].p);
            if (p.kind == K_DATA)
            {
                n_data++;
                h_data(e, p);
            }
            else if (p.kind == K_ACK || p.kind == K_NACK)
            {
                n_ack++;
                const bool pv = staged && a.pre;
                h_ack(e, p, pv ? &pre[ai - 1].U : nullptr, pv ? pre[ai - 1].dt : 0);
            }
            else if (e.w->qbb)
            {
                if (p.kind == K_PAUSE)
                    e.n.paused |= 1u << p.q;
                else
                {
                    e.n.paused &= ~(1u << p.q);
                    h_dequeue(e);
                }
            }
        }
        else if (bk == 1)
        {
            e.n.tc_at = -1;
            h_dequeue(e);
        }
        else if (bk == 2)
        {
            e.n.ns_at = -1;
            h_dequeue(e);
        }
        else if (bk == 3)
        {
            const Due x = due[di++];
            h_dcqcn_timer(e, x.flow, x.kind);
        }
        else
        {
            e.n.next_start++;
            h_start(e, sf);
        }
    }
    bool act = e.nout > 0;
    int64_t w = INT64_MAX;
    if (e.n.next_start < e.n.start_end)
        w = s.flow[s.start_list[e.n.next_start]].start;
    e.out.flush(s);
    e.n.ob_last = e.out.last;
    if (e.n.ackq_n > 0 || e.n.tc_at >= 0)
        act = true;
    if (e.n.ns_at >= 0 && e.n.ns_at < w)
        w = e.n.ns_at;
    if (e.w->nic.cc == 1)
    {
        // (the bound made exact again if a timer of this slot left it behind)
        if (e.n.due_min < t1)
        {
            const int *list = s.qps + (size_t)h * s.qps_cap;
            int64_t mn = INT64_MAX;
            for (int i = 0; i < e.n.qp_n; i++)
                for (int k = 0; k < 3; k++)
                {
                    const int64_t x = s.qp[list[i]].t[k];
                    mn = x >= 0 && x < mn ? x : mn;
                }
            e.n.due_min = mn;
        }
        if (e.n.due_min < w)
            w = e.n.due_min;
    }
    if (e.n.tc_at >= 0 && e.n.tc_at < w)
        w = e.n.tc_at;
    e.n.wake = w;
    ng = e.n;
    *wake = w;
    count(s, EV_HOST_EVENTS, n_ev);
    if (n_arr)
    {
        count(s, EV_HOST_ARRIVALS, n_arr);
        count(s, EV_HOST_ACKS, n_ack);
        count(s, EV_HOST_DATA, n_data);
    }
    if (e.nout)
        count(s, EV_HOST_FRAMES, (unsigned long long)e.nout);
    return act;
}

// ------------------------------------------------------------------ a switch's slot
// a switch port during the slot (in the warp's shared memory)
struct alignas(16) SwPort
{
    Port pt;
    OutLink out;
    PortInfo info;
    LinkInfo lin;          // its in link
    uint64_t abase;        // its arrivals' bucket in msg
    int an, first;         // its arrivals this slot; the first one's place among the staged
    int nout;              // frames it sent this slot
    int ai, aend;          // the serial path's cursor over its arrivals
    uint32_t ing0, abytes; // safe slots: its ingress bytes at the slot's start; bytes arriving on it for queue PG
    int ocnt, obase;       // safe slots: arrivals leaving by it; their place in the order array
    SArr pa;               // the unstaged serial path's next arrival
    bool have_pa;
    Chain tc;              // its TransmitComplete's chain, for the slot (p_tc)
};

// the warp's switch workspace (shared memory): its ports, staged arrivals, a safe lane's order
struct SwWork
{
    SwPort *port;  // [deg]
    Frame *fr;     // [SW_FRAMES] copies of the first staged arrivals' frames
    SArr *arr;     // [SW_STAGE]
    uint16_t *ord; // [SW_STAGE]: per egress port, its arrivals in event order
    int *flags;    // [4]: ports with an event, arrivals, safe, (unused)
};

struct SwEv
{
    const RSim *s;
    const RWorld *w;
    int x;
    SwInfo si;
    MmuSwitch mmu;
    SwPort *pe;
    bool safe; // no buffer decision can occur in this slot: lanes run egress ports apart
    TailChunk *tail; // the tail positions of the running event's port (its lane's alone)
    int64_t now;
    Chain cur;
    int ord;
    unsigned long long n_ev, n_arr;
};

TR_HD void s_transmit(SwEv &e, int port, Pkt p)
{
    const RSim &s = *e.s;
    SwPort &pe = e.pe[port];
    const int64_t tx = link_tx_ns(s, pe.out.li, p.size);
    pe.pt.tc_at = e.now + tx;
    chain_push(s, pe.tc, event_code(tx, e.ord++), e.cur, *e.tail);
    p.ord = (uint8_t)(e.ord < 255 ? e.ord : 255);
    e.ord++;
    pe.nout++;
    const int64_t ts = e.now + tx + pe.out.li.delay;
    Frame *f = pe.out.push(s, ts);
    if (!f)
        return;
    f->ts = ts;
    f->c = e.cur;
    f->p = p;
    trace_tx(s, e.now, s.H + e.x, port, p);
}

TR_HD void s_enqueue(SwEv &e, int port, int q, const Pkt &p)
{
    const RSim &s = *e.s;
    Port &pt = e.pe[port].pt;
    const size_t pi = (size_t)e.si.pbase + port;
    if (q == 0)
    {
        if (pt.q0_n >= s.q0_cap)
        {
            count(s, EV_OVF_QUEUE);
            return;
        }
        int at = pt.q0_head + pt.q0_n;
        if (at >= s.q0_cap)
            at -= s.q0_cap;
        s.q0[pi * s.q0_cap + at] = p;
        pt.q0_n++;
    }
    else
    {
        if (pt.q3_n >= s.q3_cap)
        {
            count(s, EV_OVF_QUEUE);
            return;
        }
        int at = pt.q3_head + pt.q3_n;
        if (at >= s.q3_cap)
            at -= s.q3_cap;
        s.q3[pi * s.q3_cap + at] = p;
        pt.q3_n++;
    }
    pt.bytes_total += p.size;
}

// queue 0 (PFC frames) goes first; its frames pass no buffer accounting
TR_HD void s_start_q0(SwEv &e, int port)
{
    const RSim &s = *e.s;
    Port &pt = e.pe[port].pt;
    if (pt.tc_at >= 0)
        return;
    const Pkt p = s.q0[((size_t)e.si.pbase + port) * s.q0_cap + pt.q0_head];
    pt.q0_head = pt.q0_head + 1 == s.q0_cap ? 0 : pt.q0_head + 1;
    pt.q0_n--;
    pt.bytes_total -= p.size;
    pt.tx_bytes += p.size;
    s_transmit(e, port, p);
}

// QbbNetDevice::SendPfc
TR_HD void s_send_pfc(SwEv &e, int port, bool resume)
{
    Pkt p = {};
    p.kind = resume ? K_RESUME : K_PAUSE;
    p.q = PG;
    p.size = (uint16_t)PFC_BYTES;
    count(*e.s, resume ? EV_RESUME : EV_PAUSE);
    s_enqueue(e, port, 0, p);
    if (e.pe[port].pt.q0_n > 0)
        s_start_q0(e, port);
}

// a frame of queue PG leaves: the buffer gives its bytes back, ECN may mark it, a paused ingress
// may resume, an HPCC data frame takes the port's INT word; then TransmitStart. In a safe slot only
// the ingress and egress byte counts change (no headroom is in use and no port is paused).
TR_HD void s_start_q3(SwEv &e, int port, Pkt p)
{
    const RWorld &w = *e.w;
    SwPort &pe = e.pe[port];
    SwPort &in = e.pe[p.inport];
    tb::Rng &rng = pe.pt.rng;
    unsigned r;
    if (e.safe)
    {
        sh_sub(&in.pt.mmu.ing, p.size);
        pe.pt.mmu.egr -= p.size;
        r = 0;
        if (w.ecn)
        {
            const uint32_t egr = pe.pt.mmu.egr;
            if (egr > pe.info.kmax)
                r = MMU_MARK;
            else if (egr > pe.info.kmin &&
                     tb::rand_u01(rng) < pe.info.pmax * (double)(egr - pe.info.kmin) / (double)(pe.info.kmax - pe.info.kmin))
                r = MMU_MARK;
        }
    }
    else
        r = mmu_release(w.buffer_size, e.mmu, in.pt.mmu, in.info.shift, pe.pt.mmu, p.size, w.ecn != 0, pe.info.kmin, pe.info.kmax,
                        pe.info.pmax, false, [&]() { return tb::rand_u01(rng); });
    if (r & MMU_MARK)
    {
        p.ecn = 3;
        count(*e.s, EV_MARK);
    }
    if (r & MMU_RESUME)
        s_send_pfc(e, p.inport, true);
    if (p.kind == K_DATA && w.nic.cc == 3)
        int_stamp(p.hop, p.nhop, e.now, pe.pt.tx_bytes, pe.pt.bytes_total, pe.info.bps, w.cc.int_multi);
    pe.pt.tx_bytes += p.size;
    s_transmit(e, port, p);
}

// QbbNetDevice::DequeueAndTransmit of a switch port
TR_HD void s_dequeue(SwEv &e, int port)
{
    const RSim &s = *e.s;
    Port &pt = e.pe[port].pt;
    if (pt.tc_at >= 0)
        return;
    if (pt.q0_n > 0)
    {
        s_start_q0(e, port);
        return;
    }
    if ((pt.paused >> PG & 1) || pt.q3_n == 0)
        return;
    const Pkt p = s.q3[((size_t)e.si.pbase + port) * s.q3_cap + pt.q3_head];
    pt.q3_head = pt.q3_head + 1 == s.q3_cap ? 0 : pt.q3_head + 1;
    pt.q3_n--;
    pt.bytes_total -= p.size;
    s_start_q3(e, port, p);
}

// the egress port and queue of a data frame or ACK (-1: no route) (SwitchNode::GetOutDev)
TR_HD int s_route(const RSim &s, const SwInfo &si, const RWorld &w, const Pkt &p, int *q)
{
    const bool data = p.kind == K_DATA;
    *q = (w.nic.ack_high_prio && !data) ? 0 : PG;
    // (an ACK carries its data frame's hosts: it travels from dst to src)
    const int src = p.src - si.hbase, dst = p.dst - si.hbase, to = data ? dst : src;
    const uint32_t off = s.rt[2 * ((size_t)si.rt_off + to)], n = s.rt[2 * ((size_t)si.rt_off + to) + 1];
    if (n == 0)
        return -1;
    return s.rtp[off + ecmp_choice(src, dst, p.sport, data, si.seed, (int)n)];
}

// SwitchNode::SendToDev: admission, PFC, then the egress port's queue (or straight on when idle)
TR_HD void s_forward(SwEv &e, int inport, Pkt p, int out, int q)
{
    if (out < 0)
        return;
    if (q != 0)
    {
        if (e.safe)
        {
            // below every threshold for the whole slot: no drop, no headroom, no PAUSE
            sh_add(&e.pe[inport].pt.mmu.ing, (uint32_t)p.size);
            e.pe[out].pt.mmu.egr += p.size;
        }
        else
        {
            SwPort &in = e.pe[inport];
            const unsigned r = mmu_admit(e.w->buffer_size, e.mmu, in.pt.mmu, in.info.hdrm_cap, in.info.shift, e.pe[out].pt.mmu, p.size, false);
            if (r & MMU_DROP)
            {
                count(*e.s, EV_DROP);
                return;
            }
            if (r & MMU_PAUSE)
                s_send_pfc(e, inport, false);
        }
    }
    p.inport = (uint8_t)inport;
    Port &o = e.pe[out].pt;
    if (q != 0 && o.tc_at < 0 && o.q0_n == 0 && o.q3_n == 0 && !(o.paused >> PG & 1))
    {
        s_start_q3(e, out, p);
        return;
    }
    s_enqueue(e, out, q, p);
    s_dequeue(e, out);
}

// a staged arrival's chain and contents: its copy in shared memory, or read from its link
TR_HD void arr_chain(const RSim &s, const SwWork &w, const SArr &a, Chain &c)
{
    if (a.copy != NO_COPY)
        c = w.fr[a.copy].c;
    else
        ld_chain(c, &s.msg[a.frame].c);
}
TR_HD void arr_pkt(const RSim &s, const SwWork &w, const SArr &a, Pkt &p)
{
    if (a.copy != NO_COPY)
        p = w.fr[a.copy].p;
    else
        ld_pkt(p, &s.msg[a.frame].p);
}

// an arrival's event: PFC frames pause or resume their port's egress; the others are forwarded
TR_HD void s_arrival(SwEv &e, const SwWork &w, const SArr &a)
{
    const RSim &s = *e.s;
    if (!e.safe)
        e.tail = &e.pe[a.in].pt.tail;
    Chain c;
    arr_chain(s, w, a, c);
    chain_push(s, e.cur, a.acode, c, *e.tail);
    e.ord = 0;
    e.n_ev++;
    e.n_arr++;
    if (a.kind == K_PAUSE || a.kind == K_RESUME)
    {
        if (e.w->qbb)
        {
            Pkt p;
            arr_pkt(s, w, a, p);
            if (a.kind == K_PAUSE)
                e.pe[a.in].pt.paused |= 1u << p.q;
            else
            {
                e.pe[a.in].pt.paused &= ~(1u << p.q);
                s_dequeue(e, a.in);
            }
        }
        return;
    }
    if (a.out < 0)
        return;
    Pkt p;
    arr_pkt(s, w, a, p);
    s_forward(e, a.in, p, a.out, a.q);
}

// a port's TransmitComplete
TR_HD void s_tc(SwEv &e, int port)
{
    if (!e.safe)
        e.tail = &e.pe[port].pt.tail;
    e.cur = e.pe[port].tc;
    e.ord = 0;
    e.n_ev++;
    e.pe[port].pt.tc_at = -1;
    s_dequeue(e, port);
}

// does staged arrival a run before staged arrival b (same time: by their chains)?
TR_HD bool arr_before(const RSim &s, const SwWork &w, const SArr &a, const SArr &b)
{
    if (a.ts != b.ts)
        return a.ts < b.ts;
    Chain ca, cb;
    arr_chain(s, w, a, ca);
    arr_chain(s, w, b, cb);
    return runs_before(s, a.ts, a.acode, ca, b.ts, b.acode, cb);
}

// does a port's arrival a run before its TransmitComplete at the same time?
TR_HD bool arr_before_tc(const RSim &s, const SwWork &w, const SArr &a, const Chain &tc)
{
    Chain ca;
    arr_chain(s, w, a, ca);
    return runs_before(s, a.ts, a.acode, ca, a.ts, 0, tc);
}

// A safe slot's egress port o, on its own lane: the arrivals routed to it (and PFC frames arriving
// at it) in event order, merged with its TransmitCompletes. Restricting ns-3's order to one port's
// events keeps their order, and in a safe slot ports meet only in their ingress byte counts.
TR_HD void safe_egress(SwEv &e, const SwWork &w, int o, int64_t t1, int total)
{
    const RSim &s = *e.s;
    SwPort &me = e.pe[o];
    e.tail = &me.pt.tail;
    uint16_t *list = w.ord + me.obase; // (this port's share of the order array)
    int n = 0;
    for (int j = 0; j < total; j++)
    {
        const SArr &a = w.arr[j];
        const int own = a.out >= 0 ? a.out : (a.kind == K_PAUSE || a.kind == K_RESUME ? a.in : -1);
        if (own != o)
            continue;
        // insertion in event order (an undecided tie keeps the earlier port's arrival first)
        int k = n++;
        while (k > 0 && arr_before(s, w, a, w.arr[list[k - 1]]))
        {
            list[k] = list[k - 1];
            k--;
        }
        list[k] = (uint16_t)j;
    }
    int i = 0;
    for (;;)
    {
        const int64_t ta = i < n ? w.arr[list[i]].ts : INT64_MAX, tc = me.pt.tc_at;
        const bool htc = tc >= 0 && tc < t1;
        if (ta == INT64_MAX && !htc)
            break;
        bool arr;
        if (!htc || ta == INT64_MAX)
            arr = !htc;
        else if (ta != tc)
            arr = ta < tc;
        else
            arr = arr_before_tc(s, w, w.arr[list[i]], me.tc);
        if (!arr)
        {
            e.now = tc;
            s_tc(e, o);
            continue;
        }
        const SArr &a = w.arr[list[i++]];
        e.now = a.ts;
        s_arrival(e, w, a);
    }
}

// The switch's events in one order by lane 0: every port's next arrival and TransmitComplete,
// ties by the chains (from the staged arrivals, or read from the links when they did not fit)
TR_HD void serial_events(SwEv &e, const SwWork &w, int deg, int64_t t1, bool staged)
{
    const RSim &s = *e.s;
    for (int p = 0; p < deg; p++)
    {
        SwPort &q = e.pe[p];
        q.ai = staged ? q.first : 0;
        q.aend = staged ? q.first + q.an : q.an;
        q.have_pa = false;
    }
    for (;;)
    {
        int best = -1, bk = 0;
        int64_t bt = INT64_MAX;
        const SArr *ba = nullptr;
        for (int p = 0; p < deg; p++)
        {
            SwPort &q = e.pe[p];
            const SArr *a = nullptr;
            if (q.ai < q.aend)
            {
                if (staged)
                    a = &w.arr[q.ai];
                else
                {
                    if (!q.have_pa)
                    {
                        Pkt pk;
                        stage_arrival(s, q.pa, (uint32_t)(q.abase + q.ai), q.lin, pk);
                        q.pa.in = (uint8_t)p;
                        int qi = PG;
                        q.pa.out = (int16_t)(pk.kind == K_PAUSE || pk.kind == K_RESUME ? -1 : s_route(s, e.si, *e.w, pk, &qi));
                        q.pa.q = (uint8_t)qi;
                        q.have_pa = true;
                    }
                    a = &q.pa;
                }
            }
            const int64_t ta = a ? a->ts : INT64_MAX, tc = q.pt.tc_at >= 0 && q.pt.tc_at < t1 ? q.pt.tc_at : INT64_MAX;
            for (int k = 0; k < 2; k++)
            {
                const int64_t tt = k ? tc : ta;
                if (tt == INT64_MAX || tt > bt)
                    continue;
                if (tt < bt || best < 0)
                {
                    best = p, bk = k, bt = tt, ba = a;
                    continue;
                }
                // a tie: the chains
                bool b4;
                if (k == 0 && bk == 0)
                    b4 = arr_before(s, w, *a, *ba);
                else if (k == 0)
                    b4 = arr_before_tc(s, w, *a, e.pe[best].tc);
                else if (bk == 0)
                {
                    Chain cb;
                    arr_chain(s, w, *ba, cb);
                    b4 = runs_before(s, tt, 0, e.pe[p].tc, bt, ba->acode, cb);
                }
                else
                    b4 = runs_before(s, tt, 0, e.pe[p].tc, bt, 0, e.pe[best].tc);
                if (b4)
                    best = p, bk = k, ba = a;
            }
        }
        if (best < 0)
            break;
        e.now = bt;
        if (bk == 1)
        {
            s_tc(e, best);
            continue;
        }
        const SArr a = *ba;
        SwPort &q = e.pe[best];
        q.ai++;
        q.have_pa = false;
        s_arrival(e, w, a);
    }
}

// A switch's events of slot t in ns-3's order: every port's arrivals and TransmitCompletes, by a
// group of lanes (a warp, or a block's warps). They load the ports and stage the slot's arrivals with their routes; then, when no
// buffer decision (drop, headroom, PAUSE, RESUME) can occur in the slot, each lane runs egress
// ports of its own (a safe slot), else lane 0 runs all events in one order; the lanes store the
// ports. Returns (on every lane) whether the switch sent or holds frames.
// (reference: switch_step, src/rdma/rstep.cuh:2583-3446)
#if defined(TR_PROFILE) && defined(__CUDA_ARCH__)
#define SW_PHASE(i)                                                                                                             \
    do                                                                                                                          \
    {                                                                                                                           \
        if (lane == 0)                                                                                                          \
        {                                                                                                                       \
            const long long c = clock64();                                                                                      \
            atomicAdd(&s.ev[EV_PROF_SW_PHASE + (i)], (unsigned long long)(c - ph0));                                           \
            ph0 = c;                                                                                                            \
        }                                                                                                                       \
    } while (0)
#else
#define SW_PHASE(i)                                                                                                             \
    do                                                                                                                          \
    {                                                                                                                           \
    } while (0)
#endif
TR_HD bool switch_slot(const RSim &s, int x, int64_t t, const SwWork &w, int lane, int lanes)
{
#if defined(TR_PROFILE) && defined(__CUDA_ARCH__)
    long long ph0 = clock64();
#endif
    const SwInfo si = s.sinfo[x];
    const RWorld &wp = s.world[si.world];
    const int deg = si.deg;
    const int64_t t1 = (t + 1) * s.D;
    if (lane == 0)
        w.flags[0] = w.flags[1] = w.flags[2] = w.flags[3] = 0;
    group_sync(lanes);
    for (int p = lane; p < deg; p += lanes)
    {
        SwPort &q = w.port[p];
        q.pt = s.port[si.pbase + p];
        q.info = s.pinfo[si.pbase + p];
        q.lin = s.link[q.info.link_in];
        q.out.open(s, q.info.link_out, q.pt.ob_last);
        q.an = bucket_of(s, q.info.link_in, t, &q.abase);
        q.nout = 0;
        q.abytes = 0;
        q.ocnt = 0;
        q.ing0 = q.pt.mmu.ing;
        if (q.an > 0 || (q.pt.tc_at >= 0 && q.pt.tc_at < t1))
        {
            sh_add(&w.flags[2], 1);
            q.tc = s.p_tc[si.pbase + p];
            // the queue's next frames, for the slot's dequeues
            const Pkt *q3 = s.q3 + (size_t)(si.pbase + p) * s.q3_cap;
            for (int i = 0; i < q.pt.q3_n && i < 8; i += 2)
                prefetch_l1(q3 + (q.pt.q3_head + i) % s.q3_cap);
        }
    }
    group_sync(lanes);
    if (w.flags[2] == 0)
    {
        // no event: the ports stay as they are
        bool act = false;
        for (int p = 0; p < deg; p++)
        {
            const Port &pt = w.port[p].pt;
            act |= pt.q0_n > 0 || pt.q3_n > 0 || pt.tc_at >= 0;
        }
        group_sync(lanes);
        return act;
    }
    SW_PHASE(0);
#if defined(TR_PROFILE) && defined(__CUDA_ARCH__)
    if (lane == 0)
        atomicAdd(&s.ev[EV_PROF_SW_BUSY], 1ull);
#endif
    if (lane == 0)
    {
        int total = 0;
        for (int p = 0; p < deg; p++)
        {
            w.port[p].first = total;
            total += w.port[p].an;
        }
        w.flags[1] = total;
    }
    group_sync(lanes);
    const int total = w.flags[1];
    const bool staged = total <= SW_STAGE;
    if (staged)
    {
        // the first SW_FRAMES frames copied whole into shared memory, 16 bytes a lane at a time (a
        // port's frames of the slot lie together in its link's bucket)
        const int nfr = total < SW_FRAMES ? total : SW_FRAMES;
        for (int k = lane; k < nfr * (int)(sizeof(Frame) / 16); k += lanes)
        {
            const int j = k / (int)(sizeof(Frame) / 16), word = k % (int)(sizeof(Frame) / 16);
            int p = 0;
            while (j >= w.port[p].first + w.port[p].an)
                p++;
            const Frame *src = &s.msg[w.port[p].abase + (j - w.port[p].first)];
#ifdef __CUDA_ARCH__
            reinterpret_cast<uint4 *>(&w.fr[j])[word] = __ldcg(reinterpret_cast<const uint4 *>(src) + word);
#else
            if (word == 0)
                w.fr[j] = *src;
#endif
        }
        group_sync(lanes);
        for (int j = lane; j < total; j += lanes)
        {
            int p = 0;
            while (j >= w.port[p].first + w.port[p].an)
                p++;
            SArr &a = w.arr[j];
            const uint32_t frame = (uint32_t)(w.port[p].abase + (j - w.port[p].first));
            Pkt pk;
            if (j < nfr)
            {
                const Frame &f = w.fr[j];
                pk = f.p;
                a.ts = f.ts;
                a.acode = event_code(link_tx_ns(s, w.port[p].lin, pk.size) + w.port[p].lin.delay, pk.ord);
                a.frame = frame;
                a.flow = pk.flow;
                a.size = pk.size;
                a.kind = pk.kind;
                a.pre = 0;
                a.copy = (uint16_t)j;
            }
            else
                stage_arrival(s, a, frame, w.port[p].lin, pk);
            a.in = (uint8_t)p;
            int qi = PG;
            a.out = (int16_t)(pk.kind == K_PAUSE || pk.kind == K_RESUME ? -1 : s_route(s, si, wp, pk, &qi));
            a.q = (uint8_t)qi;
            if (a.out >= 0 && a.q != 0)
                sh_add(&w.port[p].abytes, (uint32_t)a.size);
            const int own = a.out >= 0 ? a.out : (a.kind == K_PAUSE || a.kind == K_RESUME ? p : -1);
            if (own >= 0)
                sh_add(&w.port[own].ocnt, 1);
        }
        group_sync(lanes);
    }
    SW_PHASE(1);
    SwEv e;
    e.s = &s;
    e.w = &wp;
    e.x = x;
    e.si = si;
    e.mmu = s.sw[x].mmu;
    e.pe = w.port;
    e.n_ev = e.n_arr = 0;
    // a safe slot: nothing paused, no headroom in use, and every port below the lowest PFC
    // threshold the slot can reach even if all its arrivals stay (lane 0 decides for all)
    if (lane == 0)
    {
        bool safe = staged && deg <= SAFE_PORTS && !s.serial_only;
        int64_t amax = (int64_t)e.mmu.shared_used;
        for (int p = 0; p < deg; p++)
        {
            amax += w.port[p].abytes;
            if (w.port[p].pt.mmu.hdrm || w.port[p].pt.mmu.paused)
                safe = false;
        }
        const int64_t room = (int64_t)(uint32_t)(wp.buffer_size - e.mmu.total_hdrm - e.mmu.total_rsrv) - amax;
        const int64_t th_min = room > 0 ? room >> s.sw[x].max_shift : -1;
        for (int p = 0; p < deg && safe; p++)
        {
            const int64_t su = (int64_t)w.port[p].pt.mmu.ing + w.port[p].abytes - MMU_RESERVE;
            if ((su > 0 ? su : 0) >= th_min)
                safe = false;
        }
        int at = 0;
        for (int p = 0; p < deg; p++)
        {
            w.port[p].obase = at;
            at += w.port[p].ocnt;
        }
        w.flags[2] = safe;
    }
    group_sync(lanes);
    const bool safe = w.flags[2] != 0;
    e.safe = safe;
    SW_PHASE(2);
#ifdef TR_PROFILE
    if (lane == 0)
        count(s, safe ? EV_PROF_SAFE : EV_PROF_SERIAL);
#endif
    if (safe)
    {
        // egress ports spread over the warps (a warp's lanes diverge: fewer ports each, less waiting)
        const int wl = lanes < 32 ? lanes : 32, nw = lanes < 32 ? 1 : lanes / 32;
        for (int o = lane / wl + nw * (lane % wl); o < deg; o += nw * wl)
            safe_egress(e, w, o, t1, total);
#if defined(TR_PROFILE) && defined(__CUDA_ARCH__)
        atomicMax(&s.ev[EV_PROF_LANE_EV_SLOT], e.n_ev);
#endif
    }
    else if (lane == 0)
        serial_events(e, w, deg, t1, staged);
    group_sync(lanes);
    SW_PHASE(3);
    bool act = false;
    for (int p = lane; p < deg; p += lanes)
    {
        SwPort &q = w.port[p];
        q.out.flush(s);
        q.pt.ob_last = q.out.last;
        s.port[si.pbase + p] = q.pt;
        if (q.nout)
            s.p_tc[si.pbase + p] = q.tc;
    }
    group_sync(lanes);
    for (int p = 0; p < deg; p++)
    {
        const SwPort &q = w.port[p];
        act |= q.nout > 0 || q.pt.q0_n > 0 || q.pt.q3_n > 0 || q.pt.tc_at >= 0;
    }
    if (e.n_ev)
    {
        count(s, EV_SWITCH_EVENTS, e.n_ev);
        count(s, EV_SWITCH_ARRIVALS, e.n_arr);
    }
    if (lane == 0)
    {
        if (safe)
        {
            // shared_used follows from the ingress counts (modulo 2^32, as the counter)
            uint32_t d = 0;
            for (int p = 0; p < deg; p++)
            {
                const uint32_t a = w.port[p].ing0 > MMU_RESERVE ? w.port[p].ing0 - MMU_RESERVE : 0;
                const uint32_t b = w.port[p].pt.mmu.ing > MMU_RESERVE ? w.port[p].pt.mmu.ing - MMU_RESERVE : 0;
                d += b - a;
            }
            e.mmu.shared_used += d;
        }
        s.sw[x].mmu = e.mmu;
    }
    group_sync(lanes);
    SW_PHASE(4);
    return act;
}

// ------------------------------------------------------------------ the slot's end
// After every entity ran slot t: the run ends when every flow is done or at the stop time; a slot
// in which nothing was sent or held goes on at the earliest host event or frame arrival; nothing
// left at all ends the run (quiescence). (reference: slot_end, src/rdma/rstep.cuh:3451-3577)
// (activity, next_wake and flows_done: the entities' sums of the slot, read by the caller)
TR_HD void slot_close(const RSim &s, int64_t t, unsigned activity, unsigned long long next_wake, unsigned flows_done)
{
    RCtl &c = *s.ctl;
    if (flows_done >= (unsigned)s.F || t + 1 >= s.max_slots)
        c.finished = 1;
    s.pend[t % s.pend_n] = 0;
    int64_t next = t + 1;
    if (activity == 0)
    {
        int64_t ws = next_wake != ~0ull ? (int64_t)(next_wake / (unsigned long long)s.D) : INT64_MAX;
        for (int i = 1; i < s.pend_n; i++)
            if (ld_flag(&s.pend[(t + i) % s.pend_n]))
            {
                ws = t + i < ws ? t + i : ws;
                break;
            }
        if (ws != INT64_MAX && ws > next)
            next = ws < s.max_slots ? ws : s.max_slots;
        if (ws == INT64_MAX)
            c.finished = 1;
    }
    c.slot = next;
    c.slots_run++;
}

} // namespace tr
