// twins-b200: the RDMA model's NIC rules (RdmaHw, RdmaEgressQueue, RdmaQueuePair of the HPCC fork
// of ns-3.17 that the reference's twins-rdma restates): frame sizes, the send window, the queue
// pairs' round robin, the receiver's go-back-N check and the sender's handling of an ACK or NACK
// with its congestion-control dispatch, a queue pair's start, its next data frame and the NIC's
// next send time. Host and device functions of a queue pair's state; the
// caller owns queues, links, timers and event order. Bit-exact with the reference's functions
// (src/rdma/rstep.cuh), which the oracle's known-answer vectors pin.
#pragma once
#include "tr_cc.cuh"

#include <climits>

namespace tr
{

struct NicParams
{
    uint32_t mtu;           // payload per packet
    uint32_t ack_interval;  // L2_ACK_INTERVAL
    uint32_t chunk;         // L2_CHUNK_SIZE
    int64_t nack_interval;  // ns
    uint32_t seq_extra;     // 4 with 64-bit sequence numbers (ns-3.36), else 0
    int int_size;           // INT header bytes (42 with HPCC), else 0
    int var_win;            // VAR_WIN: the window scales with the rate
    int ack_high_prio;      // ACKs in queue 0
    int cc;                 // 1 DCQCN, 3 HPCC, 8 DCTCP
    int fast_react;         // HPCC: react to every ACK
    int ns336;              // tx times of ns-3.36 (integer)
};

// header bytes of a data frame, a data frame of `payload` bytes, an ACK / NACK (padded to the 60
// bytes of a minimum Ethernet frame before the 14-byte header), a PFC frame (reference:
// src/rdma/rstep.cuh:856-863)
TR_HD uint32_t data_hdr(const NicParams &P) { return 48 + P.seq_extra + (uint32_t)P.int_size; }
TR_HD uint32_t data_size(const NicParams &P, uint32_t payload) { return payload + data_hdr(P); }
TR_HD uint32_t ack_size(const NicParams &P)
{
    const int base = 12 + (int)P.seq_extra + P.int_size, pad = 60 - 14 - 20 - base;
    return (uint32_t)((pad > 0 ? pad : 0) + base + 20 + 14);
}
constexpr uint32_t PFC_SIZE = 43;

// a sending queue pair as the NIC sees it
struct QpSend
{
    uint64_t size, snd_una;
    int64_t next_avail;
    uint32_t last_pkt;
    uint8_t done;
};

// a queue pair's two parts, as next_qindex reads them
struct QpView
{
    const QpRate &rate;
    const QpSend &send;
};

TR_HD uint64_t bytes_left(const QpRate &r, const QpSend &q) { return q.size >= r.snd_nxt ? q.size - r.snd_nxt : 0; }

// the window holds no more (RdmaQueuePair::IsWinBound): bytes in flight reach the window, scaled by
// rate / line rate with VAR_WIN (at least 1) (reference: src/rdma/rstep.cuh:1036-1053)
// (VAR_WIN: with n = win * rate (64 bits, wrapping as the reference's product) and m the line rate,
// inflight >= max(1, floor(n / m)) holds exactly when inflight >= 1 and n < (inflight + 1) m, a
// 128-bit product instead of a division routine)
TR_HD bool win_bound(const NicParams &P, const QpRate &r, const QpSend &q)
{
    if (r.win == 0)
        return false;
    const uint64_t inflight = r.snd_nxt - q.snd_una;
    if (!P.var_win)
        return inflight >= r.win;
    if (inflight == 0 || inflight == ~0ull)
        return inflight != 0;
    const uint64_t n = (uint64_t)r.win * r.rate, a = inflight + 1, m = r.max_rate;
#ifdef __CUDA_ARCH__
    const uint64_t hi = __umul64hi(a, m), lo = a * m;
#else
    const unsigned __int128 am = (unsigned __int128)a * m;
    const uint64_t hi = (uint64_t)(am >> 64), lo = (uint64_t)am;
#endif
    return hi > 0 || n < lo;
}

// RdmaEgressQueue::GetNextQindex over a NIC's queue pairs list[0 .. *n): -1 the ACK queue (not
// paused and not empty), else the first queue pair after the last served one (rr), round robin,
// that has data, room in its window and is due (next_avail <= now), or -1024 for none. Finished
// queue pairs (all acknowledged) met before the pick are removed from the list from the first of
// them on, keeping the order (*n shrinks; the pick's index follows). qp(f) gives queue pair f's
// QpView (reference: src/rdma/rstep.cuh:1108-1144)
template <class Qp>
TR_HD int next_qindex(const NicParams &P, uint32_t paused, int ackq_n, int *list, int *n, int rr, int64_t now, Qp qp)
{
    const int ackq = P.ack_high_prio ? 0 : 3;
    if (!(paused >> ackq & 1) && ackq_n > 0)
        return -1;
    const bool data_paused = paused >> 3 & 1;
    int pick = -1024, first_done = INT_MAX;
    const int count = *n;
    int at = count ? rr % count : 0;
    for (int k = 0; k < count; k++)
    {
        at = at + 1 == count ? 0 : at + 1;
        const QpRate &r = qp(list[at]).rate;
        const QpSend &q = qp(list[at]).send;
        if (!data_paused && bytes_left(r, q) > 0 && !win_bound(P, r, q))
        {
            if (q.next_avail > now)
                continue;
            pick = at;
            break;
        }
        if (q.snd_una >= q.size && at < first_done)
            first_done = at;
    }
    if (first_done < INT_MAX)
    {
        int keep = first_done;
        for (int i = first_done + 1; i < count; i++)
        {
            const QpSend &q = qp(list[i]).send;
            if (q.snd_una >= q.size)
                continue;
            if (i == pick)
                pick = keep;
            list[keep++] = list[i];
        }
        *n = keep;
    }
    return pick;
}

// a queue pair starts (RdmaHw::AddQueuePair): the NIC's line rate as rate, line rate and DCQCN
// target, the flow's window and base RTT, alpha 1 before a first CNP, HPCC's reference rate and
// utilisation, sending from now (reference: src/rdma/rstep.cuh:1548-1587)
TR_HD void qp_start(const NicParams &P, QpRate &r, QpSend &q, uint64_t size, uint64_t nic_bps, uint32_t win, uint64_t base_rtt, int64_t now)
{
    r = QpRate{};
    q = QpSend{};
    q.size = size;
    r.rate = r.max_rate = r.target = nic_bps;
    r.win = win;
    r.base_rtt = base_rtt;
    r.alpha = 1;
    r.first_cnp = 1;
    if (P.cc == 3)
    {
        r.cur_rate = nic_bps;
        r.u = 1;
    }
    q.next_avail = now;
}

// the next data frame of a queue pair (RdmaHw::GetNxtPacket, PktSent, UpdateNextAvail): its
// sequence number (*seq) and size; snd_nxt moves past its payload, and the next send waits its tx
// time at the rate (or the line rate without RATE_BOUND) (reference: src/rdma/rstep.cuh:1162-1181)
TR_HD uint32_t next_data(const NicParams &P, QpRate &r, QpSend &q, int64_t now, bool rate_bound, uint32_t *seq, TxMemo *m = nullptr)
{
    const uint64_t left = bytes_left(r, q);
    const uint32_t payload = left < P.mtu ? (uint32_t)left : P.mtu;
    const uint32_t size = data_size(P, payload) & 0xFFFF;
    *seq = (uint32_t)r.snd_nxt;
    r.snd_nxt += payload;
    q.last_pkt = size;
    q.next_avail = now + tx_time_memo(m, P.ns336 != 0, rate_bound ? r.rate : r.max_rate, size);
    return size;
}

// no queue pair can send now: the earliest next_avail among list[0 .. n) (those with data left;
// all of them under ns-3.36), when later than now, is the NIC's next send; else -1 (reference:
// src/rdma/rstep.cuh:1182-1192)
template <class Qp>
TR_HD int64_t next_send_at(const NicParams &P, const int *list, int n, int64_t now, Qp qp)
{
    int64_t t = INT64_MAX;
    for (int i = 0; i < n; i++)
    {
        const QpView v = qp(list[i]);
        if (bytes_left(v.rate, v.send) == 0 && !P.ns336)
            continue;
        t = v.send.next_avail < t ? v.send.next_avail : t;
    }
    return t < INT64_MAX && t > now ? t : -1;
}

// the receiving queue pair's state (expected byte, last NACKed byte, NACK timer)
struct RxQp
{
    uint32_t expected, last_nack;
    int64_t nack_timer;
};

enum : int
{
    RX_ACK = 1,  // in order, and an ACK is due (every byte past the ACK interval, or a chunk's end)
    RX_NACK = 2, // a gap, and a NACK is due (a new gap, or the NACK interval passed)
    RX_OLD = 3,  // a duplicate
    RX_QUIET = 4, // a gap already NACKed within the interval
    RX_HELD = 5  // in order, no ACK yet
};

// RdmaHw::ReceiverCheckSeq for a data frame (seq, payload) at now: the verdict; an ACK or a NACK
// carries the expected byte (reference: src/rdma/rstep.cuh:1498-1524)
TR_HD int rx_check(const NicParams &P, RxQp &r, uint32_t seq, uint32_t payload, int64_t now)
{
    const uint32_t expected = r.expected;
    if (seq == expected)
    {
        r.expected = expected + payload;
        if (r.expected >= P.ack_interval)
            return RX_ACK;
        if (P.chunk && r.expected % P.chunk == 0)
            return RX_ACK;
        return RX_HELD;
    }
    if (seq > expected)
    {
        if (now >= r.nack_timer || r.last_nack != expected)
        {
            r.nack_timer = now + P.nack_interval;
            r.last_nack = expected;
            return RX_NACK;
        }
        return RX_QUIET;
    }
    return RX_OLD;
}

// what handling an ACK did (bits)
enum : unsigned
{
    ACK_COMPLETED = 1, // the queue pair completed (QpComplete): its DCQCN timers stop
    ACK_RATE_SET = 2,  // HPCC set the rate (the next send moved with it)
    ACK_CNP = 4        // DCQCN took a CNP (its returned timers are in the bits << 4)
};

// RdmaHw::ReceiveAck for an ACK (nack false) or NACK of byte seq, with the CNP flag: snd_una
// advances; every byte acknowledged completes the queue pair; a NACK goes back to snd_una; then
// the congestion control: DCQCN's CNP, HPCC's update (fast react on ACKs of old data), DCTCP's ACK
// (reference: src/rdma/rstep.cuh:1438-1485). A queue pair already done is the caller's to skip.
TR_HD unsigned ack_received(const NicParams &P, const CcParams &C, QpRate &r, QpSend &q, uint32_t seq, bool nack, bool cnp,
                            const uint64_t *hops, int nhop, const double *pre_u = nullptr, uint64_t pre_dt = 0, TxMemo *m = nullptr)
{
    unsigned out = 0;
    if (seq > q.snd_una)
        q.snd_una = seq;
    if (q.snd_una >= q.size)
    {
        q.done = 1;
        out |= ACK_COMPLETED;
    }
    if (nack)
        r.snd_nxt = q.snd_una;
    if (cnp && P.cc == 1 && !q.done)
        out |= ACK_CNP | dcqcn_cnp(r, C) << 4;
    if (P.cc == 3 && (seq > r.last_update_seq || P.fast_react))
    {
        const uint64_t old = r.rate;
        if (hpcc_ack(r, C, hops, nhop, !(seq > r.last_update_seq), pre_u, pre_dt))
        {
            q.next_avail = paced_after_change(q.next_avail, P.ns336 != 0, old, r.rate, q.last_pkt, m);
            out |= ACK_RATE_SET;
        }
    }
    if (P.cc == 8 && !q.done)
        dctcp_ack(r, C, seq, cnp);
    return out;
}

} // namespace tr
