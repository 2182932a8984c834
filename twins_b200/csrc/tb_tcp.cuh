// twins-b200: the host's TCP (ns-3 TcpSocketBase with NewReno / DCTCP / Cubic, TcpTxBuffer
// without SACK, TcpRxBuffer, delayed ACKs, FIN) as device functions over one host's records.
// Reference: src/step.cuh:319-2236 (function-by-function citations below).
#pragma once
#include "tb_egress.cuh"

namespace tb
{

constexpr int DUE_CAP = 64;

struct Due
{
    int64_t at;
    int flow;
    int kind; // 0 RTO, 1 delayed ACK, 2 SYN / deferred SendPendingData, 3 SYN-ACK retx, 4 LastAck, 5 FIN+ACK retx
};

// one host's context for one slot
struct HostCtx
{
    const Sim *s;
    const WorldDesc *wd;
    int h;       // global host id
    bool dctcp, cubic;
    Egress nic;
    Chain ech;   // the chain of the event being handled
    Due due[DUE_CAP];
    int nd, di;  // timers collected / handled
    int64_t slot_end;
    unsigned retx, rtos, ovf, done;
    unsigned long long pkts, snd_pkts;
};

// a timer set during the slot and due within it (due_insert, step.cuh:342-360)
TB_D void due_insert(HostCtx &c, int64_t at, int f, int kind)
{
    if (at >= c.slot_end)
        return;
    if (c.nd >= DUE_CAP)
    {
        c.ovf++;
        return;
    }
    int j = c.nd;
    while (j > c.di && c.due[j - 1].at > at)
    {
        c.due[j] = c.due[j - 1];
        j--;
    }
    c.due[j] = {at, f, kind};
    c.nd++;
}

// a frame into the host's egress (emit, step.cuh:368-384)
TB_D void emit(HostCtx &c, int f, uint8_t flags, uint32_t seq, uint32_t ack, uint16_t len, bool to_sender, int64_t now,
               uint32_t hash, int dst_local)
{
    Frame fr;
    fr.ts = now;
    fr.flow = (uint32_t)f;
    fr.sa = (flags & F_DATA) ? seq : ack;
    fr.len = len;
    fr.dst = (uint16_t)dst_local;
    fr.flags = flags | (c.dctcp ? F_ECT : 0);
    fr.to_sender = to_sender ? 1 : 0;
    fr.up = (uint16_t)(hash % (uint32_t)c.wd->ecmp_n);
    fr.ch = c.ech;
    c.nic.enqueue(fr, now);
}
TB_D void emit_snd(HostCtx &c, int f, const SndRec &S, uint8_t flags, uint32_t seq, uint32_t ack, uint16_t len, int64_t now)
{
    emit(c, f, flags, seq, ack, len, false, now, S.hash_data, S.dst_local);
}
TB_D void emit_rcv(HostCtx &c, int f, const RcvRec &R, uint8_t flags, uint32_t ack, uint16_t len, int64_t now)
{
    emit(c, f, flags, 0, ack, len, true, now, R.hash_ack, R.src_local);
}

// SendEmptyPacket(ACK) at the receiver (send_ack, step.cuh:387-407)
TB_D void send_ack(HostCtx &c, int f, RcvRec &R, uint32_t ack, bool force_ece, bool no_ece, int64_t now)
{
    bool ece = false;
    if (force_ece)
        ece = true;
    else if (!no_ece && (R.ecn_r == E_CE_RCVD || R.ecn_r == E_SENDING_ECE))
    {
        ece = true;
        R.ecn_r = E_SENDING_ECE;
    }
    R.delack_at = -1;
    R.delack_count = 0;
    emit_rcv(c, f, R, F_ACK | (ece ? F_ECE : 0), ack, CTRL_LEN, now);
}

// ------------------------------------------------------------------ the sent list (TcpTxBuffer)
// A ring of items (start sequence number, TcpTxItem flags) at it_off; an item ends where the
// next starts, the last at `high`; byte counters sack_b / lost_b / rtx_b as ns-3 keeps them.
struct Tx
{
    SndRec &S;
    uint32_t *st;
    uint8_t *fl;
    uint32_t cap;
    TB_D Tx(const Sim &s, SndRec &S_) : S(S_)
    {
        st = s.it_start + S.it_off;
        fl = s.it_fl + S.it_off;
        cap = S.it_cap;
    }
    TB_D uint32_t at(uint32_t i) const
    {
        uint32_t x = S.it_head + i;
        return x >= cap ? x - cap : x;
    }
    TB_D uint32_t beg(uint32_t i) const { return st[at(i)]; }
    TB_D uint32_t end(uint32_t i) const { return i + 1 < S.it_n ? st[at(i + 1)] : S.high; }
    TB_D uint8_t flags(uint32_t i) const { return fl[at(i)]; }
};

TB_D bool it_cand(uint8_t fl) { return (fl & (IT_LOST | IT_RETX | IT_SACKED)) == IT_LOST; }

// new flags for item i, keeping the byte counters, the sacked count and the NextSeg cursor
// (it_set, step.cuh:453-483)
TB_D void it_set(Tx &t, uint32_t i, uint8_t nf)
{
    SndRec &S = t.S;
    uint32_t k = t.at(i);
    uint8_t of = t.fl[k];
    if (of == nf)
        return;
    uint32_t len = t.end(i) - t.st[k];
    uint8_t d = of ^ nf;
    if (d & IT_SACKED)
    {
        S.sack_b += (nf & IT_SACKED) ? len : 0u - len;
        S.sacked_n += (nf & IT_SACKED) ? 1u : 0u - 1u;
    }
    if (d & IT_LOST)
        S.lost_b += (nf & IT_LOST) ? len : 0u - len;
    if (d & IT_RETX)
        S.rtx_b += (nf & IT_RETX) ? len : 0u - len;
    if (it_cand(of) != it_cand(nf))
    {
        if (it_cand(nf))
        {
            S.cand_n++;
            if (i < S.cand)
                S.cand = i;
        }
        else
            S.cand_n--;
    }
    t.fl[k] = nf;
}

// insert an item at index i (a split, or new data at the end) (it_insert, step.cuh:486-512)
TB_D bool it_insert(Tx &t, uint32_t i, uint32_t start, uint8_t fl, unsigned &ovf)
{
    SndRec &S = t.S;
    if (S.it_n >= t.cap)
    {
        ovf++;
        return false;
    }
    for (uint32_t j = S.it_n; j > i; j--)
    {
        uint32_t a = t.at(j), b = t.at(j - 1);
        t.st[a] = t.st[b];
        t.fl[a] = t.fl[b];
    }
    uint32_t k = t.at(i);
    t.st[k] = start;
    t.fl[k] = fl;
    S.it_n++;
    if (S.cand >= i && S.cand > 0)
        S.cand++;
    if (it_cand(fl))
    {
        S.cand_n++;
        if (i < S.cand)
            S.cand = i;
    }
    return true;
}

// remove item i's start, merging it into item i - 1 (it_remove_start, step.cuh:515-529)
TB_D void it_remove_start(Tx &t, uint32_t i)
{
    SndRec &S = t.S;
    for (uint32_t j = i; j + 1 < S.it_n; j++)
    {
        uint32_t a = t.at(j), b = t.at(j + 1);
        t.st[a] = t.st[b];
        t.fl[a] = t.fl[b];
    }
    S.it_n--;
    if (S.cand > i)
        S.cand--;
}

TB_D uint32_t it_lower(const Tx &t, uint32_t seq)
{
    uint32_t lo = 0, hi = t.S.it_n;
    while (lo < hi)
    {
        uint32_t m = (lo + hi) / 2;
        if (t.beg(m) < seq)
            lo = m + 1;
        else
            hi = m;
    }
    return lo;
}

TB_D uint32_t tb_sent(const SndRec &S) { return S.it_n ? S.high - S.una : 0u; }
// BytesInFlight = sent - (sacked + lost) + retransmitted, unsigned as in ns-3
TB_D uint32_t inflight(const SndRec &S) { return tb_sent(S) - (S.sack_b + S.lost_b) + S.rtx_b; }

// AddRenoSack (step.cuh:649-662)
TB_D void add_reno_sack(Tx &t)
{
    SndRec &S = t.S;
    uint32_t i = 1 + S.sacked_n;
    while (i < S.it_n && (t.flags(i) & IT_SACKED))
        i++;
    if (i < S.it_n)
    {
        it_set(t, i, t.flags(i) | IT_SACKED);
        S.sack_seen = 1;
        S.hisack = t.beg(i);
    }
}
// MarkHeadAsLost (step.cuh:672-677)
TB_D void mark_head_lost(Tx &t)
{
    if (t.S.it_n == 0)
        return;
    it_set(t, 0, (uint8_t)((t.flags(0) & ~(IT_SACKED | IT_RETX)) | IT_LOST));
}
// ResetRenoSack + SetSentListLost (step.cuh:687-712)
TB_D void all_lost(Tx &t)
{
    SndRec &S = t.S;
    for (uint32_t i = 0; i < S.it_n; i++)
        t.fl[t.at(i)] = IT_LOST;
    S.sack_b = 0;
    S.sacked_n = 0;
    S.rtx_b = 0;
    S.lost_b = tb_sent(S);
    S.cand_n = S.it_n;
    S.cand = 0;
    S.sack_seen = 0;
    S.hisack = 0;
}
// DiscardUpTo(ack): the bytes of the items removed whole (step.cuh:716-780)
TB_D uint32_t discard(Tx &t, uint32_t ack)
{
    SndRec &S = t.S;
    uint32_t delivered = 0, removed = 0;
    while (S.it_n > 0)
    {
        uint32_t k = t.at(0), b = t.st[k], e = t.end(0);
        if (ack >= e)
        {
            if (t.fl[k])
                it_set(t, 0, 0);
            S.it_head = t.at(1);
            S.it_n--;
            removed++;
            delivered += e - b;
        }
        else
        {
            if (ack > b)
            {
                uint8_t fl = t.fl[k];
                uint32_t off = ack - b;
                if (fl & IT_SACKED)
                    S.sack_b -= off;
                if (fl & IT_LOST)
                    S.lost_b -= off;
                if (fl & IT_RETX)
                    S.rtx_b -= off;
                t.st[k] = ack;
            }
            break;
        }
    }
    if (removed)
        S.cand = S.cand > removed ? S.cand - removed : 0;
    S.una = ack;
    if (S.it_n > 0 && (t.flags(0) & IT_SACKED))
    {
        it_set(t, 0, (uint8_t)(t.flags(0) & ~IT_SACKED));
        add_reno_sack(t);
        mark_head_lost(t);
    }
    if (S.hisack <= ack)
    {
        S.sack_seen = 0;
        S.hisack = 0;
    }
    return delivered;
}
// NextSeg without SACK: the first lost item neither retransmitted nor sacked, below the highest
// sack; else new data (step.cuh:784-834)
TB_D bool next_seg(Tx &t, uint32_t *seq)
{
    SndRec &S = t.S;
    if (S.cand_n > 0)
    {
        for (uint32_t i = S.cand; i < S.it_n; i++)
        {
            if (!it_cand(t.flags(i)))
                continue;
            S.cand = i;
            uint32_t b = t.beg(i);
            if (!S.sack_seen || b < S.hisack)
            {
                *seq = b;
                return true;
            }
            break;
        }
    }
    if (S.tail > S.high)
    {
        *seq = S.high;
        return true;
    }
    return false;
}
// IsLost(SND.UNA) (step.cuh:838-846)
TB_D bool head_lost(const Tx &t)
{
    const SndRec &S = t.S;
    if (!S.sack_seen || S.una >= S.hisack || S.it_n == 0)
        return false;
    return t.flags(0) & IT_LOST;
}
// IsRetransmittedDataAcked(x) (step.cuh:849-869)
TB_D bool retx_ends_at(const Tx &t, uint32_t x)
{
    const SndRec &S = t.S;
    if (S.it_n == 0 || x <= S.una || x > S.high)
        return false;
    uint32_t i = it_lower(t, x) - 1;
    if (t.end(i) != x)
        return false;
    uint8_t fl = t.flags(i);
    return !(fl & IT_SACKED) && (fl & IT_RETX);
}
// GetTransmittedSegment (step.cuh:874-916)
TB_D uint32_t retransmit(Tx &t, uint32_t i, uint32_t num, unsigned &ovf)
{
    SndRec &S = t.S;
    uint32_t len = t.end(i) - t.beg(i);
    uint32_t sz = num;
    if (i + 1 < S.it_n)
    {
        uint8_t a = t.flags(i), b = t.flags(i + 1);
        uint32_t nlen = t.end(i + 1) - t.beg(i + 1);
        if (!(b & IT_SACKED) && (a & IT_LOST) == (b & IT_LOST))
            sz = sz < len + nlen ? sz : len + nlen;
        else
            sz = sz < len ? sz : len;
    }
    else
        sz = sz < len ? sz : len;
    if (sz > len)
    {
        uint8_t a = t.flags(i), b = t.flags(i + 1);
        if ((a ^ b) & IT_RETX)
        {
            if (a & IT_RETX)
                it_set(t, i, a &= (uint8_t)~IT_RETX);
            else
                it_set(t, i + 1, b &= (uint8_t)~IT_RETX);
        }
        if (it_cand(b))
            S.cand_n--;
        it_remove_start(t, i + 1);
        len = t.end(i) - t.beg(i);
    }
    if (sz < len)
        it_insert(t, i + 1, t.beg(i) + sz, t.flags(i), ovf);
    uint8_t fl = t.flags(i);
    if (!(fl & IT_RETX))
        it_set(t, i, fl | IT_RETX);
    return sz;
}
// CopyFromSequence (step.cuh:920-975)
TB_D uint32_t tb_copy(Tx &t, uint32_t num, uint32_t seq, bool *retx, unsigned &ovf)
{
    SndRec &S = t.S;
    for (;;)
    {
        uint32_t avail = S.tail > seq ? S.tail - seq : 0;
        uint32_t sz = num < avail ? num : avail;
        if (sz == 0)
            return 0;
        if (S.high >= seq + sz)
        {
            uint32_t i = it_lower(t, seq);
            if (i >= S.it_n || t.beg(i) != seq)
            {
                ovf++; // (not an item start: cannot happen)
                return 0;
            }
            *retx = true;
            return retransmit(t, i, sz, ovf);
        }
        if (S.high <= seq)
        {
            if (!it_insert(t, S.it_n, seq, 0, ovf))
                return 0;
            S.high = seq + sz;
            *retx = false;
            return sz;
        }
        num = S.high - seq;
    }
}

// ------------------------------------------------------------------ RTT history and estimator
// m_history: first transmissions in order, a ring sharing the sent list's capacity; bit 31 of
// the count marks a retransmitted entry (step.cuh:977-1126)
TB_D uint32_t h_at(const SndRec &S, uint32_t j)
{
    uint32_t x = S.h_head + j;
    return x >= S.it_cap ? x - S.it_cap : x;
}
TB_D void rtt_history(const Sim &s, SndRec &S, uint32_t seq, uint32_t sz, bool retx, int64_t now, unsigned &ovf)
{
    uint32_t *hs = s.h_seq + S.it_off, *hc = s.h_cnt + S.it_off;
    if (!retx)
    {
        if (S.h_n >= S.it_cap)
        {
            ovf++;
            return;
        }
        uint32_t k = h_at(S, S.h_n);
        hs[k] = seq;
        hc[k] = sz;
        s.h_t[S.it_off + k] = now;
        S.h_n++;
        return;
    }
    for (uint32_t j = 0; j < S.h_n; j++)
    {
        uint32_t k = h_at(S, j);
        uint32_t cnt = hc[k] & 0x7FFFFFFFu;
        if (seq >= hs[k] && seq < hs[k] + cnt)
        {
            hc[k] = 0x80000000u | (seq + sz - hs[k]);
            return;
        }
    }
}
// RttMeanDeviation::Measurement and the RTO (step.cuh:1066-1086)
TB_D void rtt_sample(SndRec &S, int64_t m)
{
    int64_t est = S.srtt, var = S.rttvar;
    if (est < 0)
    {
        est = m;
        var = m / 2;
    }
    else
    {
        int64_t delta = m - est;
        est = ((est << 3) + delta) >> 3;
        if (delta < 0)
            delta = -delta;
        var = ((var << 2) + delta - var) >> 2;
    }
    S.srtt = est;
    S.rttvar = var;
    int64_t v = 4 * var;
    int64_t rto = est + (v > GRAN_PS ? v : GRAN_PS);
    S.rto = rto > MIN_RTO_PS ? rto : MIN_RTO_PS;
}
// EstimateRtt (step.cuh:1088-1126)
TB_D void rtt_ack(const Sim &s, SndRec &S, uint32_t ack, int64_t now)
{
    if (S.h_n == 0)
        return;
    uint32_t *hs = s.h_seq + S.it_off, *hc = s.h_cnt + S.it_off;
    uint32_t k = h_at(S, 0);
    if (!(hc[k] & 0x80000000u) && ack >= hs[k] + hc[k])
        rtt_sample(S, now - s.h_t[S.it_off + k]);
    while (S.h_n > 0)
    {
        k = h_at(S, 0);
        if (hs[k] + (hc[k] & 0x7FFFFFFFu) > ack)
            break;
        S.h_head = h_at(S, 1);
        S.h_n--;
    }
}

// ------------------------------------------------------------------ TcpCubic (step.cuh:1201-1345)
constexpr double CUB_C = 0.4, CUB_BETA = 0.7;
constexpr int64_t CUB_ACK_DELTA = 2000000000, CUB_DELAY_MIN = 4000000000, CUB_DELAY_MAX = 1000000000000,
                  CUB_DELTA = 10000000000;

// double -> uint32_t as GCC/x86-64 converts it (cvttsd2si to 64 bits, the low half; out of
// range: the "integer indefinite" 2^63)
TB_D uint32_t cub_u32(double d)
{
    int64_t v = (d >= -9223372036854775808.0 && d < 9223372036854775808.0) ? (int64_t)d : INT64_MIN;
    return (uint32_t)(uint64_t)v;
}
TB_D void cub_hystart_reset(SndRec &S, int64_t now)
{
    S.cub_roundstart = S.cub_lastack = now;
    S.cub_endseq = S.st == S_EST ? S.high + 1 : 0;
    S.cub_currrtt = INT64_MIN;
    S.cub_samples = 0;
}
TB_D double cub_root(const Sim &s, uint32_t n)
{
    // pow(n / 0.4, 1/3) as the host's libm computes it (a table), else the device pow
    if (n < (uint32_t)s.cub_k_n)
        return s.cub_k_tab[n];
    return tb_pow((double)n / CUB_C, 1 / 3.);
}
TB_D uint32_t cub_update(const Sim &s, SndRec &S, uint32_t segs, int64_t now)
{
    uint32_t seg_cwnd = S.cwnd / MSS;
    S.cub_ackcnt += segs;
    if (S.cub_epoch == INT64_MIN)
    {
        S.cub_epoch = now;
        S.cub_ackcnt = segs;
        S.cub_tcpcwnd = seg_cwnd;
        if (S.cub_lastmax <= seg_cwnd)
        {
            S.cub_k = 0.0;
            S.cub_origin = seg_cwnd;
        }
        else
        {
            S.cub_k = cub_root(s, S.cub_lastmax - seg_cwnd);
            S.cub_origin = S.cub_lastmax;
        }
    }
    int64_t t = (int64_t)((uint64_t)now + (uint64_t)S.cub_delaymin - (uint64_t)S.cub_epoch);
    double ts = get_seconds(t), kk = S.cub_k;
    double offs = ts < kk ? kk - ts : ts - kk;
    uint32_t delta = cub_u32(CUB_C * tb_pow(offs, 3));
    uint32_t target = ts < kk ? S.cub_origin - delta : S.cub_origin + delta;
    uint32_t cnt = target > seg_cwnd ? seg_cwnd / (target - seg_cwnd) : 100 * seg_cwnd;
    if (S.cub_lastmax == 0 && cnt > 20)
        cnt = 20;
    uint32_t scale = cub_u32(8 * (1024 + CUB_BETA * 1024) / 3 / (1024 - CUB_BETA * 1024));
    delta = (seg_cwnd * scale) >> 3;
    while (S.cub_ackcnt > delta)
    {
        S.cub_ackcnt -= delta;
        S.cub_tcpcwnd++;
    }
    if (S.cub_tcpcwnd > seg_cwnd)
    {
        uint32_t max_cnt = seg_cwnd / (S.cub_tcpcwnd - seg_cwnd);
        if (cnt > max_cnt)
            cnt = max_cnt;
    }
    return cnt > 2 ? cnt : 2;
}
TB_D void cub_pkts_acked(SndRec &S, int64_t now)
{
    if (S.cub_epoch != INT64_MIN && now - S.cub_epoch < CUB_DELTA)
        return;
    int64_t rtt = S.srtt;
    if (S.cub_delaymin == INT64_MIN || S.cub_delaymin > rtt)
        S.cub_delaymin = rtt;
    uint32_t cwnd = S.cwnd;
    if (!(cwnd <= S.ssthresh && cwnd >= 16 * MSS) || S.cub_found)
        return;
    if (now - S.cub_lastack <= CUB_ACK_DELTA)
    {
        S.cub_lastack = now;
        if (now - S.cub_roundstart > S.cub_delaymin)
            S.cub_found = 1;
    }
    if (S.cub_samples < 8)
    {
        if (S.cub_currrtt == INT64_MIN || S.cub_currrtt > rtt)
            S.cub_currrtt = rtt;
        S.cub_samples++;
    }
    else
    {
        int64_t dm = S.cub_delaymin;
        int64_t thresh = dm > CUB_DELAY_MAX ? CUB_DELAY_MAX : (dm < CUB_DELAY_MIN ? CUB_DELAY_MIN : dm);
        if (S.cub_currrtt > dm + thresh)
            S.cub_found = 1;
    }
    if (S.cub_found)
        S.ssthresh = cwnd;
}
TB_D void cub_increase(const Sim &s, SndRec &S, uint32_t segs, uint32_t ack, int64_t now)
{
    if (!S.cwnd_limited)
        return;
    if (S.cwnd < S.ssthresh)
    {
        if (ack + 1 > S.cub_endseq)
            cub_hystart_reset(S, now);
        S.cwnd += segs * MSS;
        segs = 0;
    }
    if (S.cwnd >= S.ssthresh && segs > 0)
    {
        S.cub_cnt += segs;
        uint32_t cnt = cub_update(s, S, segs, now);
        if (S.cub_cnt >= cnt)
        {
            S.cwnd += MSS;
            S.cub_cnt -= cnt;
        }
    }
}
TB_D uint32_t cub_ssthresh(SndRec &S)
{
    uint32_t seg_cwnd = S.cwnd / MSS;
    if (seg_cwnd < S.cub_lastmax)
        S.cub_lastmax = cub_u32((seg_cwnd * (1 + CUB_BETA)) / 2);
    else
        S.cub_lastmax = seg_cwnd;
    S.cub_epoch = INT64_MIN;
    uint32_t th = cub_u32(seg_cwnd * CUB_BETA);
    return (th > 2 ? th : 2) * MSS;
}
TB_D void cub_loss(SndRec &S, int64_t now)
{
    S.cub_origin = 0;
    S.cub_k = 0;
    S.cub_ackcnt = 0;
    S.cub_tcpcwnd = 0;
    S.cub_delaymin = INT64_MIN;
    S.cub_found = 0;
    cub_hystart_reset(S, now);
}

// ------------------------------------------------------------------ congestion control
// GetSsThresh (step.cuh:1055-1063)
TB_D uint32_t ssthresh_for(HostCtx &c, SndRec &S, uint32_t bif)
{
    if (c.cubic)
        return cub_ssthresh(S);
    if (c.dctcp)
        return (uint32_t)((1.0 - S.alpha / 2.0) * S.cwnd);
    uint32_t half = bif / 2;
    return half > 2 * MSS ? half : 2 * MSS;
}
// PktsAcked (step.cuh:1348-1381)
TB_D void pkts_acked(HostCtx &c, SndRec &S, uint32_t segs, uint32_t ack, int64_t now)
{
    if (c.cubic)
    {
        cub_pkts_acked(S, now);
        return;
    }
    if (!c.dctcp)
        return;
    S.acked_total += segs * MSS;
    if (S.ecn_s == E_ECE_RCVD)
        S.acked_ecn += segs * MSS;
    if (!S.next_seq_flag)
    {
        S.next_seq = S.nxt;
        S.next_seq_flag = 1;
    }
    if (ack >= S.next_seq)
    {
        double m = S.acked_total > 0 ? (double)S.acked_ecn / S.acked_total : 0.0;
        S.alpha = tb_fma(1.0 - DCTCP_G, S.alpha, DCTCP_G * m); // as ns-3's -march=native build fuses it
        S.next_seq = S.nxt;
        S.acked_total = 0;
        S.acked_ecn = 0;
    }
}
// IncreaseWindow: TcpLinuxReno (DCTCP), TcpNewReno, TcpCubic (step.cuh:1383-1440)
TB_D void increase_window(HostCtx &c, SndRec &S, uint32_t segs, uint32_t ack, int64_t now)
{
    if (c.cubic)
    {
        cub_increase(*c.s, S, segs, ack, now);
        return;
    }
    uint32_t cwnd = S.cwnd, ssth = S.ssthresh;
    if (c.dctcp)
    {
        if (cwnd < ssth)
        {
            if (segs >= 1)
            {
                uint64_t n = (uint64_t)cwnd + (uint64_t)segs * MSS;
                S.cwnd = (uint32_t)(n < ssth ? n : ssth);
            }
        }
        else
        {
            uint32_t w = cwnd / MSS;
            if (w == 0)
                w = 1;
            uint32_t cnt = S.cwnd_cnt;
            if (cnt >= w)
            {
                cnt = 0;
                cwnd += MSS;
            }
            cnt += segs;
            if (cnt >= w)
            {
                uint32_t delta = cnt / w;
                cnt -= delta * w;
                cwnd += delta * MSS;
            }
            S.cwnd = cwnd;
            S.cwnd_cnt = cnt;
        }
        return;
    }
    if (cwnd < ssth && segs >= 1)
    {
        cwnd += MSS;
        segs -= 1;
    }
    if (cwnd >= ssth && segs > 0)
    {
        double adder = (double)MSS * MSS / cwnd;
        if (adder < 1.0)
            adder = 1.0;
        cwnd += (uint32_t)adder;
    }
    S.cwnd = cwnd;
}

// ------------------------------------------------------------------ sending
// SendDataPacket (step.cuh:1129-1172)
TB_D uint32_t send_segment(HostCtx &c, int f, SndRec &S, uint32_t seq, uint32_t max_size, int64_t now)
{
    Tx t(*c.s, S);
    bool retx = false;
    uint32_t len = tb_copy(t, max_size, seq, &retx, c.ovf);
    if (len == 0)
        return 0;
    uint8_t flags = F_DATA;
    if (!retx && S.ecn_s == E_ECE_RCVD && S.ecn_echo_seq > S.ecn_cwr_seq)
    {
        S.ecn_s = E_CWR_SENT;
        S.ecn_cwr_seq = seq;
        flags |= F_CWR;
    }
    if ((S.fin & FIN_CLOSE) && seq + len == S.tail)
    {
        flags |= F_FIN;
        S.fin |= FIN_SENT;
    }
    emit_snd(c, f, S, flags, seq, 0, (uint16_t)(len + HDR_BYTES), now);
    if (retx)
        c.retx++;
    if (S.rto_at < 0)
    {
        S.rto_at = now + S.rto;
        chain_child(S.rchain, c.ech, code_lead(S.rto));
    }
    S.cwnd_limited = S.cwnd < inflight(S) + MSS;
    rtt_history(*c.s, S, seq, len, retx, now, c.ovf);
    if (seq + len > S.high)
        S.high = seq + len;
    return len;
}
// SendPendingData (step.cuh:1175-1199)
TB_D void send_pending(HostCtx &c, int f, SndRec &S, int64_t now)
{
    if (S.st != S_EST)
        return;
    for (int guard = 0; guard < 4096; guard++)
    {
        if (S.cong == C_OPEN && (S.fin & (FIN_SENT | FIN_ACKED)) == FIN_SENT)
            return;
        uint32_t pipe = inflight(S);
        uint32_t avail = S.cwnd > pipe ? S.cwnd - pipe : 0;
        if (avail == 0)
            return;
        uint32_t seq;
        Tx t(*c.s, S);
        if (!next_seg(t, &seq))
            return;
        uint32_t remaining = S.tail - seq;
        if (avail < MSS && remaining > avail)
            return;
        S.nxt = seq;
        uint32_t len = send_segment(c, f, S, seq, avail < MSS ? avail : MSS, now);
        if (len == 0)
            return;
        S.nxt = seq + len;
    }
}
// DoRetransmit (step.cuh:1202-1212)
TB_D void do_retransmit(HostCtx &c, int f, SndRec &S, int64_t now)
{
    uint32_t seq;
    Tx t(*c.s, S);
    if (!next_seg(t, &seq))
        seq = S.una;
    if (S.una >= S.tail)
        return;
    S.nxt = seq;
    send_segment(c, f, S, seq, MSS, now);
}
// NewAck: the RTO from the estimator (clearing backoff); no timer once the buffer is empty
// outside FIN_WAIT_1 (step.cuh:1445-1464)
TB_D void new_ack(HostCtx &c, SndRec &S, uint32_t ack, bool reset_rto, int64_t now)
{
    if (reset_rto)
    {
        int64_t est = S.srtt >= 0 ? S.srtt : INIT_RTT_PS, v = 4 * S.rttvar;
        int64_t rto = est + (v > GRAN_PS ? v : GRAN_PS);
        S.rto = rto > MIN_RTO_PS ? rto : MIN_RTO_PS;
        S.rto_at = now + S.rto;
        chain_child(S.rchain, c.ech, code_lead(S.rto));
    }
    if (ack >= S.tail && !(S.fin & FIN_SENT))
        S.rto_at = -1;
    if (ack > S.nxt)
        S.nxt = ack;
}
// EnterRecovery (step.cuh:1467-1481)
TB_D void enter_recovery(HostCtx &c, int f, SndRec &S, int64_t now)
{
    Tx t(*c.s, S);
    add_reno_sack(t);
    mark_head_lost(t);
    S.recover = S.high;
    S.recover_active = 1;
    S.cong = C_RECOVERY;
    S.ssthresh = ssthresh_for(c, S, inflight(S) + MSS);
    S.cwnd = S.ssthresh;
    send_segment(c, f, S, S.una, MSS, now);
}
// every message whose last byte is acknowledged is complete (step.cuh:1484-1499)
TB_D void messages_acked(HostCtx &c, SndRec &S, int64_t now)
{
    MsgRec *M = c.s->msgs;
    while (S.m_dn < S.m_wr && S.una >= M[S.m_first + S.m_dn].end)
    {
        M[S.m_first + S.m_dn].done = now;
        S.m_dn++;
        c.done++;
    }
    if (S.m_dn == S.m_cnt && (!S.fin_on || (S.fin & FIN_ACKED)))
    {
        S.st = S_DONE;
        S.rto_at = -1;
    }
}

// ReceivedAck + ProcessAck (step.cuh:1502-1693)
TB_D void on_ack(HostCtx &c, int f, SndRec &S, uint32_t ack, bool ece, int64_t now)
{
    if (S.st != S_EST)
        return;
    uint32_t old = S.una;
    if (ack < old)
        return;
    rtt_ack(*c.s, S, ack, now);
    bool advancing = ack > old;
    uint32_t delivered = 0;
    if (advancing)
    {
        Tx t(*c.s, S);
        delivered = discard(t, ack);
    }
    if (S.cong == C_CWR && ack > S.recover)
    {
        S.cong = C_OPEN;
        S.cwnd = S.ssthresh;
    }
    if (advancing && c.dctcp && ece)
    {
        if (S.ecn_echo_seq < (int64_t)ack)
        {
            S.ecn_echo_seq = ack;
            S.ecn_s = E_ECE_RCVD;
            if (S.cong != C_CWR)
            {
                S.ssthresh = ssthresh_for(c, S, inflight(S));
                S.cwnd = S.ssthresh;
                S.cong = C_CWR;
                S.recover = S.high;
            }
        }
    }
    else if (S.ecn_s == E_ECE_RCVD && !ece)
        S.ecn_s = E_IDLE;

    bool dupack = ack == old && ack < S.high;
    uint32_t old_dup = S.dupacks;
    if (dupack)
    {
        uint8_t cg = S.cong;
        if (cg != C_LOSS)
        {
            if (cg != C_RECOVERY)
            {
                S.dupacks++;
                old_dup = S.dupacks - 1;
            }
            if (cg == C_OPEN)
                S.cong = cg = C_DISORDER;
            Tx t(*c.s, S);
            if (cg == C_RECOVERY)
                add_reno_sack(t);
            else if (cg == C_DISORDER)
            {
                if (S.dupacks == DUPTHRESH && (old >= S.recover || !S.recover_active))
                    enter_recovery(c, f, S, now);
                else if (head_lost(t))
                    enter_recovery(c, f, S, now);
            }
        }
    }
    if (ack == old && ack == S.high)
    {
    }
    else if (ack == old && ack > S.high)
        S.nxt = ack;
    else if (ack == old)
        pkts_acked(c, S, 1, ack, now);
    else if (advancing)
    {
        uint32_t segs = delivered / MSS;
        S.ack_rem += delivered % MSS;
        if (S.ack_rem >= MSS)
        {
            segs++;
            S.ack_rem -= MSS;
        }
        if (!dupack)
            S.dupacks = 0;
        uint8_t cg = S.cong;
        if (ack < S.recover && cg == C_RECOVERY)
        {
            Tx t(*c.s, S);
            mark_head_lost(t);
            if (!retx_ends_at(t, ack + MSS))
                do_retransmit(c, f, S, now);
            pkts_acked(c, S, 1, ack, now);
            new_ack(c, S, ack, S.first_partial, now);
            S.first_partial = 0;
        }
        else if (ack < S.recover && cg == C_LOSS)
        {
            pkts_acked(c, S, segs, ack, now);
            increase_window(c, S, segs, ack, now);
            new_ack(c, S, ack, true, now);
        }
        else if (cg == C_CWR)
        {
            pkts_acked(c, S, segs, ack, now);
            new_ack(c, S, ack, true, now);
        }
        else
        {
            bool exited = false;
            if (cg == C_OPEN)
                pkts_acked(c, S, segs, ack, now);
            else if (cg == C_DISORDER)
            {
                if (segs >= old_dup)
                    pkts_acked(c, S, segs - old_dup, ack, now);
                if (!dupack)
                    S.cong = C_OPEN;
            }
            else if (cg == C_RECOVERY)
            {
                S.first_partial = 1;
                segs = (ack - old) / MSS;
                pkts_acked(c, S, segs, ack, now);
                S.cong = C_OPEN;
                exited = true;
                S.dupacks = 0;
            }
            else if (cg == C_LOSS)
            {
                S.first_partial = 1;
                segs = (ack - S.recover) / MSS;
                pkts_acked(c, S, segs, ack, now);
                S.cong = C_OPEN;
            }
            if (ack >= S.recover)
                S.recover_active = 0;
            if (exited)
            {
                new_ack(c, S, ack, true, now);
                S.cwnd = S.ssthresh;
            }
            if (S.cong == C_OPEN)
            {
                increase_window(c, S, segs, ack, now);
                new_ack(c, S, ack, true, now);
            }
        }
    }
    // ProcessWait: the ACK of the FIN moves FIN_WAIT_1 to FIN_WAIT_2
    if ((S.fin & FIN_SENT) && S.it_n == 0 && ack == S.high + 1)
        S.fin |= FIN_ACKED;
    if (advancing)
    {
        messages_acked(c, S, now);
        if (S.st == S_DONE)
            return;
    }
    send_pending(c, f, S, now);
}
// the retransmission timeout (step.cuh:1695-1725)
TB_D void on_rto(HostCtx &c, int f, SndRec &S, int64_t now)
{
    S.rto_at = -1;
    if (S.st != S_EST)
        return;
    if (S.una >= S.tail)
        return;
    c.rtos++;
    uint32_t before = inflight(S);
    S.dupacks = 0;
    {
        Tx t(*c.s, S);
        all_lost(t);
    }
    S.recover = S.high;
    S.recover_active = 1;
    int64_t r = 2 * S.rto;
    S.rto = r < 60000000000000ll ? r : 60000000000000ll;
    S.h_n = 0;
    S.ssthresh = ssthresh_for(c, S, before);
    if (c.cubic)
        cub_loss(S, now);
    S.cong = C_LOSS;
    S.cwnd = MSS;
    send_pending(c, f, S, now);
}

// ------------------------------------------------------------------ receiving
// SYN-ACK (step.cuh:1729-1743)
TB_D void send_synack(HostCtx &c, int f, RcvRec &R, int64_t now)
{
    int64_t rto = CONN_TO_PS << R.syn_n;
    R.syn_n++;
    if (R.synack_t < 0)
        R.synack_t = now;
    emit_rcv(c, f, R, F_SYN | F_ACK, 0, SYN_LEN, now);
    if (R.syn_at < 0)
    {
        R.syn_at = now + rto;
        chain_child(R.dchain, c.ech, code_lead(rto));
    }
}
TB_D void rcv_established(RcvRec &R)
{
    if (!R.est)
    {
        R.est = 1;
        R.syn_at = -1;
    }
}
// DCTCP's CE state machine (step.cuh:1756-1779)
TB_D void ce_state(HostCtx &c, int f, RcvRec &R, bool ce_now, int64_t now)
{
    if (ce_now)
    {
        if (!R.ce_state && R.reserved && R.prior_flag)
            send_ack(c, f, R, R.prior_rcv_nxt, false, true, now);
        R.ce_state = 1;
        R.ecn_r = E_CE_RCVD;
    }
    else
    {
        if (R.ce_state && R.reserved && R.prior_flag)
            send_ack(c, f, R, R.prior_rcv_nxt, true, false, now);
        R.ce_state = 0;
        if (R.ecn_r == E_CE_RCVD || R.ecn_r == E_SENDING_ECE)
            R.ecn_r = E_IDLE;
    }
    R.prior_flag = 1;
    R.prior_rcv_nxt = R.rcv_nxt;
}
// ECN at the receiving socket (step.cuh:1785-1800)
TB_D void rx_ecn(HostCtx &c, int f, RcvRec &R, const Frame &p, int64_t now)
{
    if (!c.dctcp)
        return;
    bool ce = p.flags & F_CE;
    if (ce && R.ecn_ce_seq < (int64_t)p.sa)
    {
        R.ecn_ce_seq = p.sa;
        R.ecn_r = E_CE_RCVD;
        ce_state(c, f, R, true, now);
    }
    else if (p.flags & F_ECT)
        ce_state(c, f, R, false, now);
}
// ECN of ACKs at the sending socket (step.cuh:1806-1822)
TB_D void snd_ecn(HostCtx &c, SndRec &S, const Frame &p)
{
    if (!c.dctcp)
        return;
    if ((p.flags & F_CE) && !(S.s_ce & 1))
    {
        S.s_ce = 3;
        S.ecn_s = E_CE_RCVD;
    }
    else if (p.flags & F_ECT)
    {
        S.s_ce &= ~2;
        if (S.ecn_s == E_CE_RCVD || S.ecn_s == E_SENDING_ECE)
            S.ecn_s = E_IDLE;
    }
}
// TcpRxBuffer::Add: out-of-order blocks, sorted and disjoint beyond rcv_nxt, in a ring
// (step.cuh:1827-1902)
TB_D bool rx_add(const Sim &s, RcvRec &R, uint32_t seq, uint32_t end, unsigned &ovf)
{
    uint32_t head = seq > R.rcv_nxt ? seq : R.rcv_nxt;
    if (head >= end)
        return false;
    uint32_t *bs = s.oo_s + R.oo_off, *be = s.oo_e + R.oo_off;
    const uint32_t cap = R.oo_cap, h0 = R.ooo_h;
    uint32_t n = R.ooo_n;
    auto at = [&](uint32_t i) {
        uint32_t x = h0 + i;
        return x >= cap ? x - cap : x;
    };
    uint32_t i;
    if (n == 0 || be[at(n - 1)] < head)
        i = n;
    else
    {
        uint32_t lo = 0, hi = n - 1;
        while (lo < hi)
        {
            uint32_t m = (lo + hi) / 2;
            if (be[at(m)] < head)
                lo = m + 1;
            else
                hi = m;
        }
        i = lo;
    }
    if (i < n && bs[at(i)] <= head && be[at(i)] >= end)
        return false;
    uint32_t us = head, ue = end, j = i;
    while (j < n && bs[at(j)] <= ue)
    {
        if (bs[at(j)] < us)
            us = bs[at(j)];
        if (be[at(j)] > ue)
            ue = be[at(j)];
        j++;
    }
    if (j == i)
    {
        if (n >= cap)
        {
            ovf++;
            return false;
        }
        for (uint32_t q = n; q > i; q--)
        {
            bs[at(q)] = bs[at(q - 1)];
            be[at(q)] = be[at(q - 1)];
        }
        n++;
    }
    else
    {
        uint32_t gone = j - i - 1;
        if (gone)
            for (uint32_t q = j; q < n; q++)
            {
                bs[at(q - gone)] = bs[at(q)];
                be[at(q - gone)] = be[at(q)];
            }
        n -= gone;
    }
    bs[at(i)] = us;
    be[at(i)] = ue;
    uint32_t h = h0;
    if (head == R.rcv_nxt)
    {
        R.rcv_nxt = be[at(0)];
        h = at(1);
        n--;
    }
    R.ooo_h = n ? h : 0;
    R.ooo_n = n;
    if (R.fin_seq >= 0 && R.rcv_nxt == (uint32_t)R.fin_seq)
        R.rcv_nxt++;
    return true;
}
TB_D bool rx_finished(const RcvRec &R) { return R.fin_seq >= 0 && (uint32_t)R.fin_seq < R.rcv_nxt; }
// the receiver's FIN+ACK (step.cuh:1948-1963)
TB_D void send_fin_ack(HostCtx &c, int f, RcvRec &R, int64_t now)
{
    R.delack_at = -1;
    R.delack_count = 0;
    emit_rcv(c, f, R, F_ACK | F_FIN, R.rcv_nxt, CTRL_LEN, now);
    if (R.frx_at < 0)
    {
        int64_t est = R.srtt >= 0 ? R.srtt : INIT_RTT_PS, v = 4 * R.rttvar;
        int64_t rto = est + (v > GRAN_PS ? v : GRAN_PS);
        rto = rto > MIN_RTO_PS ? rto : MIN_RTO_PS;
        R.frx_at = now + rto;
        chain_child(R.fchain, c.ech, code_lead(rto));
    }
}
TB_D int64_t last_rto(const RcvRec &R)
{
    int64_t est = R.srtt >= 0 ? R.srtt : INIT_RTT_PS, v = 4 * R.rttvar;
    return est + (v > GRAN_PS ? v : GRAN_PS);
}
// DoPeerClose, then Close at once: FIN+ACK, LAST_ACK (step.cuh:1974-1984)
TB_D void do_peer_close(HostCtx &c, int f, RcvRec &R, int64_t now)
{
    R.st = R_LAST_ACK;
    send_fin_ack(c, f, R, now);
    R.last_n = DATA_RETRIES;
    int64_t lr = last_rto(R);
    R.last_at = now + lr;
    chain_child(R.dchain, c.ech, code_lead(lr));
}
TB_D void rcv_closed(RcvRec &R)
{
    R.st = R_CLOSED;
    R.last_at = -1;
    R.frx_at = -1;
    R.delack_at = -1;
}
// ReceivedData (step.cuh:1994-2036)
TB_D void received_data(HostCtx &c, int f, RcvRec &R, uint32_t seq, uint32_t len, bool fin, int64_t now)
{
    uint32_t expected = R.rcv_nxt;
    if (!rx_add(*c.s, R, seq, seq + len, c.ovf))
    {
        send_ack(c, f, R, R.rcv_nxt, false, false, now);
        return;
    }
    if (expected < R.rcv_nxt && rx_finished(R) && !fin)
    {
        do_peer_close(c, f, R, now);
        return;
    }
    bool gap = R.ooo_n > 0;
    bool filled = R.rcv_nxt > expected + len;
    if (gap || filled)
    {
        R.reserved = 0;
        send_ack(c, f, R, R.rcv_nxt, false, false, now);
        return;
    }
    uint32_t cnt = R.delack_count + 1u;
    if (cnt >= DELACK_COUNT)
    {
        R.reserved = 0;
        send_ack(c, f, R, R.rcv_nxt, false, false, now);
    }
    else
    {
        R.delack_count = (uint8_t)cnt;
        R.reserved = 1;
        if (R.delack_at < 0)
        {
            R.delack_at = now + DELACK_PS;
            chain_child(R.dchain, c.ech, code_lead(DELACK_PS));
        }
    }
}
// a data segment (or FIN) at the receiving socket (step.cuh:2040-2101)
TB_D void on_data(HostCtx &c, int f, RcvRec &R, const Frame &p, int64_t now)
{
    if (!R.up || R.st == R_CLOSED)
        return;
    uint32_t seq = p.sa, len = payload_of(p), end = seq + len;
    bool fin = p.flags & F_FIN;
    if (len > 0 && R.est && (R.st == R_LAST_ACK ? seq != R.rcv_nxt : end < R.rcv_nxt))
    {
        send_ack(c, f, R, R.rcv_nxt, false, true, now);
        return;
    }
    rx_ecn(c, f, R, p, now);
    if ((p.flags & F_CWR) && R.est && R.st == R_OPEN && R.ecn_r != E_CE_RCVD)
        R.ecn_r = E_IDLE;
    if (!R.est)
    {
        if (fin && seq != R.rcv_nxt)
            return;
        rcv_established(R);
    }
    if (R.st == R_LAST_ACK)
    {
        if (fin || seq == R.rcv_nxt)
            rcv_closed(R);
        return;
    }
    if (!fin)
    {
        received_data(c, f, R, seq, len, false, now);
        return;
    }
    if (seq < R.rcv_nxt)
        return;
    R.fin_seq = end;
    if (R.rcv_nxt == end)
        R.rcv_nxt++;
    if (len)
        received_data(c, f, R, seq, len, true, now);
    if (!rx_finished(R))
        return;
    do_peer_close(c, f, R, now);
}
TB_D void on_delack(HostCtx &c, int f, RcvRec &R, int64_t now)
{
    R.delack_at = -1;
    R.delack_count = 0;
    R.reserved = 1;
    send_ack(c, f, R, R.rcv_nxt, false, false, now);
}
// FlowSender::Write and Socket::Send's one-step deferral of SendPendingData (step.cuh:2118-2144)
TB_D void app_write(HostCtx &c, int f, SndRec &S, int64_t now)
{
    if (S.m_wr >= S.m_due)
        return;
    MsgRec *M = c.s->msgs;
    while (S.m_wr < S.m_due)
    {
        int m = S.m_first + S.m_wr;
        M[m].est = now;
        S.tail = M[m].end;
        S.m_wr++;
    }
    if (S.fin_on && S.m_wr == S.m_cnt)
        S.fin |= FIN_CLOSE;
    uint32_t pipe = inflight(S);
    if (S.cwnd > pipe && S.syn_at < 0)
    {
        S.syn_at = now + 1;
        chain_child(S.schain, c.ech, CODE_STEP);
        due_insert(c, now + 1, f, 2);
    }
}
TB_D bool add_active(const Sim &s, int *list, int &n, int f, unsigned &ovf)
{
    if (n >= s.act_cap)
    {
        ovf++;
        return false;
    }
    list[n++] = f;
    return true;
}

// a frame at its destination host (on_frame, step.cuh:2147-2236)
TB_D void on_frame(HostCtx &c, HostRec &hr, const Frame &p, int64_t now)
{
    const Sim &s = *c.s;
    int f = (int)p.flow;
    if (p.to_sender)
    {
        SndRec &S = s.snd[f];
        if (p.flags & F_SYN)
        {
            if (S.st == S_SYN_SENT)
            {
                S.st = S_EST;
                S.syn_at = -1;
                rtt_sample(S, now - S.timing_time);
                emit_snd(c, f, S, F_ACK, 0, 0, CTRL_LEN, now);
                chain_child(c.ech, c.ech, CODE_NOW); // ConnectionSucceeded (ScheduleNow)
                app_write(c, f, S, now);
            }
        }
        else if (p.flags & F_FIN)
        {
            if (S.fin & FIN_TW)
                return;
            snd_ecn(c, S, p);
            on_ack(c, f, S, p.sa, p.flags & F_ECE, now);
            S.fin |= FIN_TW;
            emit_snd(c, f, S, F_ACK, 0, 1, CTRL_LEN, now);
        }
        else
        {
            if (S.fin & FIN_TW)
                return;
            snd_ecn(c, S, p);
            on_ack(c, f, S, p.sa, p.flags & F_ECE, now);
        }
        return;
    }
    RcvRec &R = s.rcv[f];
    if (!(p.flags & F_SYN) && R.up && R.srtt < 0 && R.synack_t >= 0)
    {
        int64_t m = now - R.synack_t;
        R.srtt = m;
        R.rttvar = m / 2;
    }
    if (p.flags & F_SYN)
    {
        if (!R.up)
        {
            R.up = 1;
            R.delack_count = DELACK_COUNT;
            add_active(s, s.act_rcv + (size_t)c.h * s.act_cap, hr.n_rcv, f, c.ovf);
        }
        if (R.est)
            return;
        c.nic.woke = now; // CompleteFork is ScheduleNow'd by the SYN's arrival
        chain_child(c.ech, c.ech, CODE_NOW);
        send_synack(c, f, R, now);
    }
    else if (p.flags & (F_DATA | F_FIN))
        on_data(c, f, R, p, now);
    else if (R.up && R.st != R_CLOSED)
    {
        rx_ecn(c, f, R, p, now);
        rcv_established(R);
        if (R.st == R_LAST_ACK)
            rcv_closed(R);
    }
}

} // namespace tb
