// twins-b200: a host's TCP sockets for one slot, as ns-3.46's TcpSocketBase runs them (NewReno, DCTCP
// over TcpLinuxReno, Cubic; TcpTxBuffer without the SACK option, so SACK is emulated from duplicate
// ACKs; TcpRxBuffer; delayed ACKs; FIN and the closing states), over one host's connection records.
// Each function cites the reference code of the same ns-3 behaviour (src/step.cuh), which fixes what
// a simultaneous event sees; the data structures and the order of the checks are this file's own.
#pragma once
#include "tb_egress.cuh"

namespace tb
{

constexpr int DUE_CAP = 64;

// a timer of the host due in the slot: the connection and which one
struct Due
{
    int64_t at;
    int flow;
    int kind; // 0 retransmission, 1 delayed ACK, 2 SYN or deferred send, 3 SYN-ACK, 4 LAST_ACK, 5 FIN+ACK
};

// one host's slot: its egress, the running event's chain, the timers due, counters
struct HostCtx
{
    const Sim *s;
    const WorldDesc *wd;
    int h;
    bool dctcp, cubic;
    Egress nic;
    Chain ech;
    Due due[DUE_CAP];
    int nd, di;
    int64_t slot_end;
    unsigned retx, rtos, ovf, done;
    unsigned long long pkts, snd_pkts;
};

// a timer armed during the slot that falls due before its end joins the slot's timers, after the
// ones of its time already there (reference: due_insert, src/step.cuh:342-360)
TB_D void timer_in_slot(HostCtx &c, int64_t at, int f, int kind)
{
    if (at >= c.slot_end)
        return;
    if (c.nd == DUE_CAP)
    {
        c.ovf++;
        return;
    }
    int j = c.nd++;
    for (; j > c.di && c.due[j - 1].at > at; j--)
        c.due[j] = c.due[j - 1];
    c.due[j] = Due{at, f, kind};
}

// ------------------------------------------------------------------ frames out
// a segment leaves the socket for the host's device queue: data carry their sequence number, the
// others their acknowledgement; the ECMP uplink is the direction's flow hash (reference: emit,
// src/step.cuh:368-384)
TB_D void to_device(HostCtx &c, int f, uint8_t flags, uint32_t num, uint16_t wire_len, bool toward_sender, uint32_t hash, int dst,
                    int64_t now)
{
    Frame fr;
    fr.ts = now;
    fr.flow = (uint32_t)f;
    fr.sa = num;
    fr.len = wire_len;
    fr.dst = (uint16_t)dst;
    fr.flags = (uint8_t)(flags | (c.dctcp ? F_ECT : 0));
    fr.to_sender = toward_sender ? 1 : 0;
    fr.up = (uint16_t)(hash % (uint32_t)c.wd->ecmp_n);
    fr.ch = c.ech;
    c.nic.enqueue(fr, now);
}
TB_D void emit_snd(HostCtx &c, int f, const SndRec &S, uint8_t flags, uint32_t num, uint16_t wire_len, int64_t now)
{
    to_device(c, f, flags, num, wire_len, false, S.hash_data, S.dst_local, now);
}
TB_D void emit_rcv(HostCtx &c, int f, const RcvRec &R, uint8_t flags, uint32_t ack, uint16_t len, int64_t now)
{
    to_device(c, f, flags, ack, len, true, R.hash_ack, R.src_local, now);
}

// the receiver's pure ACK (SendEmptyPacket): ECE while it owes the sender an echo of CE, unless this
// ACK is the one that must not carry it; it cancels a pending delayed ACK (reference: send_ack,
// src/step.cuh:387-407)
enum AckEcho
{
    ECHO_AS_STATE,
    ECHO_FORCE,
    ECHO_NEVER
};
TB_D void rcv_ack(HostCtx &c, int f, RcvRec &R, uint32_t ack, AckEcho echo, int64_t now)
{
    bool ece = echo == ECHO_FORCE;
    if (echo == ECHO_AS_STATE && (R.ecn_r == E_CE_RCVD || R.ecn_r == E_SENDING_ECE))
    {
        R.ecn_r = E_SENDING_ECE;
        ece = true;
    }
    R.delack_count = 0;
    R.delack_at = -1;
    emit_rcv(c, f, R, (uint8_t)(F_ACK | (ece ? F_ECE : 0)), ack, CTRL_LEN, now);
}

// ------------------------------------------------------------------ the sent list
// ns-3's TcpTxBuffer keeps the transmitted items in order (start, size; lost, retransmitted, sacked)
// with byte counters of the three flags and its highest sacked item. Here the items' starts form a
// ring (an item ends where the next begins, the last at `high`), and the flags of each eight ring
// positions share one 32-bit word of the connection's flag bytes: bits 0-7 lost, 8-15
// retransmitted, 16-23 sacked, bit b of a byte for position 8g + b. One load answers eight items,
// so the first retransmission candidate is a scan of a few words, and an item's three flags are one
// word's read and write. Stale bits outside the live items are never read: every item written
// writes its three bits. (The ring's capacity is a multiple of 8 and its offset too, so the words
// are aligned.) Beside ns-3's three byte counters the list counts the candidates' bytes (lost,
// neither retransmitted nor sacked), which tells in O(1) that there is none, and the sacked items,
// where the Reno emulation's next SACK starts looking. `cand_lo` is a lower bound on the first
// candidate's index (where the search for it starts): lowered where an item becomes a candidate,
// moved with the items when some leave the front or two join, raised to what a search finds.
enum : uint8_t
{
    FL_LOST = 1,
    FL_RETX = 2,
    FL_SACK = 4
};

struct SentList
{
    SndRec &S;
    uint32_t *start;
    uint32_t *fw; // flag words
    uint32_t cap;

    TB_D SentList(const Sim &s, SndRec &S_) : S(S_)
    {
        start = s.it_start + S.it_off;
        fw = reinterpret_cast<uint32_t *>(s.it_fl + S.it_off);
        cap = S.it_cap;
    }
    TB_D uint32_t pos(uint32_t i) const
    {
        const uint32_t p = S.it_head + i;
        return p >= cap ? p - cap : p;
    }
    TB_D uint32_t n() const { return S.it_n; }
    TB_D uint32_t beg(uint32_t i) const { return start[pos(i)]; }
    TB_D uint32_t end(uint32_t i) const { return i + 1 < S.it_n ? start[pos(i + 1)] : S.high; }
    TB_D static uint32_t spread(uint8_t f) { return (f & 1u) | (f & 2u) << 7 | (f & 4u) << 14; } // (flag bits -> plane bits)
    TB_D uint8_t flags_at(uint32_t p) const
    {
        const uint32_t w = fw[p >> 3] >> (p & 7);
        return (uint8_t)((w & 1u) | (w >> 7 & 2u) | (w >> 14 & 4u));
    }
    TB_D void write_at(uint32_t p, uint8_t f)
    {
        const uint32_t b = p & 7;
        fw[p >> 3] = (fw[p >> 3] & ~(0x010101u << b)) | spread(f) << b;
    }
    TB_D uint8_t flags(uint32_t i) const { return flags_at(pos(i)); }
    TB_D static bool candidate(uint8_t f) { return (f & (FL_LOST | FL_RETX | FL_SACK)) == FL_LOST; }
    TB_D static uint32_t lowest(uint32_t m) // (m != 0)
    {
#if defined(__CUDA_ARCH__)
        return (uint32_t)__ffs((int)m) - 1;
#else
        return (uint32_t)__builtin_ctz(m);
#endif
    }

    // item i's flags become f; the byte counters follow its length (TcpTxItem's flags with
    // m_lostOut, m_retrans, m_sackedOut, and the candidates' bytes), the sacked items their count
    TB_D void mark(uint32_t i, uint8_t f)
    {
        const uint32_t p = pos(i);
        const uint8_t was = flags_at(p);
        if (was == f)
            return;
        const uint32_t len = end(i) - start[p];
        auto adjust = [&](uint32_t &ctr, bool before, bool after) {
            if (before != after)
                ctr = after ? ctr + len : ctr - len;
        };
        adjust(S.sack_b, was & FL_SACK, f & FL_SACK);
        adjust(S.lost_b, was & FL_LOST, f & FL_LOST);
        adjust(S.rtx_b, was & FL_RETX, f & FL_RETX);
        adjust(S.cand_b, candidate(was), candidate(f));
        if ((was ^ f) & FL_SACK)
            S.sack_n += (f & FL_SACK) ? 1u : ~0u;
        if (candidate(f) && i < S.cand_lo)
            S.cand_lo = i;
        write_at(p, f);
    }

    TB_D uint32_t next_word(uint32_t w) const { return w + 1 == cap >> 3 ? 0 : w + 1; }
    // the flags of positions pos(i) .. pos(n - 1) move up a place (to pos(n)), word by word: each
    // plane byte shifts left, its top bit carried into the next word's bottom; positions below
    // pos(i) in its word and above pos(n) in its word keep theirs (the head of a nearly full ring)
    TB_D void flags_up(uint32_t i)
    {
        const uint32_t p0 = pos(i), pe = pos(S.it_n);
        uint32_t words = ((p0 & 7) + (S.it_n - i)) / 8 + 1; // (the words spanned by pos(i) .. pos(n))
        uint32_t w = p0 >> 3, carry = 0;
        for (bool first = true;; first = false)
        {
            const uint32_t x = fw[w];
            uint32_t y = ((x << 1) & 0xFEFEFEu) | carry;
            carry = (x >> 7) & 0x010101u;
            if (first)
            {
                const uint32_t keep = ((1u << (p0 & 7)) - 1) * 0x010101u;
                y = (x & keep) | (y & ~keep);
            }
            if (--words == 0)
            {
                const uint32_t mine = ((2u << (pe & 7)) - 1) * 0x010101u;
                fw[w] = (y & mine) | (x & ~mine);
                return;
            }
            fw[w] = y;
            w = next_word(w);
        }
    }
    // the flags of positions pos(i + 1) .. pos(n - 1) move down a place (to pos(i)), word by word
    // (the reverse of flags_up; pos(n - 1) is left with a stale copy)
    TB_D void flags_down(uint32_t i)
    {
        const uint32_t p0 = pos(i), pe = pos(S.it_n - 1);
        uint32_t words = ((p0 & 7) + (S.it_n - 1 - i)) / 8 + 1; // (the words spanned by pos(i) .. pos(n - 1))
        uint32_t w = p0 >> 3;
        for (bool first = true;; first = false)
        {
            const uint32_t x = fw[w];
            const uint32_t nx = words == 1 ? 0u : fw[next_word(w)];
            uint32_t y = ((x >> 1) & 0x7F7F7Fu) | ((nx & 0x010101u) << 7);
            if (first)
            {
                const uint32_t keep = ((1u << (p0 & 7)) - 1) * 0x010101u;
                y = (x & keep) | (y & ~keep);
            }
            if (--words == 0)
            {
                const uint32_t mine = ((2u << (pe & 7)) - 1) * 0x010101u;
                fw[w] = (y & mine) | (x & ~mine);
                return;
            }
            fw[w] = y;
            w = next_word(w);
        }
    }

    // a new item at index i, the ones from i moving up a place (new data at the end, or the second
    // half of a split); false when the ring is full (counted)
    TB_D bool open(uint32_t i, uint32_t seq, uint8_t f, unsigned &ovf)
    {
        if (S.it_n >= cap)
        {
            ovf++;
            return false;
        }
        if (i < S.it_n)
        {
            for (uint32_t j = S.it_n; j > i; j--)
                start[pos(j)] = start[pos(j - 1)];
            flags_up(i);
        }
        const uint32_t p = pos(i);
        start[p] = seq;
        if (i == S.it_n && !(p & 7) && S.it_n + 8 <= cap)
            fw[p >> 3] = spread(f); // (an append opening a word whose other positions are all free: no read)
        else
            write_at(p, f);
        S.sack_n += (f & FL_SACK) ? 1u : 0u;
        if (candidate(f) && i < S.cand_lo)
            S.cand_lo = i;
        S.it_n++;
        return true;
    }
    // item i joins item i - 1, which keeps its flags (its start is removed; the ones after it move
    // down a place); the candidates' bytes and the sacked count follow the joined item's flags
    TB_D void join_previous(uint32_t i)
    {
        const uint8_t a = flags(i - 1), b = flags(i);
        const uint32_t lb = end(i) - beg(i);
        S.cand_b += (candidate(a) ? lb : 0u) - (candidate(b) ? lb : 0u);
        S.sack_n -= (b & FL_SACK) ? 1u : 0u;
        if (S.cand_lo >= i)
            S.cand_lo--; // (the items from i move down a place)
        if (i + 1 < S.it_n)
        {
            for (uint32_t j = i; j + 1 < S.it_n; j++)
                start[pos(j)] = start[pos(j + 1)];
            flags_down(i);
        }
        S.it_n--;
    }
    // the first item at or after index from whose planes satisfy want(lost, retx, sack) (eight
    // positions a word; a set bit b: position 8g + b qualifies); n() if none
    template <class Want>
    TB_D uint32_t find(uint32_t from, Want want) const
    {
        for (uint32_t i = from; i < S.it_n;)
        {
            const uint32_t p = pos(i), b = p & 7;
            uint32_t run = 8 - b; // (items of this word from p, within the ring and the list)
            if (run > cap - p)
                run = cap - p;
            if (run > S.it_n - i)
                run = S.it_n - i;
            const uint32_t w = fw[p >> 3];
            const uint32_t m = (want(w & 0xFFu, w >> 8 & 0xFFu, w >> 16 & 0xFFu) >> b) & ((1u << run) - 1);
            if (m)
                return i + lowest(m);
            i += run;
        }
        return S.it_n;
    }
    // the first item starting at or after seq (binary search over the starts)
    TB_D uint32_t first_from(uint32_t seq) const
    {
        uint32_t lo = 0, hi = S.it_n;
        while (lo < hi)
        {
            const uint32_t m = (lo + hi) >> 1;
            if (beg(m) < seq)
                lo = m + 1;
            else
                hi = m;
        }
        return lo;
    }
};

// bytes sent and not acknowledged; BytesInFlight = sent - (sacked + lost) + retransmitted, in
// unsigned arithmetic as ns-3 computes it (reference: src/step.cuh:594-607)
TB_D uint32_t sent_bytes(const SndRec &S) { return S.it_n ? S.high - S.una : 0u; }
TB_D uint32_t inflight(const SndRec &S) { return sent_bytes(S) - (S.sack_b + S.lost_b) + S.rtx_b; }

// a retransmission candidate: lost, neither retransmitted nor sacked
TB_D uint32_t candidates(uint32_t l, uint32_t r, uint32_t k) { return l & ~r & ~k; }

// AddRenoSack: a duplicate ACK counts the first item after the sacked ones (from the second) as
// sacked; the highest sack moves there (reference: src/step.cuh:649-662)
TB_D void reno_sack_one(SentList &L)
{
    SndRec &S = L.S;
    const uint32_t i = L.find(1 + S.sack_n, [](uint32_t, uint32_t, uint32_t k) { return ~k; });
    if (i >= L.n())
        return;
    L.mark(i, (uint8_t)(L.flags(i) | FL_SACK));
    S.sack_seen = 1;
    S.hisack = L.beg(i);
}
// MarkHeadAsLost: the first item is lost, neither sacked nor retransmitted any more (reference:
// src/step.cuh:672-677)
TB_D void head_to_lost(SentList &L)
{
    if (L.n())
        L.mark(0, (uint8_t)((L.flags(0) & ~(FL_SACK | FL_RETX)) | FL_LOST));
}
// an RTO: ResetRenoSack and SetSentListLost, every item lost and nothing else (reference:
// src/step.cuh:687-712)
TB_D void everything_lost(SentList &L)
{
    SndRec &S = L.S;
    // whole words: every position of a word holding a live item reads lost, neither retransmitted
    // nor sacked (its free positions too, which no read reaches before they are written)
    for (uint32_t i = 0; i < S.it_n;)
    {
        const uint32_t p = L.pos(i);
        L.fw[p >> 3] = 0xFFu;
        i += 8 - (p & 7);
    }
    S.lost_b = S.cand_b = sent_bytes(S);
    S.sack_b = S.rtx_b = S.sack_n = S.cand_lo = 0;
    S.sack_seen = 0;
    S.hisack = 0;
}

// DiscardUpTo: the items acknowledged whole leave the list (their bytes are returned), a partly
// acknowledged first item is cut at the ACK; a sacked first item is unsacked and the Reno emulation
// moves on (the next item sacked, the first marked lost); a highest sack at or below the ACK is
// forgotten (reference: src/step.cuh:716-780)
TB_D uint32_t ack_drop(SentList &L, uint32_t ack)
{
    SndRec &S = L.S;
    // (the walk keeps the head, the count and the flags' byte sums in registers and settles the
    // record once; an item leaving keeps its stale flag bits, which no read reaches)
    const uint32_t n = S.it_n, high = S.high;
    uint32_t head = S.it_head, left = 0, gone = 0, sack = 0, lost = 0, retx = 0, cand = 0, nsack = 0;
    uint32_t b = n ? L.start[head] : 0;
    while (left < n)
    {
        const uint32_t nx = head + 1 == L.cap ? 0 : head + 1;
        const uint32_t e = left + 1 < n ? L.start[nx] : high;
        const uint8_t f = L.flags_at(head);
        const uint32_t len = ack < e ? (ack > b ? ack - b : 0) : e - b; // (whole, or the acknowledged part)
        sack += (f & FL_SACK) ? len : 0;
        lost += (f & FL_LOST) ? len : 0;
        retx += (f & FL_RETX) ? len : 0;
        cand += SentList::candidate(f) ? len : 0;
        if (ack < e)
        {
            if (ack > b)
                L.start[head] = ack;
            break;
        }
        nsack += (f & FL_SACK) ? 1 : 0;
        gone += len;
        left++;
        head = nx;
        b = e;
    }
    S.sack_b -= sack;
    S.lost_b -= lost;
    S.rtx_b -= retx;
    S.cand_b -= cand;
    S.sack_n -= nsack;
    S.it_head = head;
    S.it_n = n - left;
    S.cand_lo = S.cand_lo > left ? S.cand_lo - left : 0;
    S.una = ack;
    if (S.it_n && (L.flags(0) & FL_SACK))
    {
        L.mark(0, (uint8_t)(L.flags(0) & ~FL_SACK));
        reno_sack_one(L);
        head_to_lost(L);
    }
    if (S.hisack <= ack)
    {
        S.sack_seen = 0;
        S.hisack = 0;
    }
    return gone;
}

// NextSeg without SACK: the first retransmission candidate, if it lies below the highest sack; else
// new data beyond `high` (reference: src/step.cuh:784-834)
TB_D bool next_to_send(const SentList &L, uint32_t *seq)
{
    const SndRec &S = L.S;
    const uint32_t i = S.cand_b ? L.find(S.cand_lo, candidates) : L.n();
    if (i < L.n())
        L.S.cand_lo = i;
    if (i < L.n() && (!S.sack_seen || L.beg(i) < S.hisack))
    {
        *seq = L.beg(i);
        return true;
    }
    if (S.tail > S.high)
    {
        *seq = S.high;
        return true;
    }
    return false;
}
// IsLost(SND.UNA) (reference: src/step.cuh:838-846)
TB_D bool first_is_lost(const SentList &L)
{
    const SndRec &S = L.S;
    return S.sack_seen && S.una < S.hisack && L.n() && (L.flags(0) & FL_LOST);
}
// IsRetransmittedDataAcked(x): an item ends exactly at x, retransmitted and not sacked (reference:
// src/step.cuh:849-869)
TB_D bool retransmission_ends_at(const SentList &L, uint32_t x)
{
    const SndRec &S = L.S;
    if (!L.n() || x <= S.una || x > S.high)
        return false;
    const uint32_t i = L.first_from(x) - 1; // (the item holding byte x - 1)
    if (L.end(i) != x)
        return false;
    const uint8_t f = L.flags(i);
    return (f & FL_RETX) && !(f & FL_SACK);
}

// GetTransmittedSegment: a retransmission of up to `want` bytes from item i. It may take in the
// next item when that one is not sacked and agrees on being lost (the joined item keeps item i's
// flags, a retransmission mark of either side dropped first), or it may take part of item i (the
// rest becomes an item of its own, same flags); the item sent is marked retransmitted (reference:
// src/step.cuh:874-916)
TB_D uint32_t resend_item(SentList &L, uint32_t i, uint32_t want, unsigned &ovf)
{
    SndRec &S = L.S;
    uint32_t len = L.end(i) - L.beg(i);
    uint32_t limit = len;
    if (i + 1 < S.it_n)
    {
        const uint8_t a = L.flags(i), b = L.flags(i + 1);
        if (!(b & FL_SACK) && (a & FL_LOST) == (b & FL_LOST))
            limit = len + (L.end(i + 1) - L.beg(i + 1));
    }
    const uint32_t take = want < limit ? want : limit;
    if (take > len)
    {
        const uint8_t a = L.flags(i), b = L.flags(i + 1);
        if ((a & FL_RETX) && !(b & FL_RETX))
            L.mark(i, (uint8_t)(a & ~FL_RETX));
        else if ((b & FL_RETX) && !(a & FL_RETX))
            L.mark(i + 1, (uint8_t)(b & ~FL_RETX));
        L.join_previous(i + 1);
        len = L.end(i) - L.beg(i);
    }
    if (take < len)
        L.open(i + 1, L.beg(i) + take, L.flags(i), ovf);
    if (!(L.flags(i) & FL_RETX))
        L.mark(i, (uint8_t)(L.flags(i) | FL_RETX));
    return take;
}

// CopyFromSequence: what a send of up to `want` bytes at seq takes: a retransmission of the item
// starting there (when all of it was sent before), or new data appended as an item (when none of it
// was); a send straddling `high` is cut at `high` (reference: src/step.cuh:920-975)
TB_D uint32_t take_segment(SentList &L, uint32_t want, uint32_t seq, bool *again, unsigned &ovf)
{
    SndRec &S = L.S;
    for (;;)
    {
        const uint32_t avail = S.tail > seq ? S.tail - seq : 0;
        const uint32_t sz = want < avail ? want : avail;
        if (!sz)
            return 0;
        if (seq + sz <= S.high)
        {
            const uint32_t i = L.first_from(seq);
            if (i >= L.n() || L.beg(i) != seq)
            {
                ovf++; // (a send always starts at an item: counted, never seen)
                return 0;
            }
            *again = true;
            return resend_item(L, i, sz, ovf);
        }
        if (seq >= S.high)
        {
            if (!L.open(L.n(), seq, 0, ovf))
                return 0;
            S.high = seq + sz;
            *again = false;
            return sz;
        }
        want = S.high - seq;
    }
}

// ------------------------------------------------------------------ RTT samples and the RTO
// RttMeanDeviation's RTO: srtt + max(4 rttvar, granularity) (the initial RTT while there is no
// sample), at least the minimum RTO unless the caller takes it raw (reference: src/step.cuh:1066-1086)
TB_D int64_t rto_raw(int64_t srtt, int64_t rttvar)
{
    const int64_t v = 4 * rttvar;
    return (srtt >= 0 ? srtt : INIT_RTT_PS) + (v > GRAN_PS ? v : GRAN_PS);
}
TB_D int64_t rto_of(int64_t srtt, int64_t rttvar)
{
    const int64_t r = rto_raw(srtt, rttvar);
    return r > MIN_RTO_PS ? r : MIN_RTO_PS;
}
// a measurement m: the first sets srtt = m, rttvar = m / 2; later ones move srtt by an eighth and
// rttvar by a quarter of the difference, rounded down as ns-3's shifts round
TB_D void rtt_update(SndRec &S, int64_t m)
{
    if (S.srtt < 0)
    {
        S.srtt = m;
        S.rttvar = m / 2;
    }
    else
    {
        const int64_t d = m - S.srtt;
        S.srtt += d >> 3;
        S.rttvar = (3 * S.rttvar + (d < 0 ? -d : d)) >> 2;
    }
    S.rto = rto_of(S.srtt, S.rttvar);
}

// ns-3's RTT history (m_history): an entry per first transmission, oldest first, in a ring of the
// sent list's capacity: its first byte, one past its last, and when it left. A retransmission
// starting inside an entry stretches it to the retransmission's end and keeps its time complemented
// (negative), so that the entry gives no sample (Karn) (reference: src/step.cuh:977-1126)
struct RttLog
{
    SndRec &S;
    uint32_t *lo, *hi;
    int64_t *at;
    TB_D RttLog(const Sim &s, SndRec &S_) : S(S_), lo(s.h_seq + S_.it_off), hi(s.h_end + S_.it_off), at(s.h_t + S_.it_off) {}
    TB_D uint32_t slot(uint32_t j) const
    {
        const uint32_t x = S.h_head + j;
        return x >= S.it_cap ? x - S.it_cap : x;
    }
    TB_D void first_send(uint32_t seq, uint32_t len, int64_t now, unsigned &ovf)
    {
        if (S.h_n == S.it_cap)
        {
            ovf++;
            return;
        }
        const uint32_t k = slot(S.h_n++);
        lo[k] = seq;
        hi[k] = seq + len;
        at[k] = now;
    }
    TB_D void resend(uint32_t seq, uint32_t len)
    {
        for (uint32_t j = 0; j < S.h_n; j++)
        {
            const uint32_t k = slot(j);
            if (seq >= lo[k] && seq < hi[k])
            {
                hi[k] = seq + len;
                if (at[k] >= 0)
                    at[k] = ~at[k];
                return;
            }
        }
    }
    // an ACK: the oldest entry, covered whole and never resent, is a measurement; every entry it
    // covers whole is dropped
    TB_D void acked(uint32_t ack, int64_t now)
    {
        if (!S.h_n)
            return;
        const uint32_t k = slot(0);
        if (at[k] >= 0 && ack >= hi[k])
            rtt_update(S, now - at[k]);
        while (S.h_n && hi[slot(0)] <= ack)
        {
            S.h_head = slot(1);
            S.h_n--;
        }
    }
};

// ------------------------------------------------------------------ TcpCubic
// ns-3's TcpCubic with fast convergence, TCP friendliness and HyStart's delay exit, over the
// connection's cub_* fields; windows in segments (reference: src/step.cuh:1201-1345)
namespace cubic
{
constexpr double C = 0.4, BETA = 0.7;
constexpr int64_t ACK_DELTA = 2000000000, DELAY_MIN = 4000000000, DELAY_MAX = 1000000000000, EPOCH_GUARD = 10000000000;
// Reno's growth per cubic ACK count in TCP-friendly mode, 8 (1 + beta) / (3 (1 - beta)) in ns-3's
// 1024-scaled terms, truncated
constexpr uint32_t FRIENDLY = 15;
static_assert((uint32_t)(8 * (1024 + BETA * 1024) / 3 / (1024 - BETA * 1024)) == FRIENDLY, "Cubic's friendliness factor");

// double -> uint32_t as ns-3's x86-64 build converts it: to a 64-bit integer (out of range: the
// "integer indefinite" INT64_MIN), then its low half
TB_D uint32_t x86_u32(double d)
{
    const bool fits = d >= -9223372036854775808.0 && d < 9223372036854775808.0;
    return (uint32_t)(uint64_t)(fits ? (int64_t)d : INT64_MIN);
}
// HyStart's round: starts now, ends when the byte after the highest sent is acknowledged
TB_D void new_round(SndRec &S, int64_t now)
{
    S.cub_roundstart = S.cub_lastack = now;
    S.cub_endseq = S.st == S_EST ? S.high + 1 : 0;
    S.cub_currrtt = INT64_MIN;
    S.cub_samples = 0;
}
// K = cbrt(n / C) as the host's libm pow(n / C, 1/3) gives it (a host-made table), else the device pow
TB_D double k_of(const Sim &s, uint32_t n)
{
    return n < (uint32_t)s.cub_k_n ? s.cub_k_tab[n] : tb_pow((double)n / C, 1 / 3.);
}
// the ACKs that one more segment of window takes (ns-3's Update)
TB_D uint32_t acks_per_segment(const Sim &s, SndRec &S, uint32_t segs, int64_t now)
{
    const uint32_t w = S.cwnd / MSS;
    S.cub_ackcnt += segs;
    if (S.cub_epoch == INT64_MIN)
    {
        // a new epoch: the curve's plateau is the window before the last loss, K away
        const bool below = S.cub_lastmax > w;
        S.cub_epoch = now;
        S.cub_ackcnt = segs;
        S.cub_tcpcwnd = w;
        S.cub_k = below ? k_of(s, S.cub_lastmax - w) : 0.0;
        S.cub_origin = below ? S.cub_lastmax : w;
    }
    // the curve one minimum RTT ahead: origin -/+ C |t - K|^3
    const int64_t t = (int64_t)((uint64_t)now + (uint64_t)S.cub_delaymin - (uint64_t)S.cub_epoch);
    const double ts = get_seconds(t), K = S.cub_k;
    const bool rising = ts < K;
    const uint32_t d = x86_u32(C * tb_pow(rising ? K - ts : ts - K, 3));
    const uint32_t target = rising ? S.cub_origin - d : S.cub_origin + d;
    uint32_t cnt = target > w ? w / (target - w) : 100 * w;
    if (S.cub_lastmax == 0 && cnt > 20)
        cnt = 20;
    // TCP friendliness: the window Reno would have reached on the same ACKs bounds cnt
    const uint32_t per = (w * FRIENDLY) >> 3;
    if (S.cub_ackcnt > per)
    {
        const uint32_t k = (S.cub_ackcnt - 1) / per;
        S.cub_ackcnt -= k * per;
        S.cub_tcpcwnd += k;
    }
    if (S.cub_tcpcwnd > w)
    {
        const uint32_t bound = w / (S.cub_tcpcwnd - w);
        cnt = cnt < bound ? cnt : bound;
    }
    return cnt > 2 ? cnt : 2;
}
// PktsAcked: the minimum delay and HyStart's exit from slow start (an ACK train as long as the
// minimum delay, or an RTT rise over it in a round's first eight samples)
TB_D void on_acked(SndRec &S, int64_t now)
{
    if (S.cub_epoch != INT64_MIN && now - S.cub_epoch < EPOCH_GUARD)
        return;
    const int64_t rtt = S.srtt;
    if (S.cub_delaymin == INT64_MIN || S.cub_delaymin > rtt)
        S.cub_delaymin = rtt;
    const uint32_t w = S.cwnd;
    if (S.cub_found || w > S.ssthresh || w < 16 * MSS)
        return;
    if (now - S.cub_lastack <= ACK_DELTA)
    {
        S.cub_lastack = now;
        if (now - S.cub_roundstart > S.cub_delaymin)
            S.cub_found = 1;
    }
    if (S.cub_samples >= 8)
    {
        const int64_t dm = S.cub_delaymin;
        const int64_t slack = dm < DELAY_MIN ? DELAY_MIN : dm > DELAY_MAX ? DELAY_MAX : dm;
        if (S.cub_currrtt > dm + slack)
            S.cub_found = 1;
    }
    else
    {
        if (S.cub_currrtt == INT64_MIN || S.cub_currrtt > rtt)
            S.cub_currrtt = rtt;
        S.cub_samples++;
    }
    if (S.cub_found)
        S.ssthresh = w;
}
// IncreaseWindow: slow start by whole segments, else one segment per acks_per_segment ACKs
TB_D void grow(const Sim &s, SndRec &S, uint32_t segs, uint32_t ack, int64_t now)
{
    if (!S.cwnd_limited)
        return;
    if (S.cwnd < S.ssthresh)
    {
        if (ack + 1 > S.cub_endseq)
            new_round(S, now);
        S.cwnd += segs * MSS;
        return;
    }
    if (!segs)
        return;
    S.cub_cnt += segs;
    const uint32_t cnt = acks_per_segment(s, S, segs, now);
    if (S.cub_cnt >= cnt)
    {
        S.cwnd += MSS;
        S.cub_cnt -= cnt;
    }
}
// GetSsThresh: beta of the window; the plateau remembered (lowered further when the window did
// not regain the last one: fast convergence); a new epoch begins at the next increase
TB_D uint32_t ssthresh(SndRec &S)
{
    const uint32_t w = S.cwnd / MSS;
    S.cub_lastmax = w < S.cub_lastmax ? x86_u32((w * (1 + BETA)) / 2) : w;
    S.cub_epoch = INT64_MIN;
    const uint32_t th = x86_u32(w * BETA);
    return (th > 2 ? th : 2) * MSS;
}
// CongestionStateSet(CA_LOSS): the curve and HyStart start over
TB_D void on_loss(SndRec &S, int64_t now)
{
    S.cub_origin = 0;
    S.cub_k = 0;
    S.cub_ackcnt = 0;
    S.cub_tcpcwnd = 0;
    S.cub_delaymin = INT64_MIN;
    S.cub_found = 0;
    new_round(S, now);
}
} // namespace cubic

// ------------------------------------------------------------------ NewReno, DCTCP (over Linux Reno)
// GetSsThresh of the three (reference: src/step.cuh:1055-1063)
TB_D uint32_t ssthresh_after(HostCtx &c, SndRec &S, uint32_t flight)
{
    if (c.cubic)
        return cubic::ssthresh(S);
    if (c.dctcp)
        return (uint32_t)((1.0 - S.alpha / 2.0) * S.cwnd);
    return flight / 2 > 2 * MSS ? flight / 2 : 2 * MSS;
}
// DCTCP's alpha: once per window of data (up to the byte next after the highest sent when the
// window began), alpha <- (1 - g) alpha + g F, F the window's ECE-acknowledged fraction, in the fused
// multiply-add ns-3's -march=native build makes of it
TB_D void dctcp_acked(SndRec &S, uint32_t segs, uint32_t ack)
{
    const uint32_t bytes = segs * MSS;
    S.acked_total += bytes;
    if (S.ecn_s == E_ECE_RCVD)
        S.acked_ecn += bytes;
    if (!S.next_seq_flag)
    {
        S.next_seq_flag = 1;
        S.next_seq = S.nxt;
    }
    if (ack < S.next_seq)
        return;
    const double frac = S.acked_total ? (double)S.acked_ecn / S.acked_total : 0.0;
    S.alpha = tb_fma(1.0 - DCTCP_G, S.alpha, DCTCP_G * frac);
    S.next_seq = S.nxt;
    S.acked_total = S.acked_ecn = 0;
}
// PktsAcked (reference: src/step.cuh:1348-1381)
TB_D void acked_segments(HostCtx &c, SndRec &S, uint32_t segs, uint32_t ack, int64_t now)
{
    if (c.cubic)
        cubic::on_acked(S, now);
    else if (c.dctcp)
        dctcp_acked(S, segs, ack);
}
// TcpLinuxReno (DCTCP's window): slow start up to ssthresh; then a segment per window of ACKs,
// counted in cwnd_cnt
TB_D void linux_reno_grow(SndRec &S, uint32_t segs)
{
    if (S.cwnd < S.ssthresh)
    {
        if (segs)
        {
            const uint64_t w = (uint64_t)S.cwnd + (uint64_t)segs * MSS;
            S.cwnd = (uint32_t)(w < S.ssthresh ? w : S.ssthresh);
        }
        return;
    }
    const uint32_t per = S.cwnd / MSS ? S.cwnd / MSS : 1;
    if (S.cwnd_cnt >= per)
    {
        S.cwnd_cnt = 0;
        S.cwnd += MSS;
    }
    S.cwnd_cnt += segs;
    if (S.cwnd_cnt >= per)
    {
        const uint32_t whole = S.cwnd_cnt / per;
        S.cwnd_cnt -= whole * per;
        S.cwnd += whole * MSS;
    }
}
// TcpNewReno: one segment of slow start per ACK, then MSS^2 / cwnd (at least a byte)
TB_D void newreno_grow(SndRec &S, uint32_t segs)
{
    if (S.cwnd < S.ssthresh && segs)
    {
        S.cwnd += MSS;
        segs--;
    }
    if (S.cwnd >= S.ssthresh && segs)
    {
        const double step = (double)MSS * MSS / S.cwnd;
        S.cwnd += (uint32_t)(step > 1.0 ? step : 1.0);
    }
}
// IncreaseWindow (reference: src/step.cuh:1383-1440)
TB_D void grow_window(HostCtx &c, SndRec &S, uint32_t segs, uint32_t ack, int64_t now)
{
    if (c.cubic)
        cubic::grow(*c.s, S, segs, ack, now);
    else if (c.dctcp)
        linux_reno_grow(S, segs);
    else
        newreno_grow(S, segs);
}

// ------------------------------------------------------------------ sending
TB_D void arm_retx_timer(HostCtx &c, SndRec &S, int64_t now)
{
    S.rto_at = now + S.rto;
    chain_child(S.rchain, c.ech, code_lead(S.rto));
}
// SendDataPacket: a segment of up to max_len bytes at seq (CWR on the first new one after an echo,
// FIN on the one reaching the end of a closing stream); the retransmission timer starts if idle;
// the RTT history notes it (reference: src/step.cuh:1129-1172)
TB_D uint32_t transmit(HostCtx &c, int f, SndRec &S, uint32_t seq, uint32_t max_len, int64_t now)
{
    SentList L(*c.s, S);
    bool again = false;
    const uint32_t len = take_segment(L, max_len, seq, &again, c.ovf);
    if (!len)
        return 0;
    uint8_t flags = F_DATA;
    if (!again && S.ecn_s == E_ECE_RCVD && S.ecn_echo_seq > S.ecn_cwr_seq)
    {
        flags |= F_CWR;
        S.ecn_s = E_CWR_SENT;
        S.ecn_cwr_seq = seq;
    }
    if ((S.fin & FIN_CLOSE) && seq + len == S.tail)
    {
        flags |= F_FIN;
        S.fin |= FIN_SENT;
    }
    emit_snd(c, f, S, flags, seq, (uint16_t)(len + HDR_BYTES), now);
    c.retx += again;
    if (S.rto_at < 0)
        arm_retx_timer(c, S, now);
    S.cwnd_limited = S.cwnd < inflight(S) + MSS;
    RttLog log(*c.s, S);
    if (again)
        log.resend(seq, len);
    else
        log.first_send(seq, len, now, c.ovf);
    if (seq + len > S.high)
        S.high = seq + len;
    return len;
}
// SendPendingData: segments while the window has room (a part of a segment only when it ends the
// data), retransmissions first; nothing more in Open once the FIN is out (reference:
// src/step.cuh:1175-1199)
TB_D void send_pending(HostCtx &c, int f, SndRec &S, int64_t now)
{
    if (S.st != S_EST)
        return;
    for (int n = 0; n < 4096; n++)
    {
        if (S.cong == C_OPEN && (S.fin & (FIN_SENT | FIN_ACKED)) == FIN_SENT)
            return;
        const uint32_t flight = inflight(S);
        const uint32_t room = S.cwnd > flight ? S.cwnd - flight : 0;
        uint32_t seq;
        if (!room || !next_to_send(SentList(*c.s, S), &seq))
            return;
        if (room < MSS && S.tail - seq > room)
            return;
        S.nxt = seq;
        const uint32_t len = transmit(c, f, S, seq, room < MSS ? room : MSS, now);
        if (!len)
            return;
        S.nxt = seq + len;
    }
}
// DoRetransmit: the first retransmission candidate, else the first unacknowledged byte (reference:
// src/step.cuh:1202-1212)
TB_D void retransmit_one(HostCtx &c, int f, SndRec &S, int64_t now)
{
    if (S.una >= S.tail)
        return;
    uint32_t seq;
    if (!next_to_send(SentList(*c.s, S), &seq))
        seq = S.una;
    S.nxt = seq;
    transmit(c, f, S, seq, MSS, now);
}
// NewAck: the retransmission timer restarts from the estimator (optionally), stops once everything
// is acknowledged unless a FIN is out; nxt never trails the ACK (reference: src/step.cuh:1445-1464)
TB_D void new_ack(HostCtx &c, SndRec &S, uint32_t ack, bool restart, int64_t now)
{
    if (restart)
    {
        S.rto = rto_of(S.srtt, S.rttvar);
        arm_retx_timer(c, S, now);
    }
    if (ack >= S.tail && !(S.fin & FIN_SENT))
        S.rto_at = -1;
    if (ack > S.nxt)
        S.nxt = ack;
}
// EnterRecovery: a third duplicate (or a lost head) starts fast recovery: the Reno SACK of this
// duplicate, the head lost, recover = the highest sent, the window to ssthresh and the head resent
// (reference: src/step.cuh:1467-1481)
TB_D void enter_recovery(HostCtx &c, int f, SndRec &S, int64_t now)
{
    {
        SentList L(*c.s, S);
        reno_sack_one(L);
        head_to_lost(L);
    }
    S.cong = C_RECOVERY;
    S.recover = S.high;
    S.recover_active = 1;
    S.ssthresh = ssthresh_after(c, S, inflight(S) + MSS);
    S.cwnd = S.ssthresh;
    transmit(c, f, S, S.una, MSS, now);
}
// messages whose last byte is acknowledged are complete; the connection is done with the last
// (and its FIN's ACK, with FIN) (reference: src/step.cuh:1484-1499)
TB_D void messages_acked(HostCtx &c, SndRec &S, int64_t now)
{
    MsgRec *M = c.s->msgs + S.m_first;
    for (; S.m_dn < S.m_wr && S.una >= M[S.m_dn].end; S.m_dn++, c.done++)
        M[S.m_dn].done = now;
    if (S.m_dn == S.m_cnt && (!S.fin_on || (S.fin & FIN_ACKED)))
    {
        S.st = S_DONE;
        S.rto_at = -1;
    }
}

// ------------------------------------------------------------------ ACKs at the sender
// a duplicate ACK by congestion state: counted (Recovery counts Reno SACKs instead), Open turns
// Disorder, and in Disorder the third duplicate (past any earlier recovery point) or a lost head
// enters recovery; Loss ignores it
TB_D void duplicate_ack(HostCtx &c, int f, SndRec &S, uint32_t una_before, int64_t now)
{
    switch (S.cong)
    {
    case C_LOSS:
        return;
    case C_RECOVERY: {
        SentList L(*c.s, S);
        reno_sack_one(L);
        return;
    }
    case C_CWR:
        S.dupacks++;
        return;
    default: // Open, Disorder
        S.dupacks++;
        S.cong = C_DISORDER;
        if ((S.dupacks == DUPTHRESH && (una_before >= S.recover || !S.recover_active)) || first_is_lost(SentList(*c.s, S)))
            enter_recovery(c, f, S, now);
    }
}
// an ACK that moves una: `bytes` left the sent list; segments acknowledged with the remainder
// carried over. Partial ACKs of a recovery retransmit; otherwise the state returns to Open and the
// window grows (reference: src/step.cuh:1580-1680)
TB_D void advancing_ack(HostCtx &c, int f, SndRec &S, uint32_t ack, uint32_t una_before, uint32_t bytes, int64_t now)
{
    uint32_t segs = bytes / MSS;
    S.ack_rem += bytes % MSS;
    if (S.ack_rem >= MSS)
    {
        S.ack_rem -= MSS;
        segs++;
    }
    const uint32_t dups = S.dupacks;
    S.dupacks = 0;
    const bool partial = ack < S.recover;
    if (partial && S.cong == C_RECOVERY)
    {
        // NewReno's partial ACK: the new head is lost and resent unless it just was
        bool resend;
        {
            SentList L(*c.s, S);
            head_to_lost(L);
            resend = !retransmission_ends_at(L, ack + MSS);
        }
        if (resend)
            retransmit_one(c, f, S, now);
        acked_segments(c, S, 1, ack, now);
        new_ack(c, S, ack, S.first_partial, now);
        S.first_partial = 0;
        return;
    }
    if (partial && S.cong == C_LOSS)
    {
        acked_segments(c, S, segs, ack, now);
        grow_window(c, S, segs, ack, now);
        new_ack(c, S, ack, true, now);
        return;
    }
    if (S.cong == C_CWR)
    {
        acked_segments(c, S, segs, ack, now);
        new_ack(c, S, ack, true, now);
        return;
    }
    switch (S.cong)
    {
    case C_OPEN:
        acked_segments(c, S, segs, ack, now);
        break;
    case C_DISORDER:
        if (segs >= dups)
            acked_segments(c, S, segs - dups, ack, now);
        break;
    case C_RECOVERY: // the recovery point reached: the window deflates to ssthresh
        S.first_partial = 1;
        segs = (ack - una_before) / MSS;
        acked_segments(c, S, segs, ack, now);
        S.cwnd = S.ssthresh;
        break;
    default: // Loss, the recovery point reached
        S.first_partial = 1;
        segs = (ack - S.recover) / MSS;
        acked_segments(c, S, segs, ack, now);
    }
    S.cong = C_OPEN;
    if (!partial)
        S.recover_active = 0;
    grow_window(c, S, segs, ack, now);
    new_ack(c, S, ack, true, now);
}
// ReceivedAck and ProcessAck, for an ACK with or without ECE (reference: src/step.cuh:1502-1693)
TB_D void on_ack(HostCtx &c, int f, SndRec &S, uint32_t ack, bool ece, int64_t now)
{
    if (S.st != S_EST || ack < S.una)
        return;
    const uint32_t una_before = S.una;
    const bool moves = ack > una_before;
    RttLog(*c.s, S).acked(ack, now);
    uint32_t bytes = 0;
    if (moves)
    {
        SentList L(*c.s, S);
        bytes = ack_drop(L, ack);
    }
    if (S.cong == C_CWR && ack > S.recover)
    {
        S.cong = C_OPEN;
        S.cwnd = S.ssthresh;
    }
    // ECN: an ECE on new data (once per echo sequence) cuts the window and enters CWR; an ACK
    // without ECE ends the echo
    if (!ece)
    {
        if (S.ecn_s == E_ECE_RCVD)
            S.ecn_s = E_IDLE;
    }
    else if (moves && c.dctcp && S.ecn_echo_seq < (int64_t)ack)
    {
        S.ecn_echo_seq = ack;
        S.ecn_s = E_ECE_RCVD;
        if (S.cong != C_CWR)
        {
            S.ssthresh = ssthresh_after(c, S, inflight(S));
            S.cwnd = S.ssthresh;
            S.cong = C_CWR;
            S.recover = S.high;
        }
    }
    if (moves)
        advancing_ack(c, f, S, ack, una_before, bytes, now);
    else if (ack < S.high)
    {
        duplicate_ack(c, f, S, una_before, now);
        acked_segments(c, S, 1, ack, now);
    }
    else if (ack > S.high)
        S.nxt = ack;
    // FIN_WAIT_1 -> FIN_WAIT_2 on the FIN's ACK
    if ((S.fin & FIN_SENT) && !S.it_n && ack == S.high + 1)
        S.fin |= FIN_ACKED;
    if (moves)
    {
        messages_acked(c, S, now);
        if (S.st == S_DONE)
            return;
    }
    send_pending(c, f, S, now);
}
// the retransmission timeout: everything sent is lost, the timer backs off (at most 60 s), the
// history is dropped, the window falls to a segment in Loss and sending resumes from the head
// (reference: src/step.cuh:1695-1725)
TB_D void on_rto(HostCtx &c, int f, SndRec &S, int64_t now)
{
    S.rto_at = -1;
    if (S.st != S_EST || S.una >= S.tail)
        return;
    c.rtos++;
    const uint32_t flight = inflight(S);
    {
        SentList L(*c.s, S);
        everything_lost(L);
    }
    S.dupacks = 0;
    S.recover = S.high;
    S.recover_active = 1;
    S.rto = 2 * S.rto < 60000000000000ll ? 2 * S.rto : 60000000000000ll;
    S.h_n = 0;
    S.ssthresh = ssthresh_after(c, S, flight);
    if (c.cubic)
        cubic::on_loss(S, now);
    S.cong = C_LOSS;
    S.cwnd = MSS;
    send_pending(c, f, S, now);
}

// ------------------------------------------------------------------ the receiving socket
// SYN-ACK, its timer backing off from the connection timeout (reference: src/step.cuh:1729-1743)
TB_D void send_synack(HostCtx &c, int f, RcvRec &R, int64_t now)
{
    const int64_t to = CONN_TO_PS << R.syn_n++;
    if (R.synack_t < 0)
        R.synack_t = now;
    emit_rcv(c, f, R, F_SYN | F_ACK, 0, SYN_LEN, now);
    if (R.syn_at >= 0)
        return;
    R.syn_at = now + to;
    chain_child(R.dchain, c.ech, code_lead(to));
}
TB_D void rcv_established(RcvRec &R)
{
    if (R.est)
        return;
    R.est = 1;
    R.syn_at = -1;
}
// DCTCP's receiver: when the CE state flips while an ACK is withheld by the delayed-ACK count, that
// ACK goes out now with the old state's echo; the state and the sequence it covers are kept
// (reference: src/step.cuh:1756-1779)
TB_D void ce_flip(HostCtx &c, int f, RcvRec &R, bool ce, int64_t now)
{
    if (R.reserved && R.prior_flag && (R.ce_state != 0) != ce)
        rcv_ack(c, f, R, R.prior_rcv_nxt, ce ? ECHO_NEVER : ECHO_FORCE, now);
    R.ce_state = ce;
    if (ce)
        R.ecn_r = E_CE_RCVD;
    else if (R.ecn_r == E_CE_RCVD || R.ecn_r == E_SENDING_ECE)
        R.ecn_r = E_IDLE;
    R.prior_flag = 1;
    R.prior_rcv_nxt = R.rcv_nxt;
}
// ECN at the receiving socket: a CE mark beyond the last one seen flips the state to CE; any other
// ECT frame flips it back (reference: src/step.cuh:1785-1800)
TB_D void rcv_ecn(HostCtx &c, int f, RcvRec &R, const Frame &p, int64_t now)
{
    if (!c.dctcp)
        return;
    if ((p.flags & F_CE) && R.ecn_ce_seq < (int64_t)p.sa)
    {
        R.ecn_ce_seq = p.sa;
        R.ecn_r = E_CE_RCVD;
        ce_flip(c, f, R, true, now);
    }
    else if (p.flags & F_ECT)
        ce_flip(c, f, R, false, now);
}
// ECN of the ACKs at the sending socket (reference: src/step.cuh:1806-1822)
TB_D void snd_ecn(HostCtx &c, SndRec &S, const Frame &p)
{
    if (!c.dctcp)
        return;
    if ((p.flags & F_CE) && !(S.s_ce & 1))
    {
        S.s_ce = 3;
        S.ecn_s = E_CE_RCVD;
        return;
    }
    if (!(p.flags & F_ECT))
        return;
    S.s_ce &= ~2;
    if (S.ecn_s == E_CE_RCVD || S.ecn_s == E_SENDING_ECE)
        S.ecn_s = E_IDLE;
}

// TcpRxBuffer::Add: the bytes [seq, end) beyond rcv_nxt join the out-of-order blocks (sorted,
// disjoint, never touching; a ring at oo_off). The blocks the new bytes overlap or touch fold into
// one with them; in-order bytes move rcv_nxt to the end of that block, which never enters the ring.
// False when nothing is new (reference: src/step.cuh:1827-1902)
TB_D bool rx_add(const Sim &s, RcvRec &R, uint32_t seq, uint32_t end, unsigned &ovf)
{
    const uint32_t from = seq > R.rcv_nxt ? seq : R.rcv_nxt;
    if (from >= end)
        return false;
    uint32_t *bs = s.oo_s + R.oo_off, *be = s.oo_e + R.oo_off;
    const uint32_t cap = R.oo_cap, n = R.ooo_n;
    auto at = [&](uint32_t i) {
        const uint32_t x = R.ooo_h + i;
        return x >= cap ? x - cap : x;
    };
    // blocks [lo, hi) overlap or touch [from, end): lo = the first ending at or after `from`,
    // hi = the first starting after `end`; the common cases in O(1): bytes beyond every block (an
    // out-of-order arrival after the last), or short of the first block (in order, a gap ahead)
    uint32_t lo = n, hi = n;
    if (n && be[at(n - 1)] >= from)
    {
        lo = 0;
        if (be[at(0)] < from)
        {
            uint32_t a = 1, b = n - 1; // (the answer lies in [1, n - 1]: the last block qualifies)
            while (a < b)
            {
                const uint32_t m = (a + b) >> 1;
                if (be[at(m)] < from)
                    a = m + 1;
                else
                    b = m;
            }
            lo = a;
        }
        hi = lo;
        if (bs[at(lo)] <= end)
        {
            uint32_t a = lo + 1, b = n;
            while (a < b)
            {
                const uint32_t m = (a + b) >> 1;
                if (bs[at(m)] <= end)
                    a = m + 1;
                else
                    b = m;
            }
            hi = a;
        }
    }
    if (lo < n && bs[at(lo)] <= from && be[at(lo)] >= end)
        return false; // (held already)
    const uint32_t us = lo < hi && bs[at(lo)] < from ? bs[at(lo)] : from;
    const uint32_t ue = lo < hi && be[at(hi - 1)] > end ? be[at(hi - 1)] : end;
    if (from == R.rcv_nxt)
    {
        // in order (then lo = 0): the folded block is delivered, the blocks it swallowed leave
        R.rcv_nxt = ue;
        R.ooo_h = at(hi);
        R.ooo_n = n - hi;
    }
    else if (lo == hi)
    {
        if (n == cap)
        {
            ovf++;
            return false;
        }
        for (uint32_t i = n; i > lo; i--)
        {
            bs[at(i)] = bs[at(i - 1)];
            be[at(i)] = be[at(i - 1)];
        }
        bs[at(lo)] = us;
        be[at(lo)] = ue;
        R.ooo_n = n + 1;
    }
    else
    {
        const uint32_t gone = hi - lo - 1;
        bs[at(lo)] = us;
        be[at(lo)] = ue;
        for (uint32_t i = hi; gone && i < n; i++)
        {
            bs[at(i - gone)] = bs[at(i)];
            be[at(i - gone)] = be[at(i)];
        }
        R.ooo_n = n - gone;
    }
    if (R.fin_seq >= 0 && R.rcv_nxt == (uint32_t)R.fin_seq)
        R.rcv_nxt++;
    return true;
}
TB_D bool rx_finished(const RcvRec &R) { return R.fin_seq >= 0 && (uint32_t)R.fin_seq < R.rcv_nxt; }

// the receiver's FIN+ACK; its own retransmission timer from the receiver's estimator (reference:
// src/step.cuh:1948-1963)
TB_D void send_fin_ack(HostCtx &c, int f, RcvRec &R, int64_t now)
{
    R.delack_at = -1;
    R.delack_count = 0;
    emit_rcv(c, f, R, F_ACK | F_FIN, R.rcv_nxt, CTRL_LEN, now);
    if (R.frx_at >= 0)
        return;
    const int64_t to = rto_of(R.srtt, R.rttvar);
    R.frx_at = now + to;
    chain_child(R.fchain, c.ech, code_lead(to));
}
TB_D void arm_last_ack(HostCtx &c, RcvRec &R, int64_t now)
{
    const int64_t to = rto_raw(R.srtt, R.rttvar); // (LastAckTimeout takes the RTO unclamped)
    R.last_at = now + to;
    chain_child(R.dchain, c.ech, code_lead(to));
}
// DoPeerClose and the application's Close right after: FIN+ACK, LAST_ACK (reference:
// src/step.cuh:1974-1984)
TB_D void do_peer_close(HostCtx &c, int f, RcvRec &R, int64_t now)
{
    R.st = R_LAST_ACK;
    send_fin_ack(c, f, R, now);
    R.last_n = DATA_RETRIES;
    arm_last_ack(c, R, now);
}
TB_D void rcv_closed(RcvRec &R)
{
    R.st = R_CLOSED;
    R.last_at = R.frx_at = R.delack_at = -1;
}
// ReceivedData: new bytes into the buffer; an ACK at once for a gap (or a filled one) or every
// second segment, else the delayed-ACK timer (reference: src/step.cuh:1994-2036)
TB_D void received_data(HostCtx &c, int f, RcvRec &R, uint32_t seq, uint32_t len, bool fin, int64_t now)
{
    const uint32_t expected = R.rcv_nxt;
    if (!rx_add(*c.s, R, seq, seq + len, c.ovf))
    {
        rcv_ack(c, f, R, R.rcv_nxt, ECHO_AS_STATE, now);
        return;
    }
    if (expected < R.rcv_nxt && rx_finished(R) && !fin)
    {
        do_peer_close(c, f, R, now);
        return;
    }
    if (R.ooo_n || R.rcv_nxt > expected + len || R.delack_count + 1u >= DELACK_COUNT)
    {
        R.reserved = 0;
        rcv_ack(c, f, R, R.rcv_nxt, ECHO_AS_STATE, now);
        return;
    }
    R.delack_count++;
    R.reserved = 1;
    if (R.delack_at >= 0)
        return;
    R.delack_at = now + DELACK_PS;
    chain_child(R.dchain, c.ech, code_lead(DELACK_PS));
}
// a data segment or FIN at the receiving socket: old data get a duplicate ACK without ECE; a FIN
// is taken in order only; LAST_ACK closes on the FIN's ACK (reference: src/step.cuh:2040-2101)
TB_D void on_data(HostCtx &c, int f, RcvRec &R, const Frame &p, int64_t now)
{
    if (!R.up || R.st == R_CLOSED)
        return;
    const uint32_t seq = p.sa, len = payload_of(p), end = seq + len;
    const bool fin = p.flags & F_FIN;
    if (len && R.est && (R.st == R_LAST_ACK ? seq != R.rcv_nxt : end < R.rcv_nxt))
    {
        rcv_ack(c, f, R, R.rcv_nxt, ECHO_NEVER, now);
        return;
    }
    rcv_ecn(c, f, R, p, now);
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
    if (rx_finished(R))
        do_peer_close(c, f, R, now);
}

// ------------------------------------------------------------------ the application
// FlowSender::Write: the messages due join the stream (the last one closes it, with FIN); the send
// is deferred a step as Socket::Send defers SendPendingData (reference: src/step.cuh:2118-2144)
TB_D void app_write(HostCtx &c, int f, SndRec &S, int64_t now)
{
    if (S.m_wr >= S.m_due)
        return;
    MsgRec *M = c.s->msgs + S.m_first;
    for (; S.m_wr < S.m_due; S.m_wr++)
    {
        M[S.m_wr].est = now;
        S.tail = M[S.m_wr].end;
    }
    if (S.fin_on && S.m_wr == S.m_cnt)
        S.fin |= FIN_CLOSE;
    if (S.cwnd <= inflight(S) || S.syn_at >= 0)
        return;
    S.syn_at = now + 1;
    chain_child(S.schain, c.ech, CODE_STEP);
    timer_in_slot(c, now + 1, f, 2);
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
// a message's start time: the connection's first message opens it (SYN, the connection timeout
// armed), a later one is written to the stream if the connection is up
TB_D void app_event(HostCtx &c, HostRec &hr, int *act_snd, int m, int64_t now)
{
    const WorldDesc &wd = *c.wd;
    const int f = c.s->msgs[m].conn;
    SndRec &S = c.s->snd[f];
    if (S.m_first != m)
    {
        chain_msg_root(c.ech, m - wd.msg0);
        S.m_due++;
        if (S.st == S_EST)
            app_write(c, f, S, now);
        return;
    }
    chain_app_root(c.ech, hr.local, f - wd.conn0);
    S.m_due = 1;
    add_active(*c.s, act_snd, hr.n_snd, f, c.ovf);
    S.st = S_SYN_SENT;
    if (c.cubic)
        cubic::new_round(S, now);
    S.rto = CONN_TO_PS;
    S.syn_at = now + CONN_TO_PS;
    chain_child(S.rchain, c.ech, code_lead(CONN_TO_PS));
    S.timing_time = now;
    emit_snd(c, f, S, F_SYN, 0, SYN_LEN, now);
}

// ------------------------------------------------------------------ timers and frames
// a timer of the slot fires if it is still the one armed (reference: src/step.cuh:2380-2440)
TB_D void timer_event(HostCtx &c, const Due &d, int64_t now)
{
    const Sim &s = *c.s;
    const int f = d.flow;
    if (d.kind == 0 || d.kind == 2)
    {
        SndRec &S = s.snd[f];
        if (d.kind == 0)
        {
            if (S.rto_at == d.at)
                on_rto(c, f, S, now);
            return;
        }
        if (S.syn_at != d.at)
            return;
        if (S.st == S_EST)
        {
            S.syn_at = -1; // the deferred SendPendingData
            send_pending(c, f, S, now);
        }
        else if (S.st == S_SYN_SENT)
        {
            // the SYN again, the connection timeout doubled
            S.rto = CONN_TO_PS << ++S.syn_tries;
            S.syn_at = now + S.rto;
            chain_child(S.rchain, c.ech, code_lead(S.rto));
            emit_snd(c, f, S, F_SYN, 0, SYN_LEN, now);
        }
        return;
    }
    RcvRec &R = s.rcv[f];
    switch (d.kind)
    {
    case 1: // delayed ACK
        if (R.delack_at != d.at)
            return;
        R.delack_at = -1;
        R.reserved = 1;
        rcv_ack(c, f, R, R.rcv_nxt, ECHO_AS_STATE, now);
        return;
    case 3: // SYN-ACK again
        if (R.syn_at != d.at || R.est)
            return;
        R.syn_at = -1;
        send_synack(c, f, R, now);
        return;
    case 4: // LastAckTimeout: the FIN+ACK again, a limited number of times
        if (R.last_at != d.at || R.st != R_LAST_ACK)
            return;
        if (!R.last_n)
        {
            rcv_closed(R);
            return;
        }
        R.last_n--;
        send_fin_ack(c, f, R, now);
        arm_last_ack(c, R, now);
        return;
    default: // the FIN+ACK's own retransmission
        if (R.frx_at != d.at || R.st != R_LAST_ACK)
            return;
        R.frx_at = -1;
        send_fin_ack(c, f, R, now);
    }
}

// a frame at its destination host: at the sender a SYN-ACK (connected: ACK, then the application's
// write), an ACK, or the receiver's FIN+ACK (TIME_WAIT after its ACK); at the receiver a SYN (the
// SYN-ACK, the fork's ScheduleNow), data or FIN, or the handshake's ACK (reference: src/step.cuh:2147-2236)
TB_D void on_frame(HostCtx &c, HostRec &hr, const Frame &p, int64_t now)
{
    const Sim &s = *c.s;
    const int f = (int)p.flow;
    if (p.to_sender)
    {
        SndRec &S = s.snd[f];
        if (p.flags & F_SYN)
        {
            if (S.st != S_SYN_SENT)
                return;
            S.st = S_EST;
            S.syn_at = -1;
            rtt_update(S, now - S.timing_time);
            emit_snd(c, f, S, F_ACK, 0, CTRL_LEN, now);
            chain_child(c.ech, c.ech, CODE_NOW); // (ConnectionSucceeded is ScheduleNow'd)
            app_write(c, f, S, now);
            return;
        }
        if (S.fin & FIN_TW)
            return;
        snd_ecn(c, S, p);
        on_ack(c, f, S, p.sa, p.flags & F_ECE, now);
        if (p.flags & F_FIN)
        {
            S.fin |= FIN_TW;
            emit_snd(c, f, S, F_ACK, 1, CTRL_LEN, now);
        }
        return;
    }
    RcvRec &R = s.rcv[f];
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
        c.nic.kicked = now; // (the SYN's arrival ScheduleNow's CompleteFork)
        chain_child(c.ech, c.ech, CODE_NOW);
        send_synack(c, f, R, now);
        return;
    }
    if (R.up && R.srtt < 0 && R.synack_t >= 0)
    {
        // the receiver's first sample: from its SYN-ACK to the next frame of the connection
        R.srtt = now - R.synack_t;
        R.rttvar = R.srtt / 2;
    }
    if (p.flags & (F_DATA | F_FIN))
        on_data(c, f, R, p, now);
    else if (R.up && R.st != R_CLOSED)
    {
        rcv_ecn(c, f, R, p, now);
        rcv_established(R);
        if (R.st == R_LAST_ACK)
            rcv_closed(R);
    }
}

} // namespace tb
