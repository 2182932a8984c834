// twins-b200: the RDMA model's arithmetic (the HPCC fork of ns-3.17 that the reference's twins-rdma
// restates): its time and tx-time rules, the switches' ECMP hash, the INT hop words, and the
// congestion-control rate rules of DCQCN (Mellanox), HPCC and DCTCP-RDMA, as functions of a queue
// pair's rate state. Timers and event order are the caller's: each rule returns what it started.
// Plain C++ with no CUDA dependence (host and device); bit-exact with the reference's functions
// (src/rdma/rstep.cuh), which the oracle's known-answer vectors pin.
#pragma once
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define TR_HD __host__ __device__ __forceinline__
#else
#define TR_HD inline
#endif

namespace tr
{

// ------------------------------------------------------------------ time (ns-3.17)
// Seconds(x), x >= 0, in ns: ns-3.17 holds x in 64.64 fixed point (whole part, and the fraction
// truncated to 64 bits), multiplies by 10^9 exactly and keeps the whole part, which is
// floor(x) * 10^9 + floor(frac * 10^9 / 2^64) (reference: src/rdma/rstep.cuh:10-22)
TR_HD int64_t ns_seconds(double x)
{
    const double whole = floor(x);
    const uint64_t frac = (uint64_t)((x - whole) * 18446744073709551616.0);
#ifdef __CUDA_ARCH__
    const uint64_t part = __umul64hi(frac, 1000000000ull);
#else
    const uint64_t part = (uint64_t)(((unsigned __int128)frac * 1000000000ull) >> 64);
#endif
    return (int64_t)whole * 1000000000ll + (int64_t)part;
}

// a frame's transmission time at bps: Seconds(bytes * 8 / bps) in double (ns-3.17), or ns-3.36's
// integer bytes * 8 * 10^9 / bps (reference: src/rdma/rstep.cuh:24-28)
TR_HD int64_t tx_ns(uint64_t bps, uint32_t bytes) { return ns_seconds((double)bytes * 8 / (double)bps); }
TR_HD int64_t tx_ns36(uint64_t bps, uint32_t bytes) { return (int64_t)(((uint64_t)bytes * 8000000000ull) / bps); }
TR_HD int64_t tx_time(bool ns336, uint64_t bps, uint32_t bytes) { return ns336 ? tx_ns36(bps, bytes) : tx_ns(bps, bytes); }

// a queue pair's last tx time asked (PktSent and ChangeRate ask for the same rate and size in turn):
// the value again without the division
struct TxMemo
{
    uint64_t rate;
    uint32_t size;
    int64_t val;
};
TR_HD int64_t tx_time_memo(TxMemo *m, bool ns336, uint64_t bps, uint32_t bytes)
{
    if (!m)
        return tx_time(ns336, bps, bytes);
    if (m->rate != bps || m->size != bytes)
    {
        m->rate = bps;
        m->size = bytes;
        m->val = tx_time(ns336, bps, bytes);
    }
    return m->val;
}

// DataRate from a double: truncation (reference: src/rdma/rstep.cuh:152)
TR_HD uint64_t rate_of(double d) { return (uint64_t)d; }

// ------------------------------------------------------------------ addresses and ECMP
// a node's IPv4 address, 11.x.y.1 (reference: src/rdma/rstep.cuh:854)
TR_HD uint32_t node_ip(int id) { return 0x0b000001u + (uint32_t)(id / 256) * 0x10000u + (uint32_t)(id % 256) * 0x100u; }

// SwitchNode::EcmpHash: MurmurHash3 (x86, 32-bit) of three 32-bit words (source IP, destination
// IP, source port | destination port << 16), seeded with the switch's node id (reference:
// src/rdma/rstep.cuh:892-913)
TR_HD uint32_t ecmp_hash(uint32_t a, uint32_t b, uint32_t c, uint32_t seed)
{
    const uint32_t words[3] = {a, b, c};
    uint32_t h = seed;
    for (uint32_t k : words)
    {
        k *= 0xcc9e2d51u;
        k = k << 15 | k >> 17;
        k *= 0x1b873593u;
        h ^= k;
        h = h << 13 | h >> 19;
        h = h * 5 + 0xe6546b64u;
    }
    h ^= 12u; // (the key's length in bytes)
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// ------------------------------------------------------------------ INT hop words (IntHop)
// One 64-bit word per hop: the egress rate's code (3 bits: 25/50/100/200/400 Gb/s), the time
// (24 bits, ns), the bytes sent (20 bits, in units of 128 * multi) and the queue length (17 bits,
// in units of 80 * multi) (reference: src/rdma/rstep.cuh:864-891)
constexpr int MAX_HOP = 5;
TR_HD uint64_t hop_time(uint64_t h) { return h >> 3 & 0xFFFFFFull; }
TR_HD uint64_t hop_bytes(uint64_t h) { return h >> 27 & 0xFFFFFull; }
TR_HD uint32_t hop_qlen(uint64_t h) { return (uint32_t)(h >> 47); }
TR_HD uint64_t hop_rate(uint64_t h)
{
    const unsigned code = (unsigned)(h & 7);
    return code <= 4 ? 25000000000ull << code : 0;
}
TR_HD uint64_t hop_make(uint64_t time, uint64_t bytes, uint32_t qlen, uint64_t rate, uint32_t multi)
{
    uint64_t code = 4;
    for (uint64_t c = 0; c < 4; c++)
        if (rate == 25000000000ull << c)
        {
            code = c;
            break;
        }
    // (multi 1, the usual: the same quotients without a division routine)
    const uint64_t b = multi == 1 ? bytes >> 7 : bytes / (128ull * multi);
    const uint64_t q = multi == 1 ? qlen / 80u : qlen / (80u * multi);
    return code | (time & 0xFFFFFF) << 3 | (b & 0xFFFFF) << 27 | (q & 0x1FFFF) << 47;
}
// the differences of two words' counters, across one wrap
TR_HD uint64_t hop_time_delta(uint64_t now, uint64_t was)
{
    const uint64_t x = hop_time(now), y = hop_time(was);
    return x >= y ? x - y : x + (1u << 24) - y;
}
TR_HD uint64_t hop_bytes_delta(uint64_t now, uint64_t was, uint32_t multi)
{
    const uint64_t x = hop_bytes(now), y = hop_bytes(was);
    return (x >= y ? x - y : x + (1u << 20) - y) * 128 * multi;
}

// ------------------------------------------------------------------ rate state of a queue pair
struct CcParams
{
    double g;                   // EWMA gain (DCQCN, DCTCP)
    double rate_first_cnp;      // DCQCN: the rate's factor at the first CNP
    int clamp;                  // DCQCN: CLAMP_TARGET_RATE
    uint32_t rpg_threshold;     // DCQCN: FAST_RECOVERY_TIMES
    uint64_t rai, rhai, min_rate; // additive / hyper increase, floor (bps)
    uint64_t dctcp_rai;         // DCTCP_RATE_AI
    double u_target;            // HPCC
    uint32_t mi_thresh;         // HPCC
    int sample_feedback;        // HPCC
    uint32_t int_multi;         // HPCC: INT counter units
    uint32_t mtu;               // payload per packet
};

struct QpRate
{
    uint64_t rate, max_rate, target; // bps
    uint64_t snd_nxt;
    uint64_t base_rtt;              // ns
    uint32_t win;                   // bytes
    // DCQCN
    uint8_t alpha_cnp, dec_cnp, first_cnp;
    uint32_t rp_stage;
    double alpha;                   // (DCTCP's too)
    // HPCC: the rate the window follows, the increase stage, the utilisation, the hops last seen
    uint32_t last_update_seq;
    int32_t inc_stage;
    uint64_t cur_rate;
    double u;
    uint64_t hop[MAX_HOP];
    // DCTCP
    uint32_t high_seq, ecn_cnt, batch, ca_state;
};

// DCQCN timers a rule started (bits): the alpha update, the rate-decrease check, the rate increase
enum : unsigned
{
    T_ALPHA = 1,
    T_DEC = 2,
    T_RP = 4
};

// a CNP arrives (RdmaHw::cnp_received_mlx): marks both windows; the first CNP sets alpha to 1,
// cuts the rate by rate_first_cnp and starts the alpha timer (alpha_int) and the decrease check
// (dec_int + 1) (reference: src/rdma/rstep.cuh:1323-1342)
TR_HD unsigned dcqcn_cnp(QpRate &q, const CcParams &P)
{
    q.alpha_cnp = 1;
    q.dec_cnp = 1;
    if (!q.first_cnp)
        return 0;
    q.alpha = 1;
    q.alpha_cnp = 0;
    q.rate = rate_of((double)q.rate * P.rate_first_cnp);
    q.target = q.rate;
    q.first_cnp = 0;
    return T_ALPHA | T_DEC;
}

// the alpha timer (UpdateAlphaMlx): alpha <- (1 - g) alpha + g if a CNP came in the window, else
// (1 - g) alpha; it restarts (reference: src/rdma/rstep.cuh:1391-1402)
TR_HD unsigned dcqcn_alpha(QpRate &q, const CcParams &P)
{
    q.alpha = q.alpha_cnp ? fma(1 - P.g, q.alpha, P.g) : (1 - P.g) * q.alpha;
    q.alpha_cnp = 0;
    return T_ALPHA;
}

// the decrease check (CheckRateDecreaseMlx): it restarts; after a CNP the rate drops to
// rate (1 - alpha / 2) (not below min_rate), the target follows the rate first when clamping or
// past stage 0, and the increase timer starts again from stage 0 (reference:
// src/rdma/rstep.cuh:1403-1419)
TR_HD unsigned dcqcn_decrease(QpRate &q, const CcParams &P)
{
    if (!q.dec_cnp)
        return T_DEC;
    if (P.clamp || q.rp_stage != 0)
        q.target = q.rate;
    const uint64_t r = rate_of((double)q.rate * (1 - q.alpha / 2));
    q.rate = r > P.min_rate ? r : P.min_rate;
    q.rp_stage = 0;
    q.dec_cnp = 0;
    return T_DEC | T_RP;
}

// the increase timer (RateIncEventTimerMlx): it restarts; fast recovery halves the distance to the
// target, after rpg_threshold stages the target first grows by rai (at the threshold) or rhai
// (past it), capped at the NIC's rate (reference: src/rdma/rstep.cuh:1420-1434)
TR_HD unsigned dcqcn_increase(QpRate &q, const CcParams &P)
{
    if (q.rp_stage >= P.rpg_threshold)
    {
        q.target += q.rp_stage == P.rpg_threshold ? P.rai : P.rhai;
        if (q.target > q.max_rate)
            q.target = q.max_rate;
    }
    q.rate = rate_of((double)q.rate / 2) + rate_of((double)q.target / 2);
    q.rp_stage++;
    return T_RP;
}

// an ACK with sequence number seq, ECN-echo cnp (RdmaHw::HandleAckDctcp): alpha once per window of
// data, a cut by alpha / 2 once per window of marks, else additive increase once per window
// (reference: src/rdma/rstep.cuh:1344-1386)
TR_HD void dctcp_ack(QpRate &q, const CcParams &P, uint32_t seq, bool cnp)
{
    bool new_batch = false;
    q.ecn_cnt += cnp ? 1 : 0;
    if (seq > q.last_update_seq)
    {
        new_batch = true;
        if (q.last_update_seq == 0)
        {
            q.last_update_seq = (uint32_t)q.snd_nxt;
            q.batch = (uint32_t)(q.snd_nxt / P.mtu + 1);
        }
        else
        {
            const double frac = (double)q.ecn_cnt / (double)q.batch;
            q.alpha = fma(1 - P.g, q.alpha, P.g * (frac < 1.0 ? frac : 1.0));
            q.last_update_seq = (uint32_t)q.snd_nxt;
            q.ecn_cnt = 0;
            q.batch = (uint32_t)((q.snd_nxt - (uint64_t)seq) / P.mtu + 1);
        }
    }
    if (q.ca_state == 1 && seq > q.high_seq)
        q.ca_state = 0;
    if (cnp && q.ca_state == 0)
    {
        const uint64_t r = rate_of((double)q.rate * (1 - q.alpha / 2));
        q.rate = r > P.min_rate ? r : P.min_rate;
        q.ca_state = 1;
        q.high_seq = (uint32_t)q.snd_nxt;
    }
    if (q.ca_state == 0 && new_batch)
    {
        const uint64_t r = q.rate + P.dctcp_rai;
        q.rate = r < q.max_rate ? r : q.max_rate;
    }
}

// one hop's utilisation (UpdateRateHp): its tx rate over the interval between the two words plus
// the smaller queue's share of the window, both against the hop's rate
TR_HD double hpcc_hop_u(uint64_t now, uint64_t was, uint32_t multi, uint64_t max_rate, uint32_t win, uint64_t *tau_out)
{
    const uint64_t tau = hop_time_delta(now, was);
    const double duration = (double)tau * 1e-9;
    const double tx_rate = (double)(hop_bytes_delta(now, was, multi) * 8) / duration;
    const uint32_t qa = hop_qlen(now) * 80 * multi, qb = hop_qlen(was) * 80 * multi;
    const double lr = (double)hop_rate(now);
    *tau_out = tau;
    return tx_rate / lr + (double)(qa < qb ? qa : qb) * (double)max_rate / lr / (double)win;
}

// the largest hop utilisation U (the first of equal ones) and its interval of an ACK's nhop INT
// words against the hops the queue pair holds, without SAMPLE_FEEDBACK (hpcc_ack's loop)
TR_HD void hpcc_hops_u(const uint64_t *hops, int nhop, const uint64_t *held, uint32_t multi, uint64_t max_rate, uint32_t win, double *U_out,
                       uint64_t *dt_out)
{
    double U = 0;
    uint64_t dt = 0;
    for (int i = 0; i < nhop; i++)
    {
        uint64_t tau;
        const double u = hpcc_hop_u(hops[i], held[i], multi, max_rate, win, &tau);
        if (u > U)
        {
            U = u;
            dt = tau;
        }
    }
    *U_out = U;
    *dt_out = dt;
}

// HPCC's rate rule for an ACK carrying nhop INT words (RdmaHw::UpdateRateHp, one rate for the
// path): the largest hop utilisation U (the first of equal ones) and its interval dt set the EWMA
// u = (u (B - dt) + U dt) / B over the base RTT B (dt at most B); u / u_target >= 1 or mi_thresh
// increase stages give a multiplicative cut plus rai, else an additive step, within
// [min_rate, max_rate]. Returns whether the rate was set (the caller, holding the old rate, moves
// the next send: paced_after_change); the hops are stored, and the reference rate and stage too
// unless `fast` (fast react), and the last sequence number updated (reference:
// src/rdma/rstep.cuh:1208-1313)
// (pre: the hops' U and tau worked out ahead by hpcc_hops_u, when the queue pair's stored hops were
// known then; the same values the loop below gives)
TR_HD bool hpcc_ack(QpRate &q, const CcParams &P, const uint64_t *hops, int nhop, bool fast, const double *pre_u = nullptr,
                    uint64_t pre_dt = 0)
{
    const uint32_t next_seq = (uint32_t)q.snd_nxt;
    if (q.last_update_seq == 0)
    {
        q.last_update_seq = next_seq;
        for (int i = 0; i < nhop && i < MAX_HOP; i++)
            q.hop[i] = hops[i];
        return false;
    }
    bool set = false;
    if (nhop <= MAX_HOP)
    {
        double U = 0;
        uint64_t dt = 0;
        bool any = false;
        if (pre_u)
        {
            U = *pre_u;
            dt = pre_dt;
            any = nhop > 0;
            for (int i = 0; i < nhop; i++)
                q.hop[i] = hops[i];
        }
        else
            for (int i = 0; i < nhop; i++)
        {
            if (P.sample_feedback && hop_qlen(hops[i]) == 0 && fast)
                continue;
            any = true;
            uint64_t tau;
            const double u = hpcc_hop_u(hops[i], q.hop[i], P.int_multi, q.max_rate, q.win, &tau);
            if (u > U)
            {
                U = u;
                dt = tau;
            }
            q.hop[i] = hops[i];
        }
        if (any)
        {
            if (dt > q.base_rtt)
                dt = q.base_rtt;
            q.u = fma(q.u, (double)(q.base_rtt - dt), U * (double)dt) / (double)q.base_rtt;
            const double max_c = q.u / P.u_target;
            uint64_t new_rate;
            int32_t new_inc;
            if (max_c >= 1 || (uint32_t)q.inc_stage >= P.mi_thresh)
            {
                new_rate = rate_of((double)q.cur_rate / max_c) + P.rai;
                new_inc = 0;
            }
            else
            {
                new_rate = q.cur_rate + P.rai;
                new_inc = q.inc_stage + 1;
            }
            if (new_rate < P.min_rate)
                new_rate = P.min_rate;
            if (new_rate > q.max_rate)
                new_rate = q.max_rate;
            q.rate = new_rate;
            set = true;
            if (!fast)
            {
                q.cur_rate = new_rate;
                q.inc_stage = new_inc;
            }
        }
    }
    if (!fast && next_seq > q.last_update_seq)
        q.last_update_seq = next_seq;
    return set;
}

// a rate change's effect on pacing (ChangeRate): the next send moves by the difference of the last
// packet's tx times at the new and the old rate (reference: src/rdma/rstep.cuh:1198-1206)
TR_HD int64_t paced_after_change(int64_t next_avail, bool ns336, uint64_t old_rate, uint64_t new_rate, uint32_t last_pkt,
                                 TxMemo *m = nullptr)
{
    const int64_t st = tx_time_memo(m, ns336, old_rate, last_pkt);
    return next_avail + tx_time_memo(m, ns336, new_rate, last_pkt) - st;
}

} // namespace tr
