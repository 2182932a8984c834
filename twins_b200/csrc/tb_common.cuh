// twins-b200: constants, the 64-byte frame, ns-3 event-order chains and ns-3's arithmetic
// (hash, random streams, GetSeconds, pow), shared by the device kernels and the host set-up.
//
// Exactness: everything here is integer arithmetic or IEEE double arithmetic with no
// contraction (the library is built with --fmad=false; fma() is written where ns-3's
// -march=native build fuses).
#pragma once
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define TB_HD __host__ __device__ __forceinline__
#define TB_HDI __host__ __device__ inline
#define TB_D __device__ __forceinline__
#else
#define TB_HD inline
#define TB_HDI inline
#define TB_D inline
#endif

namespace tb
{

// ------------------------------------------------------------------ the model's constants
// (reference: src/model.h:22-48)
constexpr int64_t SLOT_PS = 1000000;     // slot = link propagation delay = lookahead (1 us)
constexpr int64_t PROP_PS = 1000000;
constexpr int64_t PS_PER_BYTE = 80;      // 100 Gbps
constexpr uint32_t MSS = 1460;
constexpr int HDR_BYTES = 42;            // IPv4 + TCP + PPP
constexpr int CTRL_LEN = 42, SYN_LEN = 46;
constexpr int MAX_TX = 300;              // frames one link can start in one slot (42 B frames: 297)
constexpr int NB = 4;                    // slots of link messages kept (receivers read t-1, t-2)
constexpr int64_t MIN_RTO_PS = 1000000000, DELACK_PS = 10000000, CONN_TO_PS = 10000000000,
                  GRAN_PS = 1000000, INIT_RTT_PS = 100000000;
constexpr uint32_t DELACK_COUNT = 2, INIT_CWND = 10 * MSS, DUPTHRESH = 3;
constexpr int DATA_RETRIES = 6;
constexpr double DCTCP_G = 0.0625;

constexpr uint8_t F_ACK = 1, F_SYN = 2, F_ECE = 4, F_ECT = 8, F_CE = 16, F_DATA = 32, F_CWR = 64, F_FIN = 128;
constexpr uint8_t FIN_CLOSE = 1, FIN_SENT = 2, FIN_ACKED = 4, FIN_TW = 8;
enum : uint8_t { S_IDLE = 0, S_SYN_SENT, S_EST, S_DONE };
enum : uint8_t { C_OPEN = 0, C_DISORDER, C_CWR, C_RECOVERY, C_LOSS };
enum : uint8_t { E_IDLE = 0, E_CE_RCVD, E_SENDING_ECE, E_ECE_RCVD, E_CWR_SENT };
enum : uint8_t { R_OPEN = 0, R_LAST_ACK, R_CLOSED };
enum : uint8_t { CC_NEWRENO = 0, CC_DCTCP = 1, CC_CUBIC = 2 };
enum : int { TOPO_FATTREE = 0, TOPO_LEAFSPINE = 1, TOPO_GRAPH = 2 };

// ------------------------------------------------------------------ event-order chains
// ns-3 runs simultaneous events in the order they were scheduled. Each frame and timer carries
// the run-length-encoded leads from its event back through its ancestors (newest first), then
// the root (an application start or a message write scheduled at set-up). Codes grow with the
// lead: ScheduleNow 1, the 1 ps Send deferral 2, TransmitComplete of len bytes len, an arrival
// 2048 + len, timers 4096 + lead / 16 ns (reference: src/step.cuh:58-159).
#ifndef TB_CHAIN_RUNS
#define TB_CHAIN_RUNS 9
#endif
constexpr int RUNS = TB_CHAIN_RUNS;

struct Chain
{
    uint16_t code[RUNS];
    uint16_t cnt[RUNS];
    uint16_t rhi, rlo; // root key (0: none)
};

constexpr uint16_t CODE_NOW = 1, CODE_STEP = 2;
TB_HD uint16_t code_tc(int len) { return (uint16_t)len; }
TB_HD uint16_t code_arrival(int len) { return (uint16_t)(2048 + len); }
TB_HD uint16_t code_lead(int64_t lead_ps)
{
    int64_t c = 4096 + lead_ps / 16000;
    return (uint16_t)(c < 0xFFFE ? c : 0xFFFE);
}

TB_HD void chain_clear(Chain &c)
{
    for (int i = 0; i < RUNS; i++)
        c.code[i] = 0, c.cnt[i] = 0;
    c.rhi = c.rlo = 0;
}
// an application start: host by host, then by connection (world-local ids)
TB_HD void chain_app_root(Chain &c, int host, int conn)
{
    chain_clear(c);
    c.rhi = (uint16_t)(0x8000 | (host + 1));
    c.rlo = (uint16_t)conn;
}
// a message write (FlowSender::SendMessage), scheduled in main() before the starts
TB_HD void chain_msg_root(Chain &c, int msg)
{
    chain_clear(c);
    c.rhi = (uint16_t)(1 + (msg >> 16));
    c.rlo = (uint16_t)msg;
}
// dst = the chain of an event that `parent` schedules with the lead `code`; dst may be parent
TB_HD void chain_child(Chain &dst, const Chain &parent, uint16_t code)
{
    if (parent.code[0] == code)
    {
        if (&dst != &parent)
            dst = parent;
        if (dst.cnt[0] < 0xFFFF)
            dst.cnt[0]++;
        return;
    }
    for (int i = RUNS - 1; i >= 1; i--)
    {
        dst.code[i] = parent.code[i - 1];
        dst.cnt[i] = parent.cnt[i - 1];
    }
    dst.code[0] = code;
    dst.cnt[0] = 1;
    dst.rhi = parent.rhi;
    dst.rlo = parent.rlo;
}
// < 0: a runs first, > 0: b runs first, 0: the recorded histories do not tell
TB_HDI int chain_cmp(const Chain &a, const Chain &b)
{
    int ia = 0, ib = 0;
    uint32_t ra = a.cnt[0], rb = b.cnt[0];
    for (;;)
    {
        uint16_t ca = a.code[ia], cb = b.code[ib];
        if (ca == 0 && cb != 0 && a.rhi != 0)
            return -1; // a reached its root, which precedes any other parent
        if (cb == 0 && ca != 0 && b.rhi != 0)
            return 1;
        if (ca == 0 || cb == 0)
            break;
        if (ca != cb)
            return ca > cb ? -1 : 1; // the larger lead: the earlier parent
        uint32_t m = ra < rb ? ra : rb;
        ra -= m;
        rb -= m;
        if (ra == 0)
        {
            if (++ia == RUNS)
                break;
            ra = a.cnt[ia];
        }
        if (rb == 0)
        {
            if (++ib == RUNS)
                break;
            rb = b.cnt[ib];
        }
    }
    uint32_t xa = (uint32_t)a.rhi << 16 | a.rlo, xb = (uint32_t)b.rhi << 16 | b.rlo;
    if (xa == 0 || xb == 0 || xa == xb)
        return 0;
    return xa < xb ? -1 : 1;
}

// ------------------------------------------------------------------ the frame
// 64 bytes with 9-run chains (a frame on a link, or queued at an egress port).
struct alignas(16) Frame
{
    int64_t ts;        // queued: its enqueue time; on a link: its arrival at the next hop (ps)
    uint32_t flow;     // connection (global id)
    uint32_t sa;       // data: first byte; otherwise the acknowledgement number
    uint16_t len;      // bytes on the wire
    uint16_t dst;      // destination host, world-local
    uint8_t flags;
    uint8_t to_sender; // travels to the connection's sender (ACK, SYN-ACK, FIN+ACK)
    uint16_t up;       // per-flow ECMP choice (flow hash % equal-cost uplinks)
    Chain ch;          // queued: the enqueue event's chain; on a link: the transmission start's
};
static_assert(sizeof(Frame) % 16 == 0, "frames move as 16-byte words");
constexpr int FRAME_WORDS = sizeof(Frame) / 16;

TB_HD uint32_t payload_of(const Frame &p) { return (p.flags & F_DATA) ? p.len - 42u : 0u; }

// ------------------------------------------------------------------ ns-3's Hash32
// MurmurHash3 x86_32 (the public algorithm) with ns-3's seed 0x8BADF00D.
TB_HD uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
TB_HDI uint32_t murmur3_32(const uint8_t *p, int n, uint32_t seed)
{
    uint32_t h = seed;
    const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    int i = 0;
    for (; i + 4 <= n; i += 4)
    {
        uint32_t k = (uint32_t)p[i] | (uint32_t)p[i + 1] << 8 | (uint32_t)p[i + 2] << 16 | (uint32_t)p[i + 3] << 24;
        h ^= rotl32(k * c1, 15) * c2;
        h = rotl32(h, 13) * 5 + 0xe6546b64u;
    }
    uint32_t k = 0;
    for (int j = n - i - 1; j >= 0; j--)
        k = (k << 8) | p[i + j];
    if (n - i)
        h ^= rotl32(k * c1, 15) * c2;
    h ^= (uint32_t)n;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
// the ECMP hash of a TCP connection direction: (src IP, dst IP, 6, sport, dport) in the
// 17-byte buffer ns-3's Ipv4GlobalRouting hashes (reference: src/main.cu:695-700)
TB_HDI uint32_t flow_hash(uint32_t a, uint32_t b, uint16_t pa, uint16_t pb)
{
    uint8_t key[17] = {(uint8_t)(a >> 24), (uint8_t)(a >> 16), (uint8_t)(a >> 8), (uint8_t)a,
                       (uint8_t)(b >> 24), (uint8_t)(b >> 16), (uint8_t)(b >> 8), (uint8_t)b,
                       6, (uint8_t)(pa >> 8), (uint8_t)pa, (uint8_t)(pb >> 8), (uint8_t)pb, 0, 0, 0, 0};
    return murmur3_32(key, 17, 0x8BADF00Du);
}

// ------------------------------------------------------------------ MRG32k3a (ns-3 RngStream)
struct Rng
{
    double s[6];
};
// RngStream::RandU01: every intermediate is an integer below 2^53, exact in doubles
// RngStream reduces each component as p - trunc(p / m) m, plus m if negative; with the
// division correctly rounded that is always the exact residue p mod m in [0, m). This computes
// the same residue without a division: the quotient from the reciprocal may be off by one either
// way, and the two corrections bring the (exact, integer-valued) remainder into [0, m).
TB_HD double mod_exact(double p, double m, double inv_m)
{
    double k = (double)(int64_t)(p * inv_m);
    double r = p - k * m;
    if (r < 0.0)
        r += m;
    if (r >= m)
        r -= m;
    return r;
}
TB_HDI double rand_u01(Rng &r)
{
    const double m1 = 4294967087.0, m2 = 4294944443.0, norm = 1.0 / (4294967087.0 + 1.0);
    const double inv1 = 1.0 / 4294967087.0, inv2 = 1.0 / 4294944443.0;
    double p1 = mod_exact(1403580.0 * r.s[1] - 810728.0 * r.s[0], m1, inv1);
    r.s[0] = r.s[1];
    r.s[1] = r.s[2];
    r.s[2] = p1;
    double p2 = mod_exact(527612.0 * r.s[5] - 1370589.0 * r.s[3], m2, inv2);
    r.s[3] = r.s[4];
    r.s[4] = r.s[5];
    r.s[5] = p2;
    return p1 > p2 ? (p1 - p2) * norm : (p1 - p2 + m1) * norm;
}
// UniformRandomVariable::GetInteger(0, n - 1) of an output u
TB_HDI uint32_t int_of_u01(double u, uint32_t n) { return (uint32_t)(0.0 + u * ((double)(n - 1) + 1.0 - 0.0)); }
TB_HDI uint32_t rand_int(Rng &r, uint32_t n) { return int_of_u01(rand_u01(r), n); }

// Look-ahead of the stream. Each component is a linear recurrence modulo its m
// (x_n = 1403580 x_{n-2} - 810728 x_{n-3} mod m1; y_n = 527612 y_{n-1} - 1370589 y_{n-3} mod m2) over the
// state (x_{-2}, x_{-1}, x_0, y_{-2}, y_{-1}, y_0), so the value the m-th draw from a state computes
// is a fixed combination of the three state values of its component: x_m = R_m . (x_{-2}, x_{-1}, x_0)
// mod m1, R_m = -810728 R_{m-3} + 1403580 R_{m-2} from R_{-2,-1,0} = the unit rows (likewise y).
// The table holds R_m of both components for m = 1..RNG_AHEAD; with them the draws of a slot are
// computed independently of one another, each from its place in the draw order.
constexpr int RNG_AHEAD = 384; // (a switch slot's staged arrivals at most)
constexpr uint64_t RNG_M1 = 4294967087ull, RNG_M2 = 4294944443ull;
struct RngAhead
{
    uint32_t r[RNG_AHEAD + 1][6]; // [m][x: 0..2, y: 3..5]; m = 0 unused
};
constexpr RngAhead make_rng_ahead()
{
    RngAhead t{};
    // a[c][d]: component c's coefficient of the value d steps back (d = 1, 2, 3), reduced into [0, m)
    const uint64_t mod[2] = {RNG_M1, RNG_M2};
    const uint64_t a[2][3] = {{0, 1403580, RNG_M1 - 810728}, {527612, 0, RNG_M2 - 1370589}};
    for (int c = 0; c < 2; c++)
    {
        uint64_t w[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}; // R_{m-3}, R_{m-2}, R_{m-1}
        for (int m = 1; m <= RNG_AHEAD; m++)
        {
            uint64_t nr[3] = {0, 0, 0};
            for (int e = 0; e < 3; e++)
                nr[e] = (a[c][2] * w[0][e] % mod[c] + a[c][1] * w[1][e] % mod[c] + a[c][0] * w[2][e] % mod[c]) % mod[c];
            for (int e = 0; e < 3; e++)
            {
                w[0][e] = w[1][e];
                w[1][e] = w[2][e];
                w[2][e] = nr[e];
                t.r[m][3 * c + e] = (uint32_t)nr[e];
            }
        }
    }
    return t;
}
// one component's value m draws ahead (row: R_m of that component; s: its three state values)
template <uint64_t M>
TB_HDI double rng_ahead_value(const uint32_t *row, const double *s)
{
    const uint64_t v = (uint64_t)row[0] * (uint64_t)s[0] % M + (uint64_t)row[1] * (uint64_t)s[1] % M + (uint64_t)row[2] * (uint64_t)s[2] % M;
    return (double)(v % M);
}
// the output of RandU01 from the two components' new values (its last line)
TB_HDI double u01_of(double p1, double p2)
{
    const double m1 = 4294967087.0, norm = 1.0 / (4294967087.0 + 1.0);
    return p1 > p2 ? (p1 - p2) * norm : (p1 - p2 + m1) * norm;
}

// ------------------------------------------------------------------ Time::GetSeconds()
// ns-3 multiplies the time (ps, as Q64.64) by int64x64's inverse of 10^12 (UmulByInvert:
// hi*hi + (hi*lo >> 64)) and GetDouble() adds the two 64-bit halves in x87 long double. The
// inverse is Invert(10^12) = floor(2^128 / 10^12) + 1. The x87 sum is the exact 128-bit value
// rounded to 64 significant bits (nearest even), then rounded to double.
constexpr uint64_t INV_1E12_HI = 18446744ull, INV_1E12_LO = 1359701234448236304ull;
typedef unsigned __int128 u128;

TB_HD int msb128(u128 v)
{
    uint64_t hi = (uint64_t)(v >> 64);
#if defined(__CUDA_ARCH__)
    return hi ? 127 - __clzll((long long)hi) : 63 - __clzll((long long)(uint64_t)v);
#else
    return hi ? 127 - __builtin_clzll(hi) : 63 - __builtin_clzll((uint64_t)v);
#endif
}
// v rounded to `bits` significant bits, nearest even (v != 0)
TB_HD u128 round_sig(u128 v, int bits)
{
    int m = msb128(v);
    if (m < bits)
        return v;
    int drop = m + 1 - bits;
    u128 half = (u128)1 << (drop - 1), rem = v & (((u128)1 << drop) - 1);
    v >>= drop;
    if (rem > half || (rem == half && (v & 1)))
        v += 1;
    return v << drop;
}
TB_HDI double get_seconds(int64_t ps)
{
    if (ps == 0)
        return 0.0;
    bool neg = ps < 0;
    u128 a = neg ? (u128)(-(__int128)ps) : (u128)ps;
    u128 v = a * INV_1E12_HI + ((a * INV_1E12_LO) >> 64);
    if (v == 0)
        return neg ? -0.0 : 0.0;
    v = round_sig(round_sig(v, 64), 53); // x87 sum, then the conversion to double
    int m = msb128(v);
    int shift = m > 52 ? m - 52 : 0;
    double d = (double)(uint64_t)(v >> shift); // exact: at most 53 bits
    int e2 = shift - 64;                       // value = d * 2^e2
    while (e2 > 0)
    {
        d *= 2.0;
        e2--;
    }
    while (e2 < 0)
    {
        int s = e2 < -60 ? 60 : -e2;
        uint64_t bits = (uint64_t)(1023 - s) << 52; // 2^-s
        double sc;
        memcpy(&sc, &bits, 8);
        d *= sc;
        e2 += s;
    }
    return neg ? -d : d;
}

// ------------------------------------------------------------------ pow for TcpCubic
// ns-3 calls glibc's pow, which is correctly rounded except within ~2^-64 (relative) of a
// rounding boundary. This pow is correctly rounded (to ~2^-100) by double-double arithmetic:
// x^3 as an exact product; otherwise exp(y log x) with log by the atanh series and exp by
// reduction to r / 2^10 and a Taylor series. Only x > 0 finite is used by Cubic; other inputs
// take the plain special cases. (Constants: ln 2 and 1/ln 2 split into two doubles, computed
// with exact decimal arithmetic.)
struct DD
{
    double hi, lo;
};
TB_HD double tb_fma(double a, double b, double c)
{
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return __builtin_fma(a, b, c);
#endif
}
TB_HD DD two_sum(double a, double b)
{
    double s = a + b, bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
TB_HD DD fast_two_sum(double a, double b)
{
    double s = a + b;
    return {s, b - (s - a)};
}
TB_HD DD two_prod(double a, double b)
{
    double p = a * b;
    return {p, tb_fma(a, b, -p)};
}
TB_HD DD dd_add(DD a, DD b)
{
    DD s = two_sum(a.hi, b.hi), t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}
TB_HD DD dd_mul(DD a, DD b)
{
    DD p = two_prod(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return fast_two_sum(p.hi, p.lo);
}
TB_HD DD dd_mul_d(DD a, double b)
{
    DD p = two_prod(a.hi, b);
    p.lo += a.lo * b;
    return fast_two_sum(p.hi, p.lo);
}
TB_HD DD dd_div(DD a, DD b)
{
    double q1 = a.hi / b.hi;
    DD r = dd_add(a, dd_mul_d(b, -q1));
    double q2 = r.hi / b.hi;
    r = dd_add(r, dd_mul_d(b, -q2));
    double q3 = r.hi / b.hi;
    DD q = fast_two_sum(q1, q2);
    return dd_add(q, DD{q3, 0.0});
}
TB_HD double dbl_from_bits(uint64_t b)
{
    double d;
    memcpy(&d, &b, 8);
    return d;
}
TB_HD uint64_t dbl_bits(double d)
{
    uint64_t b;
    memcpy(&b, &d, 8);
    return b;
}
// log(x) for a normal x > 0
TB_HDI DD dd_log(double x)
{
    const DD LN2 = {0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56};
    uint64_t b = dbl_bits(x);
    int e = (int)((b >> 52) & 0x7FF) - 1023;
    double m = dbl_from_bits((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull); // [1, 2)
    if (m > 1.4142135623730951)
    {
        m *= 0.5; // exact
        e += 1;
    }
    // log m = 2 atanh(s), s = (m - 1) / (m + 1); m - 1 and m + 1 are exact in double-double
    DD num = two_sum(m, -1.0), den = two_sum(m, 1.0);
    DD s = dd_div(num, den), s2 = dd_mul(s, s);
    DD sum = {0.0, 0.0}, term = s;
    for (int n = 1; n < 80; n += 2)
    {
        DD t = dd_div(term, DD{(double)n, 0.0});
        sum = dd_add(sum, t);
        if (t.hi == 0.0 || (t.hi < 0 ? -t.hi : t.hi) < 1e-34 * (sum.hi < 0 ? -sum.hi : sum.hi))
            break;
        term = dd_mul(term, s2);
    }
    DD lm = dd_mul_d(sum, 2.0);
    return dd_add(dd_mul_d(LN2, (double)e), lm);
}
// exp(z) for |z| < 700
TB_HDI DD dd_exp(DD z)
{
    const DD LN2 = {0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56};
    const double INV_LN2 = 0x1.71547652b82fep+0;
    double kf = z.hi * INV_LN2;
    kf = kf < 0 ? -(double)(int64_t)(-kf + 0.5) : (double)(int64_t)(kf + 0.5);
    DD r = dd_add(z, dd_mul_d(LN2, -kf));
    // exp(r) = exp(r / 1024)^1024
    r.hi *= 0x1p-10;
    r.lo *= 0x1p-10;
    DD sum = {1.0, 0.0}, term = {1.0, 0.0};
    for (int n = 1; n < 30; n++)
    {
        term = dd_div(dd_mul(term, r), DD{(double)n, 0.0});
        sum = dd_add(sum, term);
        if ((term.hi < 0 ? -term.hi : term.hi) < 1e-36)
            break;
    }
    for (int i = 0; i < 10; i++)
        sum = dd_mul(sum, sum);
    int k = (int)kf;
    // scale by 2^k in two steps (k within the normal range for Cubic's inputs)
    int k1 = k / 2, k2 = k - k1;
    double s1 = dbl_from_bits((uint64_t)(1023 + k1) << 52), s2 = dbl_from_bits((uint64_t)(1023 + k2) << 52);
    return DD{sum.hi * s1 * s2, sum.lo * s1 * s2};
}
TB_HDI double tb_pow(double x, double y)
{
    if (y == 0.0 || x == 1.0)
        return 1.0;
    if (!(x > 0.0) || x != x || y != y || x > 1.7e308 || x < 2.3e-308)
    {
        // outside Cubic's use: the plain special cases
        if (x == 0.0)
            return y > 0 ? 0.0 : dbl_from_bits(0x7FF0000000000000ull);
        double r = 1.0;
        if (y == 3.0)
            return x * x * x;
        return r * dbl_from_bits(0x7FF8000000000000ull);
    }
    if (y == 3.0)
    {
        // x^3 = (x^2) x with x^2 = p + e exact
        DD sq = two_prod(x, x);
        DD c1 = two_prod(sq.hi, x);
        DD c2 = two_prod(sq.lo, x);
        DD c = dd_add(c1, c2);
        return c.hi + c.lo;
    }
    DD l = dd_log(x);
    DD z = dd_mul_d(l, y);
    if (z.hi > 709.0 || z.hi < -708.0)
        return z.hi > 0 ? dbl_from_bits(0x7FF0000000000000ull) : 0.0;
    DD e = dd_exp(z);
    return e.hi + e.lo;
}

} // namespace tb
