// TEST INFRASTRUCTURE — the oracle (see tcp_oracle.h). A sequential CPU restatement of the
// reference TwiNS TCP slot model. Every function cites the reference file:line it restates
// (paths relative to the reference project).
#include "tcp_oracle.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <map>
#include <sstream>

namespace oracle
{
namespace
{

// ------------------------------------------------------------------ constants (src/model.h:22-48)
constexpr int64_t SLOT = 1000000;       // 1 us, the link delay and the lookahead
constexpr int64_t PROP = 1000000;
constexpr int64_t PS_PER_BYTE = 80;     // 100 Gbps
constexpr uint32_t MSS = 1460;
constexpr int HDR = 42;                 // IPv4 + TCP headers + PPP
constexpr int CTRL_LEN = 42, SYN_LEN = 46;
constexpr int64_t MIN_RTO = 1000000000, DELACK_T = 10000000, CONN_TO = 10000000000, GRAN = 1000000,
                  INIT_RTT = 100000000;
constexpr uint32_t DELACK_COUNT = 2, INIT_CWND = 10 * MSS;
constexpr uint32_t DUPTHRESH = 3;
constexpr int DATA_RETRIES = 6;
constexpr double DCTCP_G = 0.0625;

constexpr uint8_t F_ACK = 1, F_SYN = 2, F_ECE = 4, F_ECT = 8, F_CE = 16, F_DATA = 32, F_CWR = 64, F_FIN = 128;
constexpr uint8_t IT_SACKED = 1, IT_LOST = 2, IT_RETX = 4;
constexpr uint8_t FIN_CLOSE = 1, FIN_SENT = 2, FIN_ACKED = 4, FIN_TW = 8;
enum : uint8_t { S_IDLE = 0, S_SYN_SENT, S_EST, S_DONE };
enum : uint8_t { C_OPEN = 0, C_DISORDER, C_CWR, C_RECOVERY, C_LOSS };
enum : uint8_t { E_IDLE = 0, E_CE_RCVD, E_SENDING_ECE, E_ECE_RCVD, E_CWR_SENT };
enum : uint8_t { R_OPEN = 0, R_LAST_ACK, R_CLOSED };

// ------------------------------------------------------------------ ns-3 hash (src/ns3hash.h:8-47)
// MurmurHash3_x86_32 (the public algorithm), seed 0x8BADF00D as ns-3's Hash32 uses it.
uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
uint32_t murmur3_32(const uint8_t *p, int n, uint32_t seed)
{
    uint32_t h = seed;
    const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    int i = 0;
    for (; i + 4 <= n; i += 4)
    {
        uint32_t k;
        memcpy(&k, p + i, 4); // little endian
        h ^= rotl(k * c1, 15) * c2;
        h = rotl(h, 13) * 5 + 0xe6546b64u;
    }
    uint32_t k = 0;
    for (int j = n - i - 1; j >= 0; j--)
        k = (k << 8) | p[i + j];
    if (n - i)
        h ^= rotl(k * c1, 15) * c2;
    h ^= (uint32_t)n;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// the flow hash of (src IP, dst IP, TCP, sport, dport) in a 17-byte buffer (src/main.cu:695-700)
uint32_t flow_hash(uint32_t a, uint32_t b, uint16_t pa, uint16_t pb)
{
    uint8_t key[17] = {};
    key[0] = a >> 24, key[1] = a >> 16, key[2] = a >> 8, key[3] = a;
    key[4] = b >> 24, key[5] = b >> 16, key[6] = b >> 8, key[7] = b;
    key[8] = 6;
    key[9] = pa >> 8, key[10] = pa, key[11] = pb >> 8, key[12] = pb;
    return murmur3_32(key, 17, 0x8BADF00Du);
}

// ------------------------------------------------------------------ MRG32k3a (src/rng.h:29-159)
struct Rng
{
    double s[6];
};
constexpr double RM1 = 4294967087.0, RM2 = 4294944443.0, RNORM = 1.0 / (4294967087.0 + 1.0);

// RngStream::RandU01 (L'Ecuyer's published MRG32k3a in doubles)
double rand_u01(Rng &r)
{
    double *s = r.s;
    double p1 = 1403580.0 * s[1] - 810728.0 * s[0];
    int32_t k = (int32_t)(p1 / RM1);
    p1 -= k * RM1;
    if (p1 < 0.0)
        p1 += RM1;
    s[0] = s[1], s[1] = s[2], s[2] = p1;
    double p2 = 527612.0 * s[5] - 1370589.0 * s[3];
    k = (int32_t)(p2 / RM2);
    p2 -= k * RM2;
    if (p2 < 0.0)
        p2 += RM2;
    s[3] = s[4], s[4] = s[5], s[5] = p2;
    return p1 > p2 ? (p1 - p2) * RNORM : (p1 - p2 + RM1) * RNORM;
}

// UniformRandomVariable::GetInteger(0, n - 1)
uint32_t get_integer(Rng &r, uint32_t n)
{
    double u = rand_u01(r);
    return (uint32_t)(0.0 + u * ((double)(n - 1) + 1.0 - 0.0));
}

typedef unsigned __int128 u128;
struct M3
{
    uint64_t a[3][3];
};
M3 mmul(const M3 &x, const M3 &y, uint64_t m)
{
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
        {
            u128 v = 0;
            for (int t = 0; t < 3; t++)
                v += (u128)x.a[i][t] * y.a[t][j] % m;
            r.a[i][j] = (uint64_t)(v % m);
        }
    return r;
}
void mvec(const M3 &x, uint64_t v[3], uint64_t m)
{
    uint64_t r[3];
    for (int i = 0; i < 3; i++)
    {
        u128 s = 0;
        for (int t = 0; t < 3; t++)
            s += (u128)x.a[i][t] * v[t] % m;
        r[i] = (uint64_t)(s % m);
    }
    memcpy(v, r, sizeof r);
}
// v = A^(nth * 2^by) v
void advance_nth_by(M3 a, uint64_t m, uint64_t nth, int by, uint64_t v[3])
{
    for (int i = 0; i < by; i++)
        a = mmul(a, a, m);
    for (; nth; nth >>= 1)
    {
        if (nth & 1)
            mvec(a, v, m);
        a = mmul(a, a, m);
    }
}
// the state of a deterministic stream (SetStream(stream): 2^63 + stream) under RngSeed/RngRun
Rng stream_state(uint32_t seed, uint64_t stream, uint64_t run)
{
    const uint64_t m1 = 4294967087ull, m2 = 4294944443ull;
    const M3 A1 = {{{0, 1, 0}, {0, 0, 1}, {m1 - 810728, 1403580, 0}}};
    const M3 A2 = {{{0, 1, 0}, {0, 0, 1}, {m2 - 1370589, 0, 527612}}};
    uint64_t v1[3] = {seed, seed, seed}, v2[3] = {seed, seed, seed};
    uint64_t target = (1ull << 63) + stream;
    advance_nth_by(A1, m1, target, 127, v1);
    advance_nth_by(A2, m2, target, 127, v2);
    advance_nth_by(A1, m1, run, 76, v1);
    advance_nth_by(A2, m2, run, 76, v2);
    Rng r;
    for (int i = 0; i < 3; i++)
        r.s[i] = (double)v1[i], r.s[3 + i] = (double)v2[i];
    return r;
}

// ------------------------------------------------------------------ ns-3 floating point
// Time::GetSeconds() of a time in ps (src/nsmath.h:238-300): ns-3 multiplies the Q64.64 value
// of ps by int64x64_t's inverse of 10^12 (UmulByInvert) and GetDouble() sums the high and low
// words in x87 long double. This restatement uses long double itself (x86-64).
constexpr uint64_t INV_1E12_HI = 18446744ull, INV_1E12_LO = 1359701234448236304ull;
double get_seconds(int64_t ps)
{
    if (ps == 0)
        return 0.0;
    bool neg = ps < 0;
    u128 a = neg ? (u128)(-(__int128)ps) : (u128)ps;
    u128 v = a * INV_1E12_HI + ((a * INV_1E12_LO) >> 64);
    long double hi = (long double)(uint64_t)(v >> 64);
    long double lo = (long double)(uint64_t)v / 18446744073709551616.0L;
    long double r = hi;
    r += lo;
    return (double)(neg ? -r : r);
}

// ------------------------------------------------------------------ event chains (src/step.cuh:58-159)
constexpr int MAXR = 25;
int g_runs = 9; // recorded runs (9: twins, 25: twins128)

struct Chain
{
    uint16_t code[MAXR] = {};
    uint16_t cnt[MAXR] = {};
    uint16_t rhi = 0, rlo = 0; // root key
};

uint16_t code_tc(int len) { return (uint16_t)len; }
uint16_t code_arrival(int len) { return (uint16_t)(2048 + len); }
uint16_t code_lead(int64_t lead_ps)
{
    int64_t c = 4096 + lead_ps / 16000;
    return (uint16_t)(c < 0xFFFE ? c : 0xFFFE);
}
constexpr uint16_t CODE_NOW = 1, CODE_STEP = 2;

// application starts are scheduled at set-up, host by host, then by connection (step.cuh:81-87)
Chain app_root(int host, int conn)
{
    Chain c;
    c.rhi = (uint16_t)(0x8000 | (host + 1));
    c.rlo = (uint16_t)conn;
    return c;
}
// message writes are scheduled in main() before them, by message (step.cuh:89-95)
Chain msg_root(int m)
{
    Chain c;
    c.rhi = (uint16_t)(1 + (m >> 16));
    c.rlo = (uint16_t)m;
    return c;
}

// the chain of an event scheduled by `parent` with the lead `code` (chain_push, step.cuh:97-116)
Chain child(const Chain &parent, uint16_t code)
{
    Chain c = parent;
    if (parent.code[0] == code)
    {
        if (c.cnt[0] < 0xFFFF)
            c.cnt[0]++;
        return c;
    }
    for (int i = g_runs - 1; i >= 1; i--)
        c.code[i] = parent.code[i - 1], c.cnt[i] = parent.cnt[i - 1];
    c.code[0] = code;
    c.cnt[0] = 1;
    return c;
}

// < 0: a runs first; > 0: b does; 0: undecided (chain_cmp, step.cuh:123-157)
int chain_cmp(const Chain &a, const Chain &b)
{
    int ia = 0, ib = 0;
    uint32_t ra = a.cnt[0], rb = b.cnt[0];
    for (;;)
    {
        uint16_t ca = a.code[ia], cb = b.code[ib];
        if (ca == 0 && cb != 0 && a.rhi != 0)
            return -1;
        if (cb == 0 && ca != 0 && b.rhi != 0)
            return 1;
        if (ca == 0 || cb == 0)
            break;
        if (ca != cb)
            return ca > cb ? -1 : 1;
        uint32_t m = std::min(ra, rb);
        ra -= m, rb -= m;
        if (ra == 0)
        {
            if (++ia == g_runs)
                break;
            ra = a.cnt[ia];
        }
        if (rb == 0)
        {
            if (++ib == g_runs)
                break;
            rb = b.cnt[ib];
        }
    }
    uint32_t xa = (uint32_t)a.rhi << 16 | a.rlo, xb = (uint32_t)b.rhi << 16 | b.rlo;
    if (xa == 0 || xb == 0 || xa == xb)
        return 0;
    return xa < xb ? -1 : 1;
}

// ------------------------------------------------------------------ frames (src/model.h:76-88)
struct Frame
{
    int64_t ts;       // queued: enqueue time; on a link: arrival time at the next hop
    uint32_t flow;    // connection
    uint32_t sa;      // data: first byte; else the acknowledgement number
    uint16_t len;     // bytes on the wire
    int dst;          // destination host
    uint8_t flags;
    bool to_sender;
    uint16_t up;      // ECMP choice (flow hash % equal-cost uplinks)
    Chain ch;
};
uint32_t payload_of(const Frame &p) { return (p.flags & F_DATA) ? p.len - 42u : 0u; }

struct Counters
{
    uint64_t drops = 0, marks = 0, retx = 0, rtos = 0, ties = 0;
};

// ------------------------------------------------------------------ egress FIFO (src/step.cuh:163-317)
// A point-to-point device: a one-packet device queue under a RED queue disc; q holds the frames
// that have not started (the device queue's packet first).
struct Egress
{
    std::deque<Frame> q;
    int64_t link_free = 0, last_start = 0;
    Chain last; // the chain of the transmission in progress
    int red_k = 30, qcap = 200;
    // per slot
    int64_t woke = -1, idle_start = -1, slot_end = 0;
    std::vector<Frame> *out = nullptr;
    Counters *ctr = nullptr;

    void begin_slot(int64_t end, std::vector<Frame> *o)
    {
        woke = idle_start = -1;
        slot_end = end;
        out = o;
        out->clear();
    }

    // Fifo::advance (step.cuh:184-230): start every frame whose transmission begins by `until`
    void advance(int64_t until)
    {
        while (!q.empty())
        {
            const Frame &f = q.front();
            int64_t start = std::max(f.ts, link_free);
            if (start > until || start >= slot_end)
                return;
            int64_t end = start + (int64_t)f.len * PS_PER_BYTE;
            Frame o = f;
            // the parent of the start: the previous frame's TransmitComplete, unless the link
            // was idle (then the frame's enqueue event)
            if (f.ts <= link_free && link_free > last_start)
                o.ch = child(last, code_tc((int)((link_free - last_start) / PS_PER_BYTE)));
            else
                idle_start = start;
            last = o.ch;
            last_start = start;
            o.ts = end + PROP;
            out->push_back(o);
            link_free = end;
            q.pop_front();
        }
    }

    // Fifo::enqueue (step.cuh:238-316): RED (MinTh = MaxTh = K, QW = 1) on the queue disc's
    // length, which excludes the device queue's packet once ns-3's Wake has refilled it
    bool enqueue(const Frame &f, int64_t now)
    {
        advance(now);
        bool refilled = last_start < now || (woke == now && idle_start == now);
        int n = (int)q.size();
        int nq = (n > 0 && link_free > now && refilled) ? n - 1 : n;
        Frame g = f;
        g.ts = now;
        if (nq >= red_k && nq > 1)
        {
            if (g.flags & F_ECT)
            {
                g.flags |= F_CE;
                ctr->marks++;
            }
            else
            {
                ctr->drops++;
                return false;
            }
        }
        if (nq >= qcap)
        {
            ctr->drops++;
            return false;
        }
        q.push_back(g);
        return true;
    }
};

// ------------------------------------------------------------------ connections (src/model.h:118-277)
struct Item
{
    uint32_t start;
    uint8_t fl;
};
struct HistEnt
{
    uint32_t seq, cnt;
    int64_t t;
    bool retx;
};

struct Snd
{
    uint8_t st = S_IDLE, cong = C_OPEN, fin = 0;
    int m_due = 0, m_wr = 0, m_dn = 0;
    uint32_t tail = 0, una = 0, nxt = 0, high = 0;
    uint32_t cwnd = INIT_CWND, ssthresh = 0xFFFFFFFFu, dupacks = 0;
    std::vector<Item> items; // the sent list (TcpTxBuffer), an item ends where the next starts
    uint32_t sack_b = 0, lost_b = 0, rtx_b = 0, sacked_n = 0, hisack = 0;
    bool sack_seen = false;
    std::deque<HistEnt> hist; // m_history
    uint32_t recover = 0;
    bool recover_active = false, first_partial = true;
    uint32_t cwnd_cnt = 0, ack_rem = 0;
    bool cwnd_limited = false;
    uint32_t cub_cnt = 0, cub_lastmax = 0, cub_origin = 0;
    double cub_k = 0.0;
    int64_t cub_delaymin = INT64_MIN, cub_epoch = INT64_MIN;
    bool cub_found = false;
    int64_t cub_roundstart = INT64_MIN;
    uint32_t cub_endseq = 0;
    int64_t cub_lastack = INT64_MIN, cub_currrtt = INT64_MIN;
    uint32_t cub_samples = 0, cub_ackcnt = 0, cub_tcpcwnd = 0;
    int64_t ecn_echo_seq = -1, ecn_cwr_seq = -1;
    uint8_t s_ce = 0, ecn_s = E_IDLE;
    double alpha = 1.0;
    uint32_t acked_total = 0, acked_ecn = 0, next_seq = 0;
    bool next_seq_flag = false;
    int64_t srtt = -1, rttvar = 0;
    uint8_t syn_tries = 0;
    int64_t rto = MIN_RTO, rto_at = -1, timing_time = 0, syn_at = -1;
    Chain rchain, schain; // the RTO/SYN timer's chain; the deferred SendPendingData's
};

struct Rcv
{
    std::vector<std::pair<uint32_t, uint32_t>> ooo; // out-of-order blocks [s, e), sorted, disjoint
    bool up = false, est = false;
    uint8_t st = R_OPEN;
    int64_t fin_seq = -1, synack_t = -1, srtt = -1, rttvar = 0, last_at = -1;
    uint8_t last_n = 0;
    int64_t frx_at = -1;
    uint8_t syn_n = 0;
    int64_t syn_at = -1;
    uint32_t rcv_nxt = 0;
    uint8_t delack_count = 0;
    int64_t delack_at = -1;
    bool ce_state = false, prior_flag = false, reserved = false;
    uint32_t prior_rcv_nxt = 0;
    uint8_t ecn_r = E_IDLE;
    int64_t ecn_ce_seq = -1;
    Chain dchain, fchain; // delayed-ACK / SYN-ACK / LastAck timers; the FIN+ACK's retransmission
};

struct Conn
{
    int src, dst;
    uint32_t hash_data = 0, hash_ack = 0;
    int m_first = 0, m_cnt = 0;
    bool fin_on = false;
    uint64_t bytes = 0;
    Snd s;
    Rcv r;
};

struct Msg
{
    int conn, row;
    uint32_t size, end; // end: one past its last byte in the connection's stream
    int64_t start;      // ps
    int64_t est = -1, done = -1;
};

struct Due
{
    int64_t at;
    int flow;
    int kind; // 0 rto, 1 delack, 2 syn / deferred send, 3 SYN-ACK retx, 4 LastAck, 5 FIN+ACK retx
};

struct Host
{
    Egress nic;
    std::vector<int> act_snd, act_rcv;
    int pend_next = 0, pend_end = 0;
    int64_t wake = 0;
};

struct LinkMsg
{
    int64_t slot = -1;
    std::vector<Frame> f;
};

// ------------------------------------------------------------------ the world
struct World
{
    const WorldSpec &spec;
    Counters ctr;
    // topology
    TopoKind kind;
    int H = 0, S = 0, k = 0, hk = 0, L = 0, ecmp_n = 1;
    int leaves = 0, spines = 0, hpl = 0;
    std::vector<int> host_sw, host_port;      // graph
    std::vector<uint32_t> rt_off;             // graph: [epoch][S][S]
    std::vector<uint8_t> rt_n, rt_ports, port_dn;
    std::vector<int64_t> fail_t;              // ps
    int n_fail = 0;
    std::vector<int> host_in_link, sw_in_link;
    // state
    std::vector<Host> hosts;
    std::vector<Egress> ports; // [S * k]
    std::vector<Conn> conns;
    std::vector<Msg> msgs;      // connection-major
    std::vector<int> pend_msg;  // messages by (src, start, writes before starts, ...)
    std::vector<Rng> sw_rng;
    std::vector<LinkMsg> ring; // [4][L]
    bool dctcp = false, cubic = false;
    unsigned flows_done = 0;
    uint64_t host_events = 0, switch_events = 0;

    explicit World(const WorldSpec &w) : spec(w) {}

    LinkMsg &msg_at(int64_t slot, int link) { return ring[(size_t)(slot & 3) * L + link]; }
    const std::vector<Frame> *msg_of(int64_t slot, int link)
    {
        if (slot < 0)
            return nullptr;
        LinkMsg &m = msg_at(slot, link);
        return m.slot == slot ? &m.f : nullptr;
    }

    // ---------------- routing (src/step.cuh:2540-2630)
    int epoch_of(int64_t ts) const
    {
        int e = 0;
        while (e < n_fail && ts >= fail_t[e])
            e++;
        return e;
    }
    int route_up(int sw, int dst, int up, int ep) const
    {
        if (kind == TOPO_GRAPH)
        {
            int e = host_sw[dst];
            if (e == sw)
                return host_port[dst];
            size_t r = ((size_t)ep * S + sw) * S + e;
            return rt_ports[rt_off[r] + up];
        }
        if (kind == TOPO_LEAFSPINE)
        {
            if (sw < leaves)
                return dst / hpl == sw ? dst % hpl : hpl + up;
            return dst / hpl;
        }
        const int E = k * hk;
        int dst_pod = dst / (hk * hk), dst_edge = (dst / hk) % hk;
        if (sw < E)
            return (dst_pod == sw / hk && dst_edge == sw % hk) ? dst % hk : hk + up;
        if (sw < 2 * E)
            return dst_pod == (sw - E) / hk ? dst_edge : hk + up;
        return dst_pod;
    }
    int route(int sw, const Frame &p, int ep) const
    {
        if (kind == TOPO_GRAPH)
        {
            int e = host_sw[p.dst];
            if (e == sw)
                return host_port[p.dst];
            uint32_t h = p.to_sender ? conns[p.flow].hash_ack : conns[p.flow].hash_data;
            return route_up(sw, p.dst, (int)(h % rt_n[((size_t)ep * S + sw) * S + e]), ep);
        }
        return route_up(sw, p.dst, p.up, ep);
    }
    bool port_down(int sw, int q, int ep) const { return n_fail && port_dn[((size_t)ep * S + sw) * k + q]; }
    int routes_to(int sw, int dst, int ep) const
    {
        if (kind == TOPO_GRAPH)
            return host_sw[dst] == sw ? 0 : rt_n[((size_t)ep * S + sw) * S + host_sw[dst]];
        if (kind == TOPO_LEAFSPINE)
            return sw < leaves ? (dst / hpl == sw ? 0 : ecmp_n) : 1;
        const int E = k * hk;
        int dst_pod = dst / (hk * hk), dst_edge = (dst / hk) % hk;
        if (sw < E)
            return dst_pod == sw / hk && dst_edge == sw % hk ? 0 : ecmp_n;
        if (sw < 2 * E)
            return dst_pod == (sw - E) / hk ? 1 : ecmp_n;
        return 1;
    }

    // arrivals at the same instant at a switch, in ns-3's order (frame_before, step.cuh:2693-2705)
    bool frame_before(const Frame &a, const Frame &b)
    {
        if (a.len != b.len)
            return a.len > b.len;
        int c = chain_cmp(a.ch, b.ch);
        if (c == 0)
            ctr.ties++;
        return c != 0 ? c < 0 : a.flow < b.flow;
    }

    bool setup(std::string &err);
    void host_step(int h, int64_t t, unsigned &act, int64_t &wake);
    void switch_step(int sw, int64_t t, unsigned &act);
};

// ------------------------------------------------------------------ host TCP
struct HostCtx
{
    World *w;
    Host *host;
    int h;
    Chain ech; // the chain of the event being handled
    std::vector<Due> due;
    size_t di = 0;
    int64_t slot_end;
};

// due_insert (step.cuh:342-360): a timer due within this slot joins the pending ones
void due_insert(HostCtx &c, int64_t at, int f, int kind)
{
    if (at >= c.slot_end)
        return;
    size_t j = c.due.size();
    c.due.push_back({});
    while (j > c.di && c.due[j - 1].at > at)
    {
        c.due[j] = c.due[j - 1];
        j--;
    }
    c.due[j] = {at, f, kind};
}

// emit (step.cuh:368-384): a frame into the host's FIFO
void emit(HostCtx &c, int f, uint8_t flags, uint32_t seq, uint32_t ack, uint16_t len, bool to_sender, int64_t now)
{
    const Conn &C = c.w->conns[f];
    Frame fr;
    fr.ts = now;
    fr.flow = (uint32_t)f;
    fr.sa = (flags & F_DATA) ? seq : ack;
    fr.len = len;
    fr.dst = to_sender ? C.src : C.dst;
    fr.flags = flags | (c.w->dctcp ? F_ECT : 0);
    fr.to_sender = to_sender;
    fr.up = (uint16_t)((to_sender ? C.hash_ack : C.hash_data) % (uint32_t)c.w->ecmp_n);
    fr.ch = c.ech;
    c.host->nic.enqueue(fr, now);
}

// SendEmptyPacket(ACK) at the receiver (send_ack, step.cuh:387-407)
void send_ack(HostCtx &c, int f, uint32_t ack, bool force_ece, bool no_ece, int64_t now)
{
    Rcv &R = c.w->conns[f].r;
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
    emit(c, f, F_ACK | (ece ? F_ECE : 0), 0, ack, CTRL_LEN, true, now);
}

// ---- TcpTxBuffer without SACK (Reno emulation), step.cuh:409-975, on a list of items
uint32_t it_end(const Snd &S, size_t i) { return i + 1 < S.items.size() ? S.items[i + 1].start : S.high; }
uint32_t it_len(const Snd &S, size_t i) { return it_end(S, i) - S.items[i].start; }

// it_set (step.cuh:453-483): new flags, keeping the byte counters
void it_set(Snd &S, size_t i, uint8_t nf)
{
    uint8_t of = S.items[i].fl;
    if (of == nf)
        return;
    uint32_t len = it_len(S, i);
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
    S.items[i].fl = nf;
}

uint32_t tb_sent(const Snd &S) { return S.items.empty() ? 0u : S.high - S.una; }

// TcpTxBuffer::BytesInFlight (unsigned, as ns-3)
uint32_t inflight(const Snd &S) { return tb_sent(S) - (S.sack_b + S.lost_b) + S.rtx_b; }

// AddRenoSack (step.cuh:649-662): sack the first unsacked item after the head
void add_reno_sack(Snd &S)
{
    size_t i = 1 + S.sacked_n;
    while (i < S.items.size() && (S.items[i].fl & IT_SACKED))
        i++;
    if (i < S.items.size())
    {
        it_set(S, i, S.items[i].fl | IT_SACKED);
        S.sack_seen = true;
        S.hisack = S.items[i].start;
    }
}

// MarkHeadAsLost (step.cuh:672-677)
void mark_head_lost(Snd &S)
{
    if (S.items.empty())
        return;
    it_set(S, 0, (uint8_t)((S.items[0].fl & ~(IT_SACKED | IT_RETX)) | IT_LOST));
}

// ResetRenoSack + SetSentListLost(resetSack) (step.cuh:687-712)
void all_lost(Snd &S)
{
    for (auto &it : S.items)
        it.fl = IT_LOST;
    S.sack_b = 0;
    S.sacked_n = 0;
    S.rtx_b = 0;
    S.lost_b = tb_sent(S);
    S.sack_seen = false;
    S.hisack = 0;
}

// DiscardUpTo(ack) (step.cuh:716-780): returns the bytes of the items removed whole
uint32_t discard(Snd &S, uint32_t ack)
{
    uint32_t delivered = 0;
    size_t removed = 0;
    while (removed < S.items.size())
    {
        uint32_t b = S.items[removed].start, e = removed + 1 < S.items.size() ? S.items[removed + 1].start : S.high;
        if (ack >= e)
        {
            // RemoveFromCounts
            uint8_t fl = S.items[removed].fl;
            uint32_t len = e - b;
            if (fl & IT_SACKED)
                S.sack_b -= len, S.sacked_n--;
            if (fl & IT_LOST)
                S.lost_b -= len;
            if (fl & IT_RETX)
                S.rtx_b -= len;
            removed++;
            delivered += e - b;
        }
        else
        {
            if (ack > b)
            {
                uint8_t fl = S.items[removed].fl;
                uint32_t off = ack - b;
                if (fl & IT_SACKED)
                    S.sack_b -= off;
                if (fl & IT_LOST)
                    S.lost_b -= off;
                if (fl & IT_RETX)
                    S.rtx_b -= off;
                S.items[removed].start = ack;
            }
            break;
        }
    }
    S.items.erase(S.items.begin(), S.items.begin() + removed);
    S.una = ack;
    if (!S.items.empty() && (S.items[0].fl & IT_SACKED))
    {
        it_set(S, 0, (uint8_t)(S.items[0].fl & ~IT_SACKED));
        add_reno_sack(S);
        mark_head_lost(S);
    }
    if (S.hisack <= ack)
    {
        S.sack_seen = false;
        S.hisack = 0;
    }
    return delivered;
}

bool it_cand(uint8_t fl) { return (fl & (IT_LOST | IT_RETX | IT_SACKED)) == IT_LOST; }

// NextSeg without SACK (step.cuh:784-834)
bool next_seg(const Snd &S, uint32_t *seq)
{
    for (size_t i = 0; i < S.items.size(); i++)
    {
        if (!it_cand(S.items[i].fl))
            continue;
        if (!S.sack_seen || S.items[i].start < S.hisack)
        {
            *seq = S.items[i].start;
            return true;
        }
        break;
    }
    if (S.tail > S.high)
    {
        *seq = S.high;
        return true;
    }
    return false;
}

// IsLost(SND.UNA) (step.cuh:838-846)
bool head_lost(const Snd &S)
{
    if (!S.sack_seen || S.una >= S.hisack || S.items.empty())
        return false;
    return S.items[0].fl & IT_LOST;
}

size_t it_lower(const Snd &S, uint32_t seq)
{
    size_t lo = 0, hi = S.items.size();
    while (lo < hi)
    {
        size_t m = (lo + hi) / 2;
        if (S.items[m].start < seq)
            lo = m + 1;
        else
            hi = m;
    }
    return lo;
}

// IsRetransmittedDataAcked(x) (step.cuh:849-869)
bool retx_ends_at(const Snd &S, uint32_t x)
{
    if (S.items.empty() || x <= S.una || x > S.high)
        return false;
    size_t i = it_lower(S, x) - 1;
    if (it_end(S, i) != x)
        return false;
    uint8_t fl = S.items[i].fl;
    return !(fl & IT_SACKED) && (fl & IT_RETX);
}

// GetTransmittedSegment (step.cuh:874-916): merge with an unsacked successor of the same lost
// state, split to the size sent, mark retransmitted
uint32_t retransmit(Snd &S, size_t i, uint32_t num)
{
    uint32_t len = it_len(S, i);
    uint32_t sz = num;
    if (i + 1 < S.items.size())
    {
        uint8_t a = S.items[i].fl, b = S.items[i + 1].fl;
        uint32_t nlen = it_len(S, i + 1);
        if (!(b & IT_SACKED) && (a & IT_LOST) == (b & IT_LOST))
            sz = std::min(sz, len + nlen);
        else
            sz = std::min(sz, len);
    }
    else
        sz = std::min(sz, len);
    if (sz > len)
    {
        uint8_t a = S.items[i].fl, b = S.items[i + 1].fl;
        if ((a ^ b) & IT_RETX)
        {
            if (a & IT_RETX)
                it_set(S, i, (uint8_t)(a & ~IT_RETX));
            else
                it_set(S, i + 1, (uint8_t)(b & ~IT_RETX));
        }
        S.items.erase(S.items.begin() + i + 1); // the merged item keeps i's (equal) flags
        len = it_len(S, i);
    }
    if (sz < len)
        S.items.insert(S.items.begin() + i + 1, Item{S.items[i].start + sz, S.items[i].fl}); // SplitItems
    uint8_t fl = S.items[i].fl;
    if (!(fl & IT_RETX))
        it_set(S, i, fl | IT_RETX);
    return sz;
}

// CopyFromSequence (step.cuh:920-975): the segment at seq, new data or a retransmission
uint32_t tb_copy(Snd &S, uint32_t num, uint32_t seq, bool *retx, Counters &ctr)
{
    for (;;)
    {
        uint32_t avail = S.tail > seq ? S.tail - seq : 0;
        uint32_t sz = std::min(num, avail);
        if (sz == 0)
            return 0;
        if (S.high >= seq + sz)
        {
            size_t i = it_lower(S, seq);
            if (i >= S.items.size() || S.items[i].start != seq)
            {
                fprintf(stderr, "oracle: a retransmission off an item boundary\n");
                return 0;
            }
            *retx = true;
            return retransmit(S, i, sz);
        }
        if (S.high <= seq)
        {
            S.items.push_back(Item{seq, 0});
            S.high = seq + sz;
            *retx = false;
            return sz;
        }
        num = S.high - seq; // partly sent: resend the sent part
    }
    (void)ctr;
}

// UpdateRttHistory (step.cuh:1014-1045)
void rtt_history(Snd &S, uint32_t seq, uint32_t sz, bool retx, int64_t now)
{
    if (!retx)
    {
        S.hist.push_back(HistEnt{seq, sz, now, false});
        return;
    }
    for (auto &h : S.hist)
        if (seq >= h.seq && seq < h.seq + h.cnt)
        {
            h.retx = true;
            h.cnt = seq + sz - h.seq;
            return;
        }
}

// RttMeanDeviation::Measurement and the RFC 6298 RTO (step.cuh:1066-1086)
void rtt_sample(Snd &S, int64_t m)
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
    int64_t rto = est + std::max(v, GRAN);
    S.rto = std::max(rto, MIN_RTO);
}

// EstimateRtt (step.cuh:1088-1126)
void rtt_ack(Snd &S, uint32_t ack, int64_t now)
{
    if (S.hist.empty())
        return;
    const HistEnt &h = S.hist.front();
    if (!h.retx && ack >= h.seq + h.cnt)
        rtt_sample(S, now - h.t);
    while (!S.hist.empty() && S.hist.front().seq + S.hist.front().cnt <= ack)
        S.hist.pop_front();
}

// ---- TcpCubic (step.cuh:1201-1345)
constexpr double CUB_C = 0.4, CUB_BETA = 0.7;
constexpr int64_t CUB_ACK_DELTA = 2000000000, CUB_DELAY_MIN = 4000000000, CUB_DELAY_MAX = 1000000000000,
                  CUB_DELTA = 10000000000;

// double -> uint32_t as GCC/x86-64 converts it (cvttsd2si into 64 bits, then the low half)
uint32_t cub_u32(double d)
{
    int64_t v;
    if (d >= -9223372036854775808.0 && d < 9223372036854775808.0)
        v = (int64_t)d;
    else
        v = INT64_MIN; // the x86 "integer indefinite" value
    return (uint32_t)(uint64_t)v;
}

void cub_hystart_reset(Snd &S, int64_t now)
{
    S.cub_roundstart = S.cub_lastack = now;
    S.cub_endseq = S.st == S_EST ? S.high + 1 : 0;
    S.cub_currrtt = INT64_MIN;
    S.cub_samples = 0;
}

uint32_t cub_update(Snd &S, uint32_t segs, int64_t now)
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
            S.cub_k = std::pow((double)(S.cub_lastmax - seg_cwnd) / CUB_C, 1 / 3.);
            S.cub_origin = S.cub_lastmax;
        }
    }
    int64_t t = (int64_t)((uint64_t)now + (uint64_t)S.cub_delaymin - (uint64_t)S.cub_epoch);
    double ts = get_seconds(t), kk = S.cub_k;
    double offs = ts < kk ? kk - ts : ts - kk;
    uint32_t delta = cub_u32(CUB_C * std::pow(offs, 3));
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

void cub_pkts_acked(Snd &S, int64_t now)
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
            S.cub_found = true;
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
            S.cub_found = true;
    }
    if (S.cub_found)
        S.ssthresh = cwnd;
}

void cub_increase(Snd &S, uint32_t segs, uint32_t ack, int64_t now)
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
        uint32_t cnt = cub_update(S, segs, now);
        if (S.cub_cnt >= cnt)
        {
            S.cwnd += MSS;
            S.cub_cnt -= cnt;
        }
    }
}

uint32_t cub_ssthresh(Snd &S)
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

void cub_loss(Snd &S, int64_t now)
{
    S.cub_origin = 0;
    S.cub_k = 0;
    S.cub_ackcnt = 0;
    S.cub_tcpcwnd = 0;
    S.cub_delaymin = INT64_MIN;
    S.cub_found = false;
    cub_hystart_reset(S, now);
}

// ssthresh_for (step.cuh:1055-1063)
uint32_t ssthresh_for(HostCtx &c, Snd &S, uint32_t bif)
{
    if (c.w->cubic)
        return cub_ssthresh(S);
    if (c.w->dctcp)
        return (uint32_t)((1.0 - S.alpha / 2.0) * S.cwnd);
    uint32_t half = bif / 2;
    return half > 2 * MSS ? half : 2 * MSS;
}

// PktsAcked (step.cuh:1348-1381)
void pkts_acked(HostCtx &c, Snd &S, uint32_t segs, uint32_t ack, int64_t now)
{
    if (c.w->cubic)
    {
        cub_pkts_acked(S, now);
        return;
    }
    if (!c.w->dctcp)
        return;
    S.acked_total += segs * MSS;
    if (S.ecn_s == E_ECE_RCVD)
        S.acked_ecn += segs * MSS;
    if (!S.next_seq_flag)
    {
        S.next_seq = S.nxt;
        S.next_seq_flag = true;
    }
    if (ack >= S.next_seq)
    {
        double m = S.acked_total > 0 ? (double)S.acked_ecn / S.acked_total : 0.0;
        S.alpha = std::fma(1.0 - DCTCP_G, S.alpha, DCTCP_G * m); // ns-3's -march=native contraction
        S.next_seq = S.nxt;
        S.acked_total = 0;
        S.acked_ecn = 0;
    }
}

// IncreaseWindow (step.cuh:1383-1440): TcpLinuxReno (DCTCP), TcpNewReno, TcpCubic
void increase_window(HostCtx &c, Snd &S, uint32_t segs, uint32_t ack, int64_t now)
{
    if (c.w->cubic)
    {
        cub_increase(S, segs, ack, now);
        return;
    }
    uint32_t cwnd = S.cwnd, ssth = S.ssthresh;
    if (c.w->dctcp)
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

// SendDataPacket (step.cuh:1129-1172)
uint32_t send_segment(HostCtx &c, int f, uint32_t seq, uint32_t max_size, int64_t now)
{
    Conn &C = c.w->conns[f];
    Snd &S = C.s;
    bool retx = false;
    uint32_t len = tb_copy(S, max_size, seq, &retx, c.w->ctr);
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
    emit(c, f, flags, seq, 0, (uint16_t)(len + HDR), false, now);
    if (retx)
        c.w->ctr.retx++;
    if (S.rto_at < 0)
    {
        S.rto_at = now + S.rto;
        S.rchain = child(c.ech, code_lead(S.rto));
    }
    S.cwnd_limited = S.cwnd < inflight(S) + MSS;
    rtt_history(S, seq, len, retx, now);
    if (seq + len > S.high)
        S.high = seq + len;
    return len;
}

// SendPendingData (step.cuh:1175-1199)
void send_pending(HostCtx &c, int f, int64_t now)
{
    Snd &S = c.w->conns[f].s;
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
        if (!next_seg(S, &seq))
            return;
        uint32_t remaining = S.tail - seq;
        if (avail < MSS && remaining > avail)
            return;
        S.nxt = seq;
        uint32_t len = send_segment(c, f, seq, avail < MSS ? avail : MSS, now);
        if (len == 0)
            return;
        S.nxt = seq + len;
    }
}

// DoRetransmit (step.cuh:1202-1212)
void do_retransmit(HostCtx &c, int f, int64_t now)
{
    Snd &S = c.w->conns[f].s;
    uint32_t seq;
    if (!next_seg(S, &seq))
        seq = S.una;
    if (S.una >= S.tail)
        return;
    S.nxt = seq;
    send_segment(c, f, seq, MSS, now);
}

// NewAck's timer handling (step.cuh:1445-1464)
void new_ack(HostCtx &c, int f, uint32_t ack, bool reset_rto, int64_t now)
{
    Snd &S = c.w->conns[f].s;
    if (reset_rto)
    {
        int64_t est = S.srtt >= 0 ? S.srtt : INIT_RTT, v = 4 * S.rttvar;
        int64_t rto = est + std::max(v, GRAN);
        S.rto = std::max(rto, MIN_RTO);
        S.rto_at = now + S.rto;
        S.rchain = child(c.ech, code_lead(S.rto));
    }
    if (ack >= S.tail && !(S.fin & FIN_SENT))
        S.rto_at = -1;
    if (ack > S.nxt)
        S.nxt = ack;
}

// EnterRecovery (step.cuh:1467-1481)
void enter_recovery(HostCtx &c, int f, int64_t now)
{
    Snd &S = c.w->conns[f].s;
    add_reno_sack(S);
    mark_head_lost(S);
    S.recover = S.high;
    S.recover_active = true;
    S.cong = C_RECOVERY;
    S.ssthresh = ssthresh_for(c, S, inflight(S) + MSS);
    S.cwnd = S.ssthresh;
    send_segment(c, f, S.una, MSS, now);
}

// messages_acked (step.cuh:1484-1499)
void messages_acked(HostCtx &c, int f, int64_t now)
{
    Conn &C = c.w->conns[f];
    Snd &S = C.s;
    while (S.m_dn < S.m_wr && S.una >= c.w->msgs[C.m_first + S.m_dn].end)
    {
        c.w->msgs[C.m_first + S.m_dn].done = now;
        S.m_dn++;
        c.w->flows_done++;
    }
    if (S.m_dn == C.m_cnt && (!C.fin_on || (S.fin & FIN_ACKED)))
    {
        S.st = S_DONE;
        S.rto_at = -1;
    }
}

// ReceivedAck + ProcessAck (step.cuh:1502-1693)
void on_ack(HostCtx &c, int f, uint32_t ack, bool ece, int64_t now)
{
    Snd &S = c.w->conns[f].s;
    if (S.st != S_EST)
        return;
    uint32_t old = S.una;
    if (ack < old)
        return;
    rtt_ack(S, ack, now);
    bool advancing = ack > old;
    uint32_t delivered = 0;
    if (advancing)
        delivered = discard(S, ack);
    if (S.cong == C_CWR && ack > S.recover)
    {
        S.cong = C_OPEN;
        S.cwnd = S.ssthresh;
    }
    if (advancing && c.w->dctcp && ece)
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
            if (cg == C_RECOVERY)
                add_reno_sack(S);
            else if (cg == C_DISORDER)
            {
                if (S.dupacks == DUPTHRESH && (old >= S.recover || !S.recover_active))
                    enter_recovery(c, f, now);
                else if (head_lost(S))
                    enter_recovery(c, f, now);
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
            mark_head_lost(S);
            if (!retx_ends_at(S, ack + MSS))
                do_retransmit(c, f, now);
            pkts_acked(c, S, 1, ack, now);
            new_ack(c, f, ack, S.first_partial, now);
            S.first_partial = false;
        }
        else if (ack < S.recover && cg == C_LOSS)
        {
            pkts_acked(c, S, segs, ack, now);
            increase_window(c, S, segs, ack, now);
            new_ack(c, f, ack, true, now);
        }
        else if (cg == C_CWR)
        {
            pkts_acked(c, S, segs, ack, now);
            new_ack(c, f, ack, true, now);
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
                S.first_partial = true;
                segs = (ack - old) / MSS;
                pkts_acked(c, S, segs, ack, now);
                S.cong = C_OPEN;
                exited = true;
                S.dupacks = 0;
            }
            else if (cg == C_LOSS)
            {
                S.first_partial = true;
                segs = (ack - S.recover) / MSS;
                pkts_acked(c, S, segs, ack, now);
                S.cong = C_OPEN;
            }
            if (ack >= S.recover)
                S.recover_active = false;
            if (exited)
            {
                new_ack(c, f, ack, true, now);
                S.cwnd = S.ssthresh;
            }
            if (S.cong == C_OPEN)
            {
                increase_window(c, S, segs, ack, now);
                new_ack(c, f, ack, true, now);
            }
        }
    }
    // ProcessWait: the ACK of the FIN (FIN_WAIT_1 -> FIN_WAIT_2)
    if ((S.fin & FIN_SENT) && S.items.empty() && ack == S.high + 1)
        S.fin |= FIN_ACKED;
    if (advancing)
    {
        messages_acked(c, f, now);
        if (S.st == S_DONE)
            return;
    }
    send_pending(c, f, now);
}

// the retransmission timeout (on_rto, step.cuh:1695-1725)
void on_rto(HostCtx &c, int f, int64_t now)
{
    Snd &S = c.w->conns[f].s;
    S.rto_at = -1;
    if (S.st != S_EST)
        return;
    if (S.una >= S.tail)
        return;
    c.w->ctr.rtos++;
    uint32_t before = inflight(S);
    S.dupacks = 0;
    all_lost(S);
    S.recover = S.high;
    S.recover_active = true;
    int64_t r = 2 * S.rto;
    S.rto = r < 60000000000000ll ? r : 60000000000000ll;
    S.hist.clear();
    S.ssthresh = ssthresh_for(c, S, before);
    if (c.w->cubic)
        cub_loss(S, now);
    S.cong = C_LOSS;
    S.cwnd = MSS;
    send_pending(c, f, now);
}

// the receiver's SYN-ACK (send_synack, step.cuh:1729-1743)
void send_synack(HostCtx &c, int f, int64_t now)
{
    Rcv &R = c.w->conns[f].r;
    int64_t rto = CONN_TO << R.syn_n;
    R.syn_n++;
    if (R.synack_t < 0)
        R.synack_t = now;
    emit(c, f, F_SYN | F_ACK, 0, 0, SYN_LEN, true, now);
    if (R.syn_at < 0)
    {
        R.syn_at = now + rto;
        R.dchain = child(c.ech, code_lead(rto));
    }
}

void rcv_established(Rcv &R)
{
    if (!R.est)
    {
        R.est = true;
        R.syn_at = -1;
    }
}

// DCTCP's CE state machine at the receiver (ce_state, step.cuh:1756-1779)
void ce_state(HostCtx &c, int f, bool ce_now, int64_t now)
{
    Rcv &R = c.w->conns[f].r;
    if (ce_now)
    {
        if (!R.ce_state && R.reserved && R.prior_flag)
            send_ack(c, f, R.prior_rcv_nxt, false, true, now);
        R.ce_state = true;
        R.ecn_r = E_CE_RCVD;
    }
    else
    {
        if (R.ce_state && R.reserved && R.prior_flag)
            send_ack(c, f, R.prior_rcv_nxt, true, false, now);
        R.ce_state = false;
        if (R.ecn_r == E_CE_RCVD || R.ecn_r == E_SENDING_ECE)
            R.ecn_r = E_IDLE;
    }
    R.prior_flag = true;
    R.prior_rcv_nxt = R.rcv_nxt;
}

// ECN at the receiving socket (rx_ecn, step.cuh:1785-1800)
void rx_ecn(HostCtx &c, int f, const Frame &p, int64_t now)
{
    if (!c.w->dctcp)
        return;
    Rcv &R = c.w->conns[f].r;
    bool ce = p.flags & F_CE;
    if (ce && R.ecn_ce_seq < (int64_t)p.sa)
    {
        R.ecn_ce_seq = p.sa;
        R.ecn_r = E_CE_RCVD;
        ce_state(c, f, true, now);
    }
    else if (p.flags & F_ECT)
        ce_state(c, f, false, now);
}

// ECN of ACKs at the sending socket (snd_ecn, step.cuh:1806-1822)
void snd_ecn(HostCtx &c, Snd &S, const Frame &p)
{
    if (!c.w->dctcp)
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

// TcpRxBuffer::Add (rx_add, step.cuh:1827-1902): out-of-order data as sorted disjoint blocks
bool rx_add(Rcv &R, uint32_t seq, uint32_t end)
{
    uint32_t head = std::max(seq, R.rcv_nxt);
    if (head >= end)
        return false;
    auto &B = R.ooo;
    size_t n = B.size(), i = 0;
    while (i < n && B[i].second < head)
        i++;
    if (i < n && B[i].first <= head && B[i].second >= end)
        return false;
    uint32_t us = head, ue = end;
    size_t j = i;
    while (j < n && B[j].first <= ue)
    {
        us = std::min(us, B[j].first);
        ue = std::max(ue, B[j].second);
        j++;
    }
    B.erase(B.begin() + i, B.begin() + j);
    B.insert(B.begin() + i, {us, ue});
    if (head == R.rcv_nxt)
    {
        R.rcv_nxt = B[0].second;
        B.erase(B.begin());
    }
    if (R.fin_seq >= 0 && R.rcv_nxt == (uint32_t)R.fin_seq)
        R.rcv_nxt++;
    return true;
}

bool rx_finished(const Rcv &R) { return R.fin_seq >= 0 && (uint32_t)R.fin_seq < R.rcv_nxt; }

// the receiver's FIN+ACK (send_fin_ack, step.cuh:1948-1963)
void send_fin_ack(HostCtx &c, int f, int64_t now)
{
    Rcv &R = c.w->conns[f].r;
    R.delack_at = -1;
    R.delack_count = 0;
    emit(c, f, F_ACK | F_FIN, 0, R.rcv_nxt, CTRL_LEN, true, now);
    if (R.frx_at < 0)
    {
        int64_t est = R.srtt >= 0 ? R.srtt : INIT_RTT, v = 4 * R.rttvar;
        int64_t rto = std::max(est + std::max(v, GRAN), MIN_RTO);
        R.frx_at = now + rto;
        R.fchain = child(c.ech, code_lead(rto));
    }
}

int64_t last_rto(const Rcv &R)
{
    int64_t est = R.srtt >= 0 ? R.srtt : INIT_RTT, v = 4 * R.rttvar;
    return est + std::max(v, GRAN);
}

// DoPeerClose then Close (do_peer_close, step.cuh:1974-1984)
void do_peer_close(HostCtx &c, int f, int64_t now)
{
    Rcv &R = c.w->conns[f].r;
    R.st = R_LAST_ACK;
    send_fin_ack(c, f, now);
    R.last_n = DATA_RETRIES;
    int64_t lr = last_rto(R);
    R.last_at = now + lr;
    R.dchain = child(c.ech, code_lead(lr));
}

void rcv_closed(Rcv &R)
{
    R.st = R_CLOSED;
    R.last_at = -1;
    R.frx_at = -1;
    R.delack_at = -1;
}

// ReceivedData (received_data, step.cuh:1994-2036)
void received_data(HostCtx &c, int f, uint32_t seq, uint32_t len, bool fin, int64_t now)
{
    Rcv &R = c.w->conns[f].r;
    uint32_t expected = R.rcv_nxt;
    if (!rx_add(R, seq, seq + len))
    {
        send_ack(c, f, R.rcv_nxt, false, false, now);
        return;
    }
    if (expected < R.rcv_nxt && rx_finished(R) && !fin)
    {
        do_peer_close(c, f, now);
        return;
    }
    bool gap = !R.ooo.empty();
    bool filled = R.rcv_nxt > expected + len;
    if (gap || filled)
    {
        R.reserved = false;
        send_ack(c, f, R.rcv_nxt, false, false, now);
        return;
    }
    uint32_t cnt = R.delack_count + 1u;
    if (cnt >= DELACK_COUNT)
    {
        R.reserved = false;
        send_ack(c, f, R.rcv_nxt, false, false, now);
    }
    else
    {
        R.delack_count = (uint8_t)cnt;
        R.reserved = true;
        if (R.delack_at < 0)
        {
            R.delack_at = now + DELACK_T;
            R.dchain = child(c.ech, code_lead(DELACK_T));
        }
    }
}

// a data segment (or FIN) at the receiving socket (on_data, step.cuh:2040-2101)
void on_data(HostCtx &c, int f, const Frame &p, int64_t now)
{
    Rcv &R = c.w->conns[f].r;
    if (!R.up || R.st == R_CLOSED)
        return;
    uint32_t seq = p.sa, len = payload_of(p), end = seq + len;
    bool fin = p.flags & F_FIN;
    if (len > 0 && R.est && (R.st == R_LAST_ACK ? seq != R.rcv_nxt : end < R.rcv_nxt))
    {
        send_ack(c, f, R.rcv_nxt, false, true, now);
        return;
    }
    rx_ecn(c, f, p, now);
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
        received_data(c, f, seq, len, false, now);
        return;
    }
    if (seq < R.rcv_nxt)
        return;
    R.fin_seq = end;
    if (R.rcv_nxt == end)
        R.rcv_nxt++;
    if (len)
        received_data(c, f, seq, len, true, now);
    if (!rx_finished(R))
        return;
    do_peer_close(c, f, now);
}

void on_delack(HostCtx &c, int f, int64_t now)
{
    Rcv &R = c.w->conns[f].r;
    R.delack_at = -1;
    R.delack_count = 0;
    R.reserved = true;
    send_ack(c, f, R.rcv_nxt, false, false, now);
}

// FlowSender::Write + Socket::Send's one-step deferral (app_write, step.cuh:2118-2144)
void app_write(HostCtx &c, int f, int64_t now)
{
    Conn &C = c.w->conns[f];
    Snd &S = C.s;
    if (S.m_wr >= S.m_due)
        return;
    while (S.m_wr < S.m_due)
    {
        Msg &m = c.w->msgs[C.m_first + S.m_wr];
        m.est = now;
        S.tail = m.end;
        S.m_wr++;
    }
    if (C.fin_on && S.m_wr == C.m_cnt)
        S.fin |= FIN_CLOSE;
    uint32_t pipe = inflight(S);
    if (S.cwnd > pipe && S.syn_at < 0)
    {
        S.syn_at = now + 1;
        S.schain = child(c.ech, CODE_STEP);
        due_insert(c, now + 1, f, 2);
    }
}

// a frame at its destination host (on_frame, step.cuh:2147-2236)
void on_frame(HostCtx &c, const Frame &p, int64_t now)
{
    int f = (int)p.flow;
    Conn &C = c.w->conns[f];
    if (p.to_sender)
    {
        Snd &S = C.s;
        if (p.flags & F_SYN)
        {
            if (S.st == S_SYN_SENT)
            {
                S.st = S_EST;
                S.syn_at = -1;
                rtt_sample(S, now - S.timing_time);
                emit(c, f, F_ACK, 0, 0, CTRL_LEN, false, now);
                c.ech = child(c.ech, CODE_NOW); // ConnectionSucceeded (ScheduleNow)
                app_write(c, f, now);
            }
        }
        else if (p.flags & F_FIN)
        {
            if (S.fin & FIN_TW)
                return;
            snd_ecn(c, S, p);
            on_ack(c, f, p.sa, p.flags & F_ECE, now);
            S.fin |= FIN_TW;
            emit(c, f, F_ACK, 0, 1, CTRL_LEN, false, now);
        }
        else
        {
            if (S.fin & FIN_TW)
                return;
            snd_ecn(c, S, p);
            on_ack(c, f, p.sa, p.flags & F_ECE, now);
        }
        return;
    }
    Rcv &R = C.r;
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
            R.up = true;
            R.delack_count = DELACK_COUNT;
            c.host->act_rcv.push_back(f);
        }
        if (R.est)
            return;
        c.host->nic.woke = now; // CompleteFork is ScheduleNow'd by the SYN's arrival
        c.ech = child(c.ech, CODE_NOW);
        send_synack(c, f, now);
    }
    else if (p.flags & (F_DATA | F_FIN))
        on_data(c, f, p, now);
    else if (R.up && R.st != R_CLOSED)
    {
        rx_ecn(c, f, p, now);
        rcv_established(R);
        if (R.st == R_LAST_ACK)
            rcv_closed(R);
    }
}

// the chain of a timer (due_chain, step.cuh:2241-2247)
const Chain &due_chain(const World &w, const Due &d)
{
    const Conn &C = w.conns[d.flow];
    switch (d.kind)
    {
    case 1:
    case 3:
    case 4:
        return C.r.dchain;
    case 5:
        return C.r.fchain;
    case 2:
        return C.s.st == S_EST ? C.s.schain : C.s.rchain;
    default:
        return C.s.rchain;
    }
}

bool timer_before_arrival(World &w, const Due &d, const Frame &p)
{
    Chain arr = child(p.ch, code_arrival(p.len));
    int r = chain_cmp(due_chain(w, d), arr);
    if (r == 0)
        w.ctr.ties++;
    return r <= 0;
}

bool rcv_idle_for_good(const Conn &C)
{
    const Rcv &R = C.r;
    if (R.delack_at >= 0 || R.syn_at >= 0 || R.last_at >= 0 || R.frx_at >= 0)
        return false;
    if (C.fin_on)
        return R.st == R_CLOSED;
    return R.est && R.rcv_nxt >= C.bytes;
}

} // namespace

// ------------------------------------------------------------------ one host, one slot
// host_step (src/step.cuh:2266-2528)
void World::host_step(int h, int64_t t, unsigned &act, int64_t &wake_out)
{
    const int64_t S0 = t * SLOT, E0 = S0 + SLOT;
    Host &hs = hosts[h];
    int link = host_in_link[h];
    // arrivals: the tail of slot t-2's message from S0 on, then the head of slot t-1's
    const std::vector<Frame> *m2 = msg_of(t - 2, link), *m1 = msg_of(t - 1, link);
    size_t i2 = 0, n2 = m2 ? m2->size() : 0, i1 = 0, n1 = m1 ? m1->size() : 0;
    while (i2 < n2 && (*m2)[i2].ts < S0)
        i2++;
    bool input = i2 < n2 || (n1 > 0 && (*m1)[0].ts < E0);
    if (!input && t < hs.wake && hs.nic.q.empty())
    {
        wake_out = hs.wake;
        return;
    }
    LinkMsg &out = msg_at(t, h);
    out.slot = t;
    hs.nic.begin_slot(E0, &out.f);
    HostCtx c{this, &hs, h, Chain(), {}, 0, E0};
    // timers due in this slot, by time (collection order among equal times)
    for (int f : hs.act_snd)
    {
        const Snd &S = conns[f].s;
        if (S.rto_at >= 0 && S.rto_at < E0)
            c.due.push_back({S.rto_at, f, 0});
        if (S.syn_at >= 0 && S.syn_at < E0)
            c.due.push_back({S.syn_at, f, 2});
    }
    for (int f : hs.act_rcv)
    {
        const Rcv &R = conns[f].r;
        if (R.delack_at >= 0 && R.delack_at < E0)
            c.due.push_back({R.delack_at, f, 1});
        if (R.syn_at >= 0 && R.syn_at < E0)
            c.due.push_back({R.syn_at, f, 3});
        if (R.last_at >= 0 && R.last_at < E0)
            c.due.push_back({R.last_at, f, 4});
        if (R.frx_at >= 0 && R.frx_at < E0)
            c.due.push_back({R.frx_at, f, 5});
    }
    std::stable_sort(c.due.begin(), c.due.end(), [](const Due &a, const Due &b) { return a.at < b.at; });
    size_t ns_before = hs.act_snd.size();
    (void)ns_before;
    int pn = hs.pend_next, pe = hs.pend_end;
    for (;;)
    {
        int64_t tr = INT64_MAX, td = INT64_MAX, tp = INT64_MAX;
        if (i2 < n2)
            tr = (*m2)[i2].ts;
        else if (i1 < n1 && (*m1)[i1].ts < E0)
            tr = (*m1)[i1].ts;
        if (c.di < c.due.size())
            td = c.due[c.di].at;
        if (pn < pe && msgs[pend_msg[pn]].start < E0)
            tp = msgs[pend_msg[pn]].start;
        int64_t now = std::min(tr, std::min(td, tp));
        if (now == INT64_MAX)
            break;
        if (now < S0)
            now = S0;
        hs.nic.advance(now);
        if (now == tp && conns[msgs[pend_msg[pn]].conn].m_first != pend_msg[pn])
        {
            // a later message of a connection (FlowSender::SendMessage)
            int m = pend_msg[pn++], f = msgs[m].conn;
            c.ech = msg_root(m);
            conns[f].s.m_due++;
            if (conns[f].s.st == S_EST)
                app_write(c, f, now);
        }
        else if (now == tp)
        {
            // a connection's application starts: SYN
            int m = pend_msg[pn++], f = msgs[m].conn;
            Snd &S = conns[f].s;
            c.ech = app_root(h, f);
            S.m_due = 1;
            hs.act_snd.push_back(f);
            S.st = S_SYN_SENT;
            if (cubic)
                cub_hystart_reset(S, now);
            S.rto = CONN_TO;
            S.syn_at = now + CONN_TO;
            S.rchain = child(c.ech, code_lead(CONN_TO));
            S.timing_time = now;
            emit(c, f, F_SYN, 0, 0, SYN_LEN, false, now);
        }
        else if (now == td && (now != tr || timer_before_arrival(*this, c.due[c.di], i2 < n2 ? (*m2)[i2] : (*m1)[i1])))
        {
            Due d = c.due[c.di++];
            c.ech = due_chain(*this, d);
            Conn &C = conns[d.flow];
            if (d.kind == 0 && C.s.rto_at == d.at)
                on_rto(c, d.flow, now);
            else if (d.kind == 1 && C.r.delack_at == d.at)
                on_delack(c, d.flow, now);
            else if (d.kind == 4 && C.r.last_at == d.at && C.r.st == R_LAST_ACK)
            {
                if (C.r.last_n == 0)
                    rcv_closed(C.r);
                else
                {
                    C.r.last_n--;
                    send_fin_ack(c, d.flow, now);
                    int64_t lr = last_rto(C.r);
                    C.r.last_at = now + lr;
                    C.r.dchain = child(c.ech, code_lead(lr));
                }
            }
            else if (d.kind == 5 && C.r.frx_at == d.at && C.r.st == R_LAST_ACK)
            {
                C.r.frx_at = -1;
                send_fin_ack(c, d.flow, now);
            }
            else if (d.kind == 3 && C.r.syn_at == d.at && !C.r.est)
            {
                C.r.syn_at = -1;
                send_synack(c, d.flow, now);
            }
            else if (d.kind == 2 && C.s.syn_at == d.at && C.s.st == S_EST)
            {
                C.s.syn_at = -1;
                send_pending(c, d.flow, now);
            }
            else if (d.kind == 2 && C.s.syn_at == d.at && C.s.st == S_SYN_SENT)
            {
                int tries = ++C.s.syn_tries;
                C.s.rto = CONN_TO << tries;
                C.s.syn_at = now + C.s.rto;
                C.s.rchain = child(c.ech, code_lead(C.s.rto));
                emit(c, d.flow, F_SYN, 0, 0, SYN_LEN, false, now);
            }
        }
        else
        {
            const Frame &p = i2 < n2 ? (*m2)[i2++] : (*m1)[i1++];
            host_events++;
            c.ech = child(p.ch, code_arrival(p.len));
            on_frame(c, p, now);
        }
    }
    hs.nic.advance(E0 - 1);
    hs.pend_next = pn;
    // drop finished connections from the active lists; the next wake-up
    int64_t next = INT64_MAX;
    {
        std::vector<int> keep;
        for (int f : hs.act_snd)
        {
            const Snd &S = conns[f].s;
            if (S.st == S_DONE)
                continue;
            keep.push_back(f);
            if (S.rto_at >= 0)
                next = std::min(next, S.rto_at);
            if (S.syn_at >= 0)
                next = std::min(next, S.syn_at);
        }
        hs.act_snd.swap(keep);
    }
    {
        std::vector<int> keep;
        for (int f : hs.act_rcv)
        {
            const Conn &C = conns[f];
            if (rcv_idle_for_good(C))
                continue;
            keep.push_back(f);
            const Rcv &R = C.r;
            for (int64_t a : {R.delack_at, R.syn_at, R.last_at, R.frx_at})
                if (a >= 0)
                    next = std::min(next, a);
        }
        hs.act_rcv.swap(keep);
    }
    if (pn < pe)
        next = std::min(next, msgs[pend_msg[pn]].start);
    hs.wake = !hs.nic.q.empty() ? t + 1 : (next == INT64_MAX ? INT64_MAX : next / SLOT);
    wake_out = hs.wake;
    if (!out.f.empty() || !hs.nic.q.empty())
        act = 1;
}

// ------------------------------------------------------------------ one switch, one slot
// switch_step (src/step.cuh:2748-2886), spray_draws (:2709-2745)
void World::switch_step(int sw, int64_t t, unsigned &act)
{
    const int64_t S0 = t * SLOT, E0 = S0 + SLOT;
    // each ingress port's frames this slot: the tail of msg[t-2], the head of msg[t-1]
    std::vector<std::vector<const Frame *>> in(k);
    for (int q = 0; q < k; q++)
    {
        int link = sw_in_link[(size_t)sw * k + q];
        if (link < 0)
            continue;
        if (const std::vector<Frame> *m2 = msg_of(t - 2, link))
            for (const Frame &f : *m2)
                if (f.ts >= S0)
                    in[q].push_back(&f);
        if (const std::vector<Frame> *m1 = msg_of(t - 1, link))
            for (const Frame &f : *m1)
            {
                if (f.ts >= E0)
                    break;
                in[q].push_back(&f);
            }
        switch_events += in[q].size();
    }
    std::vector<std::vector<int>> ups;
    const bool spray = spec.spray;
    if (spray)
    {
        // one draw per forwarded packet, in the order the packets arrive at the node
        ups.assign(k, {});
        for (int q = 0; q < k; q++)
            ups[q].assign(in[q].size(), 0);
        std::vector<size_t> pos(k, 0);
        Rng &st = sw_rng[sw];
        for (;;)
        {
            int best = -1;
            const Frame *bf = nullptr;
            for (int q = 0; q < k; q++)
            {
                if (pos[q] >= in[q].size())
                    continue;
                const Frame *f = in[q][pos[q]];
                if (best < 0 || f->ts < bf->ts || (f->ts == bf->ts && frame_before(*f, *bf)))
                {
                    best = q;
                    bf = f;
                }
            }
            if (best < 0)
                break;
            int ep = n_fail ? epoch_of(bf->ts) : 0;
            if (port_down(sw, best, ep))
            {
                pos[best]++;
                continue;
            }
            int nr = routes_to(sw, bf->dst, ep);
            ups[best][pos[best]] = nr ? (int)get_integer(st, (uint32_t)nr) : 0;
            pos[best]++;
        }
    }
    // to egress ports, in ingress order, then by (time, ns-3 order) (insertion sort)
    std::vector<std::vector<const Frame *>> eg(k);
    for (int q = 0; q < k; q++)
        for (size_t j = 0; j < in[q].size(); j++)
        {
            const Frame &p = *in[q][j];
            int ep = n_fail ? epoch_of(p.ts) : 0;
            if (port_down(sw, q, ep))
            {
                ctr.drops++;
                continue;
            }
            int e = spray ? route_up(sw, p.dst, ups[q][j], ep) : route(sw, p, ep);
            eg[e].push_back(&p);
        }
    for (int e = 0; e < k; e++)
    {
        std::vector<const Frame *> &v = eg[e];
        for (size_t i = 1; i < v.size(); i++)
        {
            const Frame *x = v[i];
            size_t j = i;
            while (j > 0 && (v[j - 1]->ts > x->ts || (v[j - 1]->ts == x->ts && frame_before(*x, *v[j - 1]))))
            {
                v[j] = v[j - 1];
                j--;
            }
            v[j] = x;
        }
        Egress &port = ports[(size_t)sw * k + e];
        int out_link = H + sw * k + e;
        LinkMsg &out = msg_at(t, out_link);
        out.slot = t;
        port.begin_slot(E0, &out.f);
        for (const Frame *x : v)
        {
            Frame p = *x;
            p.ch = child(x->ch, code_arrival(x->len));
            port.enqueue(p, p.ts);
        }
        port.advance(E0 - 1);
        if (!out.f.empty() || !port.q.empty())
            act = 1;
    }
}

// ------------------------------------------------------------------ set-up (src/main.cu:139-1015)
int hosts_of(const Topology &t)
{
    if (t.kind == TOPO_GRAPH)
        return t.g_hosts;
    if (t.kind == TOPO_LEAFSPINE)
        return t.leaves * t.hpl;
    return t.k * t.k * t.k / 4;
}

std::vector<FlowRow> load_flows(const std::string &path, int H)
{
    std::vector<FlowRow> out;
    std::ifstream in(path);
    if (!in)
        return out;
    std::string line;
    while (std::getline(in, line))
    {
        if (line.empty() || !isdigit((unsigned char)line[0]))
            continue;
        std::stringstream ss(line);
        std::string f;
        std::vector<int64_t> v;
        while (std::getline(ss, f, ','))
            v.push_back(std::stoll(f));
        if (v.size() == 3)
            out.push_back({(int)v[0], (int)((v[0] + H / 2) % H), v[1], v[2], -1});
        else if (v.size() == 4)
            out.push_back({(int)v[0], (int)v[1], v[2], v[3], -1});
        else if (v.size() >= 5)
            out.push_back({(int)v[0], (int)v[1], v[2], v[3], v[4]});
    }
    return out;
}

bool load_topofile(const std::string &path, Topology &t, std::string &err)
{
    std::ifstream in(path);
    if (!in)
    {
        err = "cannot open " + path;
        return false;
    }
    t.kind = TOPO_GRAPH;
    std::string key;
    auto node = [](const std::string &x) { return x[0] == 'h' ? std::stoi(x.substr(1)) : -1 - std::stoi(x.substr(1)); };
    while (in >> key)
    {
        if (key == "hosts")
            in >> t.g_hosts;
        else if (key == "switches")
            in >> t.g_switches;
        else if (key == "link")
        {
            std::string a, b;
            in >> a >> b;
            t.g_links.push_back({node(a), node(b)});
        }
        else
            std::getline(in, key);
    }
    return true;
}

bool parse_fail_spec(const std::string &spec, Topology &t, std::string &err)
{
    std::stringstream fs(spec);
    std::string item;
    while (std::getline(fs, item, ','))
    {
        if (item.empty())
            continue;
        std::vector<std::string> v;
        std::stringstream is(item);
        for (std::string x; std::getline(is, x, ':');)
            v.push_back(x);
        if (v.size() < 3)
        {
            err = "--fail: T:sA:sB[:up]";
            return false;
        }
        t.fails.push_back({std::stoll(v[0]), std::stoi(v[1].substr(1)), std::stoi(v[2].substr(1)), v.size() > 3 && v[3] == "up"});
    }
    return true;
}

bool World::setup(std::string &err)
{
    const Topology &T = spec.topo;
    kind = T.kind;
    dctcp = spec.cc == CC_DCTCP;
    cubic = spec.cc == CC_CUBIC;
    g_runs = spec.chain_runs;
    std::vector<std::vector<std::pair<int, int>>> adj; // graph: switch -> (port, neighbour)
    if (kind == TOPO_GRAPH)
    {
        H = T.g_hosts;
        S = T.g_switches;
        std::vector<int> deg(S, 0);
        host_sw.assign(H, -1);
        host_port.assign(H, 0);
        adj.assign(S, {});
        for (auto &l : T.g_links)
        {
            if (l.second >= 0 || (l.first >= 0 && host_sw[l.first] >= 0))
            {
                err = "hosts need exactly one link, as its first endpoint";
                return false;
            }
            int b = -1 - l.second, pb = deg[b]++;
            if (l.first >= 0)
            {
                host_sw[l.first] = b;
                host_port[l.first] = pb;
            }
            else
            {
                int a = -1 - l.first, pa = deg[a]++;
                adj[a].push_back({pa, b});
                adj[b].push_back({pb, a});
            }
        }
        for (int h = 0; h < H; h++)
            if (host_sw[h] < 0)
            {
                err = "a host has no link";
                return false;
            }
        k = 0;
        for (int d : deg)
            k = std::max(k, d);
        // link failures: the first link between two switches; epochs in time order
        struct F
        {
            int64_t t;
            int a, pa, b, pb;
            bool up;
        };
        std::vector<F> fails;
        for (const LinkFail &lf : T.fails)
        {
            F x{lf.t_ns * 1000, lf.a, -1, lf.b, -1, lf.up};
            for (auto &pn : adj[x.a])
                if (pn.second == x.b && x.pa < 0)
                    x.pa = pn.first;
            for (auto &pn : adj[x.b])
                if (pn.second == x.a && x.pb < 0)
                    x.pb = pn.first;
            if (x.pa < 0)
            {
                err = "--fail: no such link";
                return false;
            }
            fails.push_back(x);
        }
        std::stable_sort(fails.begin(), fails.end(), [](const F &x, const F &y) { return x.t < y.t; });
        n_fail = (int)fails.size();
        int NE = n_fail + 1;
        for (auto &x : fails)
            fail_t.push_back(x.t);
        rt_off.assign((size_t)NE * S * S, 0);
        rt_n.assign((size_t)NE * S * S, 0);
        port_dn.assign((size_t)NE * S * k, 0);
        std::vector<uint8_t> dn((size_t)S * k, 0);
        for (int ep = 0; ep < NE; ep++)
        {
            if (ep > 0)
            {
                const F &x = fails[ep - 1];
                dn[(size_t)x.a * k + x.pa] = dn[(size_t)x.b * k + x.pb] = x.up ? 0 : 1;
            }
            std::copy(dn.begin(), dn.end(), port_dn.begin() + (size_t)ep * S * k);
            // BFS hop counts to every switch e; equal-cost ports towards a closer neighbour, in
            // port order (src/main.cu:420-456)
            for (int e = 0; e < S; e++)
            {
                std::vector<int> dist(S, -1), todo{e};
                dist[e] = 0;
                for (size_t i = 0; i < todo.size(); i++)
                    for (auto &pn : adj[todo[i]])
                        if (!dn[(size_t)todo[i] * k + pn.first] && dist[pn.second] < 0)
                        {
                            dist[pn.second] = dist[todo[i]] + 1;
                            todo.push_back(pn.second);
                        }
                for (int x = 0; x < S; x++)
                {
                    if (x == e)
                        continue;
                    if (dist[x] < 0)
                    {
                        err = "a switch cannot reach another";
                        return false;
                    }
                    std::vector<int> pts;
                    for (auto &pn : adj[x])
                        if (!dn[(size_t)x * k + pn.first] && dist[pn.second] == dist[x] - 1)
                            pts.push_back(pn.first);
                    std::sort(pts.begin(), pts.end());
                    size_t r = ((size_t)ep * S + x) * S + e;
                    rt_off[r] = (uint32_t)rt_ports.size();
                    rt_n[r] = (uint8_t)pts.size();
                    for (int p : pts)
                        rt_ports.push_back((uint8_t)p);
                }
            }
        }
        ecmp_n = 1;
    }
    else if (kind == TOPO_LEAFSPINE)
    {
        leaves = T.leaves, spines = T.spines, hpl = T.hpl;
        k = std::max(hpl + spines, leaves);
        H = leaves * hpl;
        S = leaves + spines;
        ecmp_n = spines;
    }
    else
    {
        k = T.k;
        H = k * k * k / 4;
        S = k * k + k * k / 4;
        ecmp_n = k / 2;
    }
    hk = k / 2;
    L = H + S * k;

    // ---- messages over connections (src/main.cu:531-648)
    const std::vector<FlowRow> &rows = spec.flows;
    const int M = (int)rows.size();
    std::vector<std::vector<int>> conn_rows;
    std::vector<int> row_conn(M);
    std::map<int64_t, int> by_id;
    for (int i = 0; i < M; i++)
    {
        const FlowRow &r = rows[i];
        if (r.src < 0 || r.src >= H || r.dst < 0 || r.dst >= H || r.src == r.dst)
        {
            err = "a flow's hosts are out of range";
            return false;
        }
        int c;
        if (r.conn < 0 || !by_id.count(r.conn))
        {
            c = (int)conn_rows.size();
            conn_rows.push_back({});
            if (r.conn >= 0)
                by_id[r.conn] = c;
        }
        else
        {
            c = by_id[r.conn];
            const FlowRow &first = rows[conn_rows[c][0]];
            if (first.src != r.src || first.dst != r.dst || r.start_ns < rows[conn_rows[c].back()].start_ns)
            {
                err = "the flows of a connection need the same hosts and later starts";
                return false;
            }
        }
        conn_rows[c].push_back(i);
        row_conn[i] = c;
    }
    const int F = (int)conn_rows.size();
    std::vector<int> mnew(M);
    msgs.clear();
    conns.assign(F, Conn());
    for (int c = 0; c < F; c++)
    {
        Conn &C = conns[c];
        const FlowRow &first = rows[conn_rows[c][0]];
        C.src = first.src;
        C.dst = first.dst;
        C.m_first = (int)msgs.size();
        C.m_cnt = (int)conn_rows[c].size();
        C.fin_on = spec.fin;
        uint64_t off = 0;
        for (int i : conn_rows[c])
        {
            off += (uint64_t)rows[i].size;
            if (off >= 0xFFFFFFFFull)
            {
                err = "a connection carries 4 GB or more";
                return false;
            }
            Msg m;
            m.conn = c;
            m.row = i;
            m.size = (uint32_t)rows[i].size;
            m.end = (uint32_t)off;
            m.start = rows[i].start_ns * 1000;
            mnew[i] = (int)msgs.size();
            msgs.push_back(m);
        }
        C.bytes = off;
    }
    // each host's application events in ns-3's order at equal times: message writes (scheduled in
    // main) before connection starts (scheduled as nodes initialize) (src/main.cu:590-612)
    {
        auto is_first = [&](int i) { return conn_rows[row_conn[i]][0] == i; };
        std::vector<int> byrow(M);
        for (int i = 0; i < M; i++)
            byrow[i] = i;
        std::stable_sort(byrow.begin(), byrow.end(), [&](int a, int b) {
            if (rows[a].src != rows[b].src)
                return rows[a].src < rows[b].src;
            if (rows[a].start_ns != rows[b].start_ns)
                return rows[a].start_ns < rows[b].start_ns;
            bool fa = is_first(a), fb = is_first(b);
            if (fa != fb)
                return !fa;
            return fa ? row_conn[a] < row_conn[b] : a < b;
        });
        pend_msg.resize(M);
        for (int i = 0; i < M; i++)
            pend_msg[i] = mnew[byrow[i]];
    }
    hosts.assign(H, Host());
    {
        int i = 0;
        for (int h = 0; h < H; h++)
        {
            hosts[h].pend_next = i;
            while (i < M && rows[msgs[pend_msg[i]].row].src == h)
                i++;
            hosts[h].pend_end = i;
        }
    }
    // ECMP hashes (src/main.cu:674-723): IPs 10.(n>>8).(n&255).1, sink port 1000, source ports
    // from 49153 in the order the host's senders bind (by start, then connection)
    {
        std::vector<int> hsub(H);
        for (int h = 0; h < H; h++)
            hsub[h] = h;
        if (kind == TOPO_GRAPH)
            for (int i = 0; i < (int)T.g_links.size(); i++)
                if (T.g_links[i].first >= 0)
                    hsub[T.g_links[i].first] = i;
        auto ip = [&](int h) { return 0x0a000001u | (uint32_t)(hsub[h] & 0xFFFF) << 8; };
        std::vector<int> byhost(F);
        for (int c = 0; c < F; c++)
            byhost[c] = c;
        std::stable_sort(byhost.begin(), byhost.end(), [&](int a, int b) {
            const FlowRow &x = rows[conn_rows[a][0]], &y = rows[conn_rows[b][0]];
            return x.src != y.src ? x.src < y.src : x.start_ns < y.start_ns;
        });
        for (int i = 0, n = 0; i < F; i++, n++)
        {
            const int c = byhost[i];
            if (i > 0 && conns[byhost[i - 1]].src != conns[c].src)
                n = 0;
            const uint16_t sport = (uint16_t)(49153 + n), dport = 1000;
            const uint32_t a = ip(conns[c].src), b = ip(conns[c].dst);
            conns[c].hash_data = flow_hash(a, b, sport, dport);
            conns[c].hash_ack = flow_hash(b, a, dport, sport);
        }
        if (spec.have_hashes)
            for (int i = 0; i < M; i++)
                if (conn_rows[row_conn[i]][0] == i)
                {
                    conns[row_conn[i]].hash_data = spec.hash_data[i];
                    conns[row_conn[i]].hash_ack = spec.hash_ack[i];
                }
    }
    // ---- ports and links (src/main.cu:807-1005)
    for (Host &h : hosts)
    {
        h.nic.red_k = spec.red_k;
        h.nic.qcap = spec.qcap;
        h.nic.ctr = &ctr;
        h.wake = 0; // every host runs the first slot
    }
    ports.assign((size_t)S * k, Egress());
    for (Egress &e : ports)
    {
        e.red_k = spec.red_k;
        e.qcap = spec.qcap;
        e.ctr = &ctr;
    }
    host_in_link.assign(H, -1);
    sw_in_link.assign((size_t)S * k, -1);
    auto sw_link = [&](int sw, int p) { return H + sw * k + p; };
    if (kind == TOPO_GRAPH)
    {
        for (int h = 0; h < H; h++)
        {
            host_in_link[h] = sw_link(host_sw[h], host_port[h]);
            sw_in_link[(size_t)host_sw[h] * k + host_port[h]] = h;
        }
        for (int x = 0; x < S; x++)
            for (auto &pn : adj[x])
            {
                int y = pn.second, nth = 0;
                for (auto &q : adj[x])
                    if (q.second == y && q.first < pn.first)
                        nth++;
                for (auto &q : adj[y])
                    if (q.second == x && nth-- == 0)
                    {
                        sw_in_link[(size_t)x * k + pn.first] = sw_link(y, q.first);
                        break;
                    }
            }
    }
    else if (kind == TOPO_LEAFSPINE)
    {
        for (int h = 0; h < H; h++)
        {
            int l = h / hpl, p = h % hpl;
            host_in_link[h] = sw_link(l, p);
            sw_in_link[(size_t)l * k + p] = h;
        }
        for (int l = 0; l < leaves; l++)
            for (int j = 0; j < spines; j++)
            {
                int sp = leaves + j;
                sw_in_link[(size_t)l * k + hpl + j] = sw_link(sp, l);
                sw_in_link[(size_t)sp * k + l] = sw_link(l, hpl + j);
            }
    }
    else
    {
        const int E = k * hk;
        for (int h = 0; h < H; h++)
        {
            int e = h / hk, p = h % hk;
            host_in_link[h] = sw_link(e, p);
            sw_in_link[(size_t)e * k + p] = h;
        }
        for (int pod = 0; pod < k; pod++)
            for (int j = 0; j < hk; j++)
            {
                int agg = E + pod * hk + j;
                for (int x = 0; x < hk; x++)
                {
                    int e2 = pod * hk + x;
                    sw_in_link[(size_t)agg * k + x] = sw_link(e2, j + hk);
                    sw_in_link[(size_t)e2 * k + j + hk] = sw_link(agg, x);
                }
            }
        for (int i = 0; i < hk; i++)
            for (int j = 0; j < hk; j++)
            {
                int core = k * k + i * hk + j;
                for (int pod = 0; pod < k; pod++)
                {
                    int agg = E + pod * hk + i;
                    sw_in_link[(size_t)core * k + pod] = sw_link(agg, j + hk);
                    sw_in_link[(size_t)agg * k + j + hk] = sw_link(core, pod);
                }
            }
    }
    ring.assign((size_t)4 * L, LinkMsg());
    if (spec.spray)
    {
        // node i's Ipv4GlobalRouting draws from stream i; switches are nodes H.. (main.cu:1006-1015)
        sw_rng.resize(S);
        for (int sw = 0; sw < S; sw++)
            sw_rng[sw] = stream_state(spec.rng_seed, (uint64_t)(H + sw), spec.rng_run);
    }
    return true;
}

// ------------------------------------------------------------------ the slot loop (src/kernel.cuh:79-112)
WorldResult run_world(const WorldSpec &spec)
{
    WorldResult res;
    World w(spec);
    std::string err;
    if (!w.setup(err))
    {
        fprintf(stderr, "oracle: %s\n", err.c_str());
        res.slots = -1;
        return res;
    }
    const unsigned M = (unsigned)w.msgs.size();
    int64_t t = 0;
    unsigned prev = 1;
    bool first = true;
    while (M > 0)
    {
        unsigned cur = first ? 1u : 0u; // no skip before the first slots have run
        first = false;
        int64_t nw = INT64_MAX;
        bool any_host = false;
        for (int h = 0; h < w.H; h++)
        {
            int64_t wk = INT64_MAX;
            w.host_step(h, t, cur, wk);
            nw = std::min(nw, wk);
            any_host = true;
        }
        for (int sw = 0; sw < w.S; sw++)
            w.switch_step(sw, t, cur);
        res.slots_run++;
        bool finish = w.flows_done >= M || t + 1 >= spec.max_slots;
        int64_t next = t + 1;
        if (cur == 0 && prev == 0 && any_host && nw > next)
            next = nw < spec.max_slots ? nw : spec.max_slots;
        prev = cur;
        t = next;
        if (finish)
            break;
    }
    res.slots = t;
    res.est_ns.assign(M, -1);
    res.done_ns.assign(M, -1);
    res.hash_data.assign(M, 0);
    res.hash_ack.assign(M, 0);
    for (const Msg &m : w.msgs)
    {
        res.est_ns[m.row] = m.est >= 0 ? m.est / 1000 : -1;
        res.done_ns[m.row] = m.done >= 0 ? m.done / 1000 : -1;
        res.hash_data[m.row] = w.conns[m.conn].hash_data;
        res.hash_ack[m.row] = w.conns[m.conn].hash_ack;
    }
    res.drops = w.ctr.drops;
    res.marks = w.ctr.marks;
    res.retx = w.ctr.retx;
    res.rtos = w.ctr.rtos;
    res.ties = w.ctr.ties;
    res.host_events = w.host_events;
    res.switch_events = w.switch_events;
    res.events = w.host_events + w.switch_events;
    res.completed = w.flows_done;
    return res;
}

} // namespace oracle
