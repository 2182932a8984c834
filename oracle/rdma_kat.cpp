// Test infrastructure, not product code: known answers of the reference's RDMA arithmetic.
//
// Built by `make -C oracle ref-rdma-kat` against the reference's own device code
// (src/rdma/rstep.cuh, compiled for the CPU with its TWINS_CPU shim, src/gpu_runtime.h), so that
// every answer below is the reference's. It prints one JSON object per case on stdout:
//   {"fn": name, ...inputs..., ...outputs...}
// with every double as the hex string of its IEEE-754 bits. tests/golden/make_rdma_kat.py turns
// the output into tests/golden/rdma_kat.json.gz, against which tests/test_rdma_cc.py checks the
// restatement in twins_b200/csrc/tr_cc.cuh.
//
// Cases: ns_seconds, tx times (ns-3.17 and ns-3.36), node addresses, ECMP hashes, INT hop words,
// HPCC's per-hop utilisation, and sequences of events on one queue pair for DCQCN (CNPs and the
// three timers), DCTCP (ACKs) and HPCC (ACKs with INT hops, fast react, sample feedback).
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <vector>

#include "rdma/rstep.cuh"

thread_local twins_dim3 threadIdx, blockIdx, blockDim, gridDim;
namespace rdma
{
// (the CPU build's island hooks: every tail node here is this process's own)
uint64_t g_tail_side = 0;
TailNode island_remote(uint64_t) { return TailNode{}; }
} // namespace rdma

namespace
{
uint64_t rng_state = 0x2545F4914F6CDD1Dull;
uint64_t next64()
{
    uint64_t z = (rng_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
uint64_t below(uint64_t n) { return next64() % n; }
double unit() { return (double)(next64() >> 11) * (1.0 / 9007199254740992.0); }

const char *hx(double d, char *buf)
{
    uint64_t b;
    memcpy(&b, &d, 8);
    snprintf(buf, 24, "0x%016llx", (unsigned long long)b);
    return buf;
}

const uint64_t RATES[5] = {25000000000ull, 50000000000ull, 100000000000ull, 200000000000ull, 400000000000ull};

void kat_time()
{
    char a[24];
    const double fixed[] = {0.0, 1e-9, 1e-6, 1.5e-6, 0.25, 1.0, 2.0 / 3.0, 1e-3 + 1e-12, 123.456789, 4096.0 / 1e11};
    for (double x : fixed)
        printf("{\"fn\":\"ns_seconds\",\"x\":\"%s\",\"ns\":%lld}\n", hx(x, a), (long long)rdma::ns_seconds(x));
    for (int i = 0; i < 200; i++)
    {
        const double x = i % 3 == 0 ? unit() * 1e-3 : i % 3 == 1 ? unit() * 10 : (double)below(1u << 30) * 1e-9;
        printf("{\"fn\":\"ns_seconds\",\"x\":\"%s\",\"ns\":%lld}\n", hx(x, a), (long long)rdma::ns_seconds(x));
    }
    for (int i = 0; i < 200; i++)
    {
        const uint64_t bps = i % 2 ? RATES[below(5)] : (1 + below(400)) * 1000000000ull + below(1000) * 1000000ull;
        const uint32_t bytes = (uint32_t)(i % 4 == 0 ? below(10000) : below(70000));
        printf("{\"fn\":\"tx\",\"bps\":%llu,\"bytes\":%u,\"ns17\":%lld,\"ns36\":%lld}\n", (unsigned long long)bps, bytes,
               (long long)rdma::tx_ns(bps, bytes), (long long)rdma::tx_ns36(bps, bytes));
    }
}

void kat_hash()
{
    for (int i = 0; i < 200; i++)
    {
        const int x = i < 100 ? (int)below(70000) : i;
        const uint32_t w0 = i % 2 ? rdma::node_ip(x) : (uint32_t)next64(), w1 = (uint32_t)next64(), w2 = (uint32_t)next64(),
                       seed = (uint32_t)below(5000);
        printf("{\"fn\":\"ecmp\",\"id\":%d,\"ip\":%u,\"w\":[%u,%u,%u],\"seed\":%u,\"h\":%u}\n", x, rdma::node_ip(x), w0, w1, w2, seed,
               rdma::ecmp_hash(w0, w1, w2, seed));
    }
}

void kat_hops()
{
    char a[24];
    for (int i = 0; i < 200; i++)
    {
        const uint32_t multi = i % 3 == 0 ? 1 : (uint32_t)(1 + below(4));
        const uint64_t rate = RATES[below(5)];
        // (odd cases: the time and byte counters wrap between the two words)
        const bool wrap = i % 2 == 1;
        const uint64_t unit_b = 128ull * multi;
        const uint64_t t0 = wrap ? (1ull << 24) * (1 + below(2)) - 1 - below(20000) : below(1ull << 25);
        const uint64_t b0 = wrap ? (1ull << 20) * unit_b * (1 + below(2)) - below(1ull << 21) : below(1ull << 30);
        const uint64_t t1 = t0 + 1 + below(20000), b1 = b0 + below(1ull << 22);
        const uint32_t q0 = (uint32_t)below(1u << 22), q1 = (uint32_t)below(1u << 22);
        const uint64_t h0 = rdma::hop_make(t0, b0, q0, rate, multi), h1 = rdma::hop_make(t1, b1, q1, rate, multi);
        rdma::Params P{};
        P.int_multi = multi;
        const uint64_t max_rate = RATES[below(5)];
        const uint32_t win = (uint32_t)(10000 + below(200000));
        double U;
        uint64_t dt;
        rdma::hpcc_hops(P, &h1, 1, &h0, max_rate, win, &U, &dt);
        printf("{\"fn\":\"hop\",\"t\":[%llu,%llu],\"b\":[%llu,%llu],\"q\":[%u,%u],\"rate\":%llu,\"multi\":%u,\"h\":[%llu,%llu],"
               "\"dtime\":%llu,\"dbytes\":%llu,\"max_rate\":%llu,\"win\":%u,\"U\":\"%s\",\"dt\":%llu}\n",
               (unsigned long long)t0, (unsigned long long)t1, (unsigned long long)b0, (unsigned long long)b1, q0, q1,
               (unsigned long long)rate, multi, (unsigned long long)h0, (unsigned long long)h1,
               (unsigned long long)rdma::hop_time_delta(h1, h0), (unsigned long long)rdma::hop_bytes_delta(h1, h0, multi),
               (unsigned long long)max_rate, win, hx(U, a), (unsigned long long)dt);
    }
}

// the rate state printed after each event
void print_state(const char *fn, int seq, int step, int ev, const rdma::SndQP &q, unsigned started, int set)
{
    char a[24], b[24];
    printf("{\"fn\":\"%s\",\"seq\":%d,\"step\":%d,\"ev\":%d,\"rate\":%llu,\"target\":%llu,\"alpha\":\"%s\",\"rp_stage\":%u,"
           "\"alpha_cnp\":%u,\"dec_cnp\":%u,\"first_cnp\":%u,\"started\":%u,\"lus\":%u,\"inc\":%d,\"cur_rate\":%llu,\"u\":\"%s\","
           "\"hop\":[%llu,%llu,%llu,%llu,%llu],\"set\":%d,\"next_avail\":%lld}\n",
           fn, seq, step, ev, (unsigned long long)q.rate, (unsigned long long)q.target, hx(q.alpha, a), q.rp_stage, q.alpha_cnp,
           q.dec_cnp, q.first_cnp, started, q.last_update_seq, q.inc_stage, (unsigned long long)q.cur_rate, hx(q.u, b),
           (unsigned long long)q.hop[0], (unsigned long long)q.hop[1], (unsigned long long)q.hop[2], (unsigned long long)q.hop[3],
           (unsigned long long)q.hop[4], set, (long long)q.next_avail);
}

struct Harness
{
    rdma::Sim s{};
    rdma::Params P{};
    rdma::SndQP qp[1]{};
    rdma::QPChains qc[1]{};
    rdma::HCtx<1> c{};
    Harness()
    {
        s.qp = qp;
        s.qc = qc;
        c.s = &s;
        c.P = &P;
        c.now = 1000000;
        c.stv[0].ns_at = -1;
        c.stv[0].due_min = INT64_MAX;
    }
    void params_line(const char *fn, int seq)
    {
        char a[24], b[24], d[24];
        printf("{\"fn\":\"%s_params\",\"seq\":%d,\"g\":\"%s\",\"rate_first_cnp\":\"%s\",\"clamp\":%d,\"rpg_threshold\":%u,"
               "\"rai\":%llu,\"rhai\":%llu,\"min_rate\":%llu,\"dctcp_rai\":%llu,\"u_target\":\"%s\",\"mi_thresh\":%u,"
               "\"sample_feedback\":%d,\"int_multi\":%u,\"mtu\":%u}\n",
               fn, seq, hx(P.g, a), hx(P.rate_first_cnp, b), P.clamp, P.rpg_threshold, (unsigned long long)P.rai,
               (unsigned long long)P.rhai, (unsigned long long)P.min_rate, (unsigned long long)P.dctcp_rai, hx(P.u_target, d),
               P.mi_thresh, P.sample_feedback, P.int_multi, P.mtu);
    }
    void qp_line(const char *fn, int seq)
    {
        const rdma::SndQP &q = qp[0];
        printf("{\"fn\":\"%s_qp\",\"seq\":%d,\"rate\":%llu,\"max_rate\":%llu,\"snd_nxt\":%llu,\"base_rtt\":%llu,\"win\":%u,"
               "\"last_pkt\":%u,\"next_avail\":%lld}\n",
               fn, seq, (unsigned long long)q.rate, (unsigned long long)q.max_rate, (unsigned long long)q.snd_nxt,
               (unsigned long long)q.base_rtt, q.win, q.last_pkt, (long long)q.next_avail);
    }
};

void kat_dcqcn()
{
    for (int seq = 0; seq < 24; seq++)
    {
        Harness H;
        H.P.g = 1.0 / (double)(16 << below(4));
        H.P.rate_first_cnp = seq % 2 ? 1.0 : 0.5 + 0.5 * unit();
        H.P.clamp = (int)below(2);
        H.P.alpha_int = 1 + (int64_t)below(100000);
        H.P.dec_int = 1 + (int64_t)below(100000);
        H.P.rp_int = 1 + (int64_t)below(100000);
        H.P.rpg_threshold = (uint32_t)(1 + below(6));
        H.P.rai = (1 + below(100)) * 1000000ull;
        H.P.rhai = (1 + below(1000)) * 1000000ull;
        H.P.min_rate = (1 + below(1000)) * 1000000ull;
        rdma::SndQP &q = H.qp[0];
        q.max_rate = RATES[below(5)];
        q.rate = q.max_rate;
        q.target = q.max_rate;
        q.first_cnp = 1;
        q.alpha = 1;
        H.params_line("dcqcn", seq);
        H.qp_line("dcqcn", seq);
        for (int step = 0; step < 16; step++)
        {
            const int ev = (int)below(4); // 0 CNP, 1 alpha timer, 2 decrease check, 3 increase timer
            q.t_alpha = q.t_dec = q.t_rp = -1;
            if (ev == 0)
                rdma::dcqcn_cnp(H.c, 0, q);
            else
                rdma::dcqcn_timer(H.c, 0, ev - 1);
            const unsigned started = (q.t_alpha >= 0 ? 1u : 0u) | (q.t_dec >= 0 ? 2u : 0u) | (q.t_rp >= 0 ? 4u : 0u);
            print_state("dcqcn", seq, step, ev, q, started, 0);
            H.c.now += 1 + (int64_t)below(50000);
        }
    }
}

void kat_dctcp()
{
    for (int seq = 0; seq < 24; seq++)
    {
        Harness H;
        H.P.g = 1.0 / (double)(16 << below(4));
        H.P.min_rate = (1 + below(1000)) * 1000000ull;
        H.P.dctcp_rai = (1 + below(1000)) * 1000000ull;
        H.P.mtu = 1000 + (uint32_t)below(8) * 500;
        rdma::SndQP &q = H.qp[0];
        q.max_rate = RATES[below(5)];
        q.rate = q.max_rate;
        q.snd_nxt = H.P.mtu * (1 + below(20));
        H.params_line("dctcp", seq);
        H.qp_line("dctcp", seq);
        uint32_t acked = 0;
        for (int step = 0; step < 16; step++)
        {
            rdma::Pkt p{};
            // the sender runs ahead; an ACK covers up to what was sent (or, after a NACK, less)
            q.snd_nxt += H.P.mtu * below(6);
            acked += (uint32_t)(H.P.mtu * below(4));
            if (acked > q.snd_nxt)
                acked = (uint32_t)q.snd_nxt;
            p.seq = step % 7 == 6 ? (uint32_t)q.snd_nxt + H.P.mtu : acked;
            p.cnp = (uint8_t)(below(3) == 0);
            rdma::dctcp_ack(H.c, q, p);
            printf("{\"fn\":\"dctcp\",\"seq\":%d,\"step\":%d,\"ack\":%u,\"cnp\":%u,\"snd_nxt\":%llu,\"rate\":%llu,\"alpha\":\"", seq, step,
                   p.seq, p.cnp, (unsigned long long)q.snd_nxt, (unsigned long long)q.rate);
            char a[24];
            printf("%s\",\"lus\":%u,\"batch\":%u,\"ecn_cnt\":%u,\"ca_state\":%u,\"high_seq\":%u}\n", hx(q.alpha, a), q.last_update_seq,
                   q.batch, q.ecn_cnt, q.ca_state, q.high_seq);
        }
    }
}

void kat_hpcc()
{
    for (int seq = 0; seq < 24; seq++)
    {
        Harness H;
        H.P.u_target = 0.95;
        H.P.mi_thresh = (uint32_t)below(6);
        H.P.rai = (1 + below(100)) * 1000000ull;
        H.P.min_rate = (1 + below(1000)) * 1000000ull;
        H.P.sample_feedback = seq % 4 == 3;
        H.P.int_multi = seq % 3 == 0 ? 1 : (uint32_t)(1 + below(4));
        H.P.mtu = 1000;
        rdma::SndQP &q = H.qp[0];
        q.max_rate = RATES[below(5)];
        q.rate = q.max_rate;
        q.cur_rate = q.max_rate;
        q.base_rtt = 2000 + below(20000);
        q.win = (uint32_t)(q.max_rate / 8 * q.base_rtt / 1000000000ull) + 1000;
        q.u = 1;
        q.last_pkt = 1048;
        q.next_avail = 5000000;
        q.snd_nxt = 1000;
        H.params_line("hpcc", seq);
        H.qp_line("hpcc", seq);
        const int nhop = 1 + (int)below(5);
        uint64_t t[5], b[5];
        uint64_t rate[5];
        for (int i = 0; i < nhop; i++)
        {
            t[i] = below(1ull << 24);
            b[i] = below(1ull << 26);
            rate[i] = RATES[below(5)];
        }
        for (int step = 0; step < 16; step++)
        {
            rdma::Pkt p{};
            p.nhop = (uint16_t)nhop;
            for (int i = 0; i < nhop; i++)
            {
                t[i] += 200 + below(4000);
                b[i] += below(rate[i] / 8 / 1000000ull * 4);
                const uint32_t ql = below(3) == 0 ? 0 : (uint32_t)below(400000);
                p.hop[i] = rdma::hop_make(t[i], b[i], ql, rate[i], H.P.int_multi);
            }
            q.snd_nxt += 1000 * below(8);
            const bool fast = below(2) == 1;
            q.tx_rate = 12345; // (change_rate leaves the new rate here: whether it ran)
            q.tx_size = 0;
            rdma::hpcc_update(H.c, q, p, fast);
            const int set = q.tx_rate != 12345;
            printf("{\"fn\":\"hpcc_ack\",\"seq\":%d,\"step\":%d,\"fast\":%d,\"nhop\":%d,\"snd_nxt\":%llu,\"hops\":[%llu,%llu,%llu,%llu,%llu]}\n",
                   seq, step, (int)fast, nhop, (unsigned long long)q.snd_nxt, (unsigned long long)p.hop[0], (unsigned long long)p.hop[1],
                   (unsigned long long)p.hop[2], (unsigned long long)p.hop[3], (unsigned long long)p.hop[4]);
            print_state("hpcc", seq, step, fast, q, 0, set);
        }
    }
}
// a queue pair's whole rate state, as JSON
void state_json(const char *key, const rdma::SndQP &q, bool hpcc)
{
    char a[24], b[24];
    printf("\"%s\":{\"rate\":%llu,\"max_rate\":%llu,\"target\":%llu,\"snd_nxt\":%llu,\"base_rtt\":%llu,\"win\":%u,"
           "\"alpha_cnp\":%u,\"dec_cnp\":%u,\"first_cnp\":%u,\"rp_stage\":%u,\"alpha\":\"%s\",\"lus\":%u,\"inc\":%d,",
           key, (unsigned long long)q.rate, (unsigned long long)q.max_rate, (unsigned long long)q.target, (unsigned long long)q.snd_nxt,
           (unsigned long long)q.base_rtt, q.win, q.alpha_cnp, q.dec_cnp, q.first_cnp, q.rp_stage, hx(q.alpha, a), q.last_update_seq,
           q.inc_stage);
    // (HPCC's and DCTCP's fields share their room in the reference's queue pair)
    if (hpcc)
        printf("\"cur_rate\":%llu,\"u\":\"%s\",", (unsigned long long)q.cur_rate, hx(q.u, b));
    else
        printf("\"high_seq\":%u,\"ecn_cnt\":%u,\"batch\":%u,\"ca_state\":%u,", q.high_seq, q.ecn_cnt, q.batch, q.ca_state);
    printf("\"hop\":[%llu,%llu,%llu,%llu,%llu],\"next_avail\":%lld,\"last_pkt\":%u}", (unsigned long long)q.hop[0],
           (unsigned long long)q.hop[1], (unsigned long long)q.hop[2], (unsigned long long)q.hop[3], (unsigned long long)q.hop[4],
           (long long)q.next_avail, q.last_pkt);
}

void random_params(rdma::Params &P)
{
    P.g = 1.0 / 1024 + unit() * 0.12;
    P.rate_first_cnp = 0.3 + 0.7 * unit();
    P.clamp = (int)below(2);
    P.alpha_int = P.dec_int = P.rp_int = 55;
    P.rpg_threshold = (uint32_t)(1 + below(6));
    P.rai = (1 + below(100)) * 1000000ull + below(1000);
    P.rhai = (1 + below(1000)) * 1000000ull + below(1000);
    P.min_rate = (1 + below(1000)) * 1000000ull;
    P.dctcp_rai = (1 + below(1000)) * 1000000ull;
    P.u_target = 0.5 + 0.5 * unit();
    P.mi_thresh = (uint32_t)below(8);
    P.sample_feedback = (int)below(2);
    P.int_multi = (uint32_t)(1 + below(4));
    P.mtu = 500 + (uint32_t)below(4000);
}

void params_json(const rdma::Params &P)
{
    char a[24], b[24], d[24];
    printf("\"P\":{\"g\":\"%s\",\"rate_first_cnp\":\"%s\",\"clamp\":%d,\"rpg_threshold\":%u,\"rai\":%llu,\"rhai\":%llu,"
           "\"min_rate\":%llu,\"dctcp_rai\":%llu,\"u_target\":\"%s\",\"mi_thresh\":%u,\"sample_feedback\":%d,\"int_multi\":%u,"
           "\"mtu\":%u}",
           hx(P.g, a), hx(P.rate_first_cnp, b), P.clamp, P.rpg_threshold, (unsigned long long)P.rai, (unsigned long long)P.rhai,
           (unsigned long long)P.min_rate, (unsigned long long)P.dctcp_rai, hx(P.u_target, d), P.mi_thresh, P.sample_feedback,
           P.int_multi, P.mtu);
}

// one event on a queue pair in a random state, for each rule
void kat_single()
{
    for (int i = 0; i < 900; i++)
    {
        Harness H;
        random_params(H.P);
        rdma::SndQP &q = H.qp[0];
        q.max_rate = RATES[below(5)];
        q.rate = H.P.min_rate + below(q.max_rate - H.P.min_rate + 1);
        q.target = below(q.max_rate + 1);
        q.snd_nxt = below(1ull << 31);
        q.base_rtt = 1000 + below(30000);
        q.win = (uint32_t)(1000 + below(1u << 22));
        q.last_pkt = (uint32_t)(64 + below(9000));
        q.next_avail = (int64_t)below(1ull << 40);
        const int kind = i % 3; // 0 DCQCN, 1 DCTCP, 2 HPCC
        if (kind == 0)
        {
            q.alpha = unit();
            q.rp_stage = (uint32_t)below(10);
            q.alpha_cnp = (uint8_t)below(2);
            q.dec_cnp = (uint8_t)below(2);
            q.first_cnp = (uint8_t)below(2);
            const int ev = (int)below(4);
            printf("{\"fn\":\"dcqcn1\",\"ev\":%d,", ev);
            params_json(H.P);
            printf(",");
            state_json("a", q, false);
            q.t_alpha = q.t_dec = q.t_rp = -1;
            if (ev == 0)
                rdma::dcqcn_cnp(H.c, 0, q);
            else
                rdma::dcqcn_timer(H.c, 0, ev - 1);
            const unsigned started = (q.t_alpha >= 0 ? 1u : 0u) | (q.t_dec >= 0 ? 2u : 0u) | (q.t_rp >= 0 ? 4u : 0u);
            printf(",\"started\":%u,", started);
            state_json("b", q, false);
            printf("}\n");
        }
        else if (kind == 1)
        {
            q.alpha = unit();
            q.last_update_seq = below(4) == 0 ? 0 : (uint32_t)below(1u << 31);
            q.batch = (uint32_t)(1 + below(100));
            q.ecn_cnt = (uint32_t)below(q.batch + 5);
            q.ca_state = (uint32_t)below(2);
            q.high_seq = (uint32_t)below(1u << 31);
            rdma::Pkt p{};
            p.seq = below(2) ? (uint32_t)below(1u << 31) : (uint32_t)(q.snd_nxt - below(1u << 16));
            p.cnp = (uint8_t)below(2);
            printf("{\"fn\":\"dctcp1\",\"ack\":%u,\"cnp\":%u,", p.seq, p.cnp);
            params_json(H.P);
            printf(",");
            state_json("a", q, false);
            rdma::dctcp_ack(H.c, q, p);
            printf(",");
            state_json("b", q, false);
            printf("}\n");
        }
        else
        {
            q.u = unit() * 3;
            q.inc_stage = (int32_t)below(9);
            q.cur_rate = H.P.min_rate + below(q.max_rate - H.P.min_rate + 1);
            q.last_update_seq = below(5) == 0 ? 0 : (uint32_t)below(1u << 31);
            rdma::Pkt p{};
            p.nhop = (uint16_t)(below(8) == 0 ? 6 : 1 + below(5)); // (more than MAX_HOP: ignored)
            for (int k = 0; k < 5; k++)
            {
                const uint64_t rate = RATES[below(5)];
                const uint64_t t0 = below(1ull << 24), b0 = below(1ull << 30);
                q.hop[k] = rdma::hop_make(t0, b0, (uint32_t)below(1u << 21), rate, H.P.int_multi);
                p.hop[k] = rdma::hop_make(t0 + 1 + below(30000), b0 + below(1ull << 22), below(3) == 0 ? 0 : (uint32_t)below(1u << 21),
                                          rate, H.P.int_multi);
            }
            // ties: hop 1 has hop 0's utilisation over twice the interval (the first of equal hops
            // sets dt); idle hops: no bytes and an empty queue (utilisation 0 sets nothing)
            const int shape = (int)below(4);
            if (shape == 1 && p.nhop >= 2)
            {
                const uint64_t rate = RATES[below(5)], unit_b = 128ull * H.P.int_multi;
                const uint64_t tau = 1 + below(8000), db = below(2000) * unit_b, t0 = below(1ull << 23), t1 = below(1ull << 23);
                const uint64_t b0 = below(1ull << 12) * unit_b, b1 = below(1ull << 12) * unit_b;
                const uint32_t qa = (uint32_t)below(1u << 20), qb = (uint32_t)below(1u << 20);
                q.hop[0] = rdma::hop_make(t0, b0, qa, rate, H.P.int_multi);
                p.hop[0] = rdma::hop_make(t0 + tau, b0 + db, qb, rate, H.P.int_multi);
                q.hop[1] = rdma::hop_make(t1, b1, qa, rate, H.P.int_multi);
                p.hop[1] = rdma::hop_make(t1 + 2 * tau, b1 + 2 * db, qb, rate, H.P.int_multi);
            }
            else if (shape == 2)
                for (int k = 0; k < p.nhop && k < 5; k++)
                    if (below(2))
                    {
                        const uint64_t rate = RATES[below(5)], t0 = below(1ull << 23), b0 = below(1ull << 30);
                        q.hop[k] = rdma::hop_make(t0, b0, (uint32_t)below(1u << 20), rate, H.P.int_multi);
                        p.hop[k] = rdma::hop_make(t0 + 1 + below(8000), b0, 0, rate, H.P.int_multi);
                    }
            const int fast = (int)below(2);
            printf("{\"fn\":\"hpcc1\",\"fast\":%d,\"nhop\":%d,\"hops\":[%llu,%llu,%llu,%llu,%llu],", fast, p.nhop,
                   (unsigned long long)p.hop[0], (unsigned long long)p.hop[1], (unsigned long long)p.hop[2], (unsigned long long)p.hop[3],
                   (unsigned long long)p.hop[4]);
            params_json(H.P);
            printf(",");
            state_json("a", q, true);
            q.tx_rate = 12345;
            q.tx_size = 0;
            rdma::hpcc_update(H.c, q, p, fast != 0);
            printf(",\"set\":%d,", q.tx_rate != 12345 ? 1 : 0);
            state_json("b", q, true);
            printf("}\n");
        }
    }
}
// the NIC: frame sizes, the window, the round robin, the receiver's check, ACK handling
void kat_nic()
{
    for (int extra = 0; extra <= 4; extra += 4)
        for (int isz = 0; isz <= 42; isz += 42)
        {
            rdma::Params P{};
            P.seq_extra = (uint32_t)extra;
            P.int_size = isz;
            const uint32_t payload = (uint32_t)below(4097);
            printf("{\"fn\":\"sizes\",\"seq_extra\":%d,\"int_size\":%d,\"payload\":%u,\"data\":%u,\"ack\":%u}\n", extra, isz, payload,
                   rdma::data_size(P, payload), rdma::ack_size(P));
        }
    // the round robin over a NIC's queue pairs
    for (int i = 0; i < 250; i++)
    {
        Harness H;
        H.P.var_win = (int)below(2);
        H.P.ack_high_prio = (int)below(2);
        const int n = 1 + (int)below(8);
        static rdma::SndQP qps[8];
        static int list[8];
        H.s.qp = qps;
        H.s.qps = list;
        H.s.qps_cap = 8;
        const int64_t now = 1000000 + (int64_t)below(1000);
        printf("{\"fn\":\"rr\",\"var_win\":%d,\"ack_high_prio\":%d,\"now\":%lld,\"qps\":[", H.P.var_win, H.P.ack_high_prio, (long long)now);
        for (int k = 0; k < 8; k++)
        {
            rdma::SndQP &q = qps[k];
            q = rdma::SndQP{};
            q.size = 1 + below(100000);
            const int st = (int)below(5); // done, all sent, window-bound, late, ready
            q.snd_una = st == 0 ? q.size : below(q.size);
            q.snd_nxt = st <= 1 ? q.size : q.snd_una + below(q.size - q.snd_una);
            q.max_rate = RATES[below(5)];
            q.rate = 1 + below(q.max_rate);
            q.win = below(4) == 0 ? 0 : (uint32_t)(1 + below(st == 2 ? q.snd_nxt - q.snd_una + 1 : 200000));
            // (due exactly now, or one ns later, a third of the time)
            q.next_avail = st == 3 ? now + 1 + (below(3) ? (int64_t)below(1000) : 0) : now - (below(3) ? (int64_t)below(1000) : 0);
            printf("%s[%llu,%llu,%llu,%llu,%llu,%u,%lld]", k ? "," : "", (unsigned long long)q.size, (unsigned long long)q.snd_nxt,
                   (unsigned long long)q.snd_una, (unsigned long long)q.rate, (unsigned long long)q.max_rate, q.win, (long long)q.next_avail);
        }
        for (int k = 0; k < 8; k++)
            list[k] = k;
        for (int k = 7; k > 0; k--) // (a shuffled list)
        {
            const int j = (int)below(k + 1), t = list[k];
            list[k] = list[j], list[j] = t;
        }
        rdma::Host &h = H.c.stv[0];
        h.paused = below(4) == 0 ? (uint32_t)below(16) : 0;
        h.ackq_n = below(3) == 0 ? (int)below(3) : 0;
        h.qp_n = n;
        h.rr = (int)below(40);
        H.c.now = now;
        printf("],\"paused\":%u,\"ackq_n\":%d,\"n\":%d,\"rr\":%d,\"list\":[", h.paused, h.ackq_n, n, h.rr);
        for (int k = 0; k < n; k++)
            printf("%s%d", k ? "," : "", list[k]);
        const int pick = rdma::next_qindex(H.c);
        printf("],\"pick\":%d,\"n_after\":%d,\"list_after\":[", pick, h.qp_n);
        for (int k = 0; k < h.qp_n; k++)
            printf("%s%d", k ? "," : "", list[k]);
        printf("]}\n");
    }
    // a data frame at the receiver (ReceiverCheckSeq) and the ACK or NACK it queues
    for (int i = 0; i < 400; i++)
    {
        Harness H;
        static rdma::RcvQP rx[1];
        static rdma::FlowInfo fi[1];
        static rdma::Pkt ackq[8];
        static unsigned long long ev[64];
        H.s.rx = rx;
        H.s.fi = fi;
        H.s.ackq = ackq;
        H.s.ackq_cap = 8;
        H.s.ev = ev;
        H.P.seq_extra = below(2) ? 4 : 0;
        H.P.int_size = below(2) ? 42 : 0;
        H.P.ack_interval = below(2) ? 1 : (uint32_t)(1 + below(20000));
        H.P.chunk = below(2) ? 0 : (uint32_t)(1000 * (1 + below(4)));
        H.P.nack_interval = 500000;
        fi[0] = rdma::FlowInfo{};
        fi[0].size = 1ull << 40;
        rx[0].expected = (uint32_t)(1000 * below(30));
        rx[0].last_nack = below(2) ? rx[0].expected : (uint32_t)(1000 * below(30));
        rx[0].nack_timer = below(4) == 0 ? 1000000 : (int64_t)below(2000000); // (at times expiring exactly now)
        H.c.stv[0].tc_at = 1; // (the device is busy: the ACK stays queued)
        H.c.stv[0].ackq_head = (int)below(8);
        H.c.stv[0].ackq_n = 0;
        H.c.now = 1000000;
        rdma::Pkt p{};
        p.kind = rdma::K_DATA;
        const uint32_t payload = 1 + (uint32_t)below(1000);
        p.size = (uint16_t)rdma::data_size(H.P, payload);
        p.seq = below(3) == 0 ? rx[0].expected : (uint32_t)(1000 * below(30));
        p.ecn = below(2) ? 3 : 0;
        printf("{\"fn\":\"rx\",\"seq_extra\":%u,\"int_size\":%d,\"ack_interval\":%u,\"chunk\":%u,\"nack_interval\":%lld,\"now\":%lld,"
               "\"expected\":%u,\"last_nack\":%u,\"nack_timer\":%lld,\"seq\":%u,\"payload\":%u,\"ecn\":%u,",
               H.P.seq_extra, H.P.int_size, H.P.ack_interval, H.P.chunk, (long long)H.P.nack_interval, (long long)H.c.now, rx[0].expected,
               rx[0].last_nack, (long long)rx[0].nack_timer, p.seq, payload, p.ecn);
        rdma::h_data(H.c, p);
        const rdma::Pkt &a = ackq[H.c.stv[0].ackq_head];
        const int queued = H.c.stv[0].ackq_n;
        printf("\"expected_after\":%u,\"last_nack_after\":%u,\"nack_timer_after\":%lld,\"queued\":%d,\"kind\":%u,\"ack_seq\":%u,"
               "\"cnp\":%u,\"size\":%u}\n",
               rx[0].expected, rx[0].last_nack, (long long)rx[0].nack_timer, queued, queued ? a.kind : 0, queued ? a.seq : 0,
               queued ? a.cnp : 0, queued ? a.size : 0);
    }
    // an ACK or NACK at the sender, with each congestion control
    for (int i = 0; i < 360; i++)
    {
        Harness H;
        static rdma::FlowInfo fi[1];
        static int64_t fct[1];
        static unsigned done_n;
        static unsigned long long ev[64];
        random_params(H.P);
        H.s.fi = fi;
        H.s.fct = fct;
        H.s.flows_done = &done_n;
        H.s.ev = ev;
        H.s.dag = 0;
        fi[0] = rdma::FlowInfo{};
        fi[0].start = 1000;
        fct[0] = -1;
        const int ccs[3] = {1, 3, 8};
        H.P.cc = ccs[i % 3];
        H.P.fast_react = (int)below(2);
        H.c.stv[0].tc_at = 1;
        rdma::SndQP &q = H.qp[0];
        q.max_rate = RATES[below(5)];
        q.rate = H.P.min_rate + below(q.max_rate - H.P.min_rate + 1);
        q.target = q.max_rate;
        q.size = 1000 + below(1u << 20);
        q.snd_una = below(q.size);
        q.snd_nxt = q.snd_una + below(q.size - q.snd_una + 1);
        q.base_rtt = 1000 + below(30000);
        q.win = (uint32_t)(1000 + below(1u << 22));
        q.last_pkt = (uint32_t)(64 + below(9000));
        q.next_avail = (int64_t)below(1ull << 40);
        q.first_cnp = (uint8_t)below(2);
        q.alpha = unit();
        q.t_alpha = q.t_dec = q.t_rp = -1;
        if (H.P.cc == 3)
        {
            q.u = unit() * 2;
            q.cur_rate = q.rate;
            q.inc_stage = (int32_t)below(6);
            q.last_update_seq = below(5) == 0 ? 0 : (uint32_t)below(q.size + 1);
        }
        else if (H.P.cc == 8)
        {
            q.last_update_seq = below(4) == 0 ? 0 : (uint32_t)below(q.size + 1);
            q.batch = (uint32_t)(1 + below(100));
            q.ecn_cnt = (uint32_t)below(q.batch + 5);
            q.ca_state = (uint32_t)below(2);
            q.high_seq = (uint32_t)below(q.size + 1);
        }
        rdma::Pkt p{};
        p.kind = below(4) == 0 ? rdma::K_NACK : rdma::K_ACK;
        p.seq = below(6) == 0 ? (uint32_t)q.size : (uint32_t)below(q.snd_nxt + 1);
        p.cnp = (uint8_t)below(2);
        p.nhop = (uint16_t)(1 + below(5));
        for (int k = 0; k < 5; k++)
        {
            const uint64_t rate = RATES[below(5)];
            const uint64_t t0 = below(1ull << 24), b0 = below(1ull << 30);
            q.hop[k] = rdma::hop_make(t0, b0, (uint32_t)below(1u << 21), rate, H.P.int_multi);
            p.hop[k] = rdma::hop_make(t0 + 1 + below(30000), b0 + below(1ull << 22), (uint32_t)below(1u << 21), rate, H.P.int_multi);
        }
        // (HPCC's state has other fields: its cases are "ack_hp")
        printf("{\"fn\":\"%s\",\"cc\":%d,\"fast_react\":%d,\"nack\":%d,\"seq\":%u,\"cnp\":%u,\"nhop\":%u,"
               "\"hops\":[%llu,%llu,%llu,%llu,%llu],\"size\":%llu,\"snd_una\":%llu,",
               H.P.cc == 3 ? "ack_hp" : "ack", H.P.cc, H.P.fast_react, p.kind == rdma::K_NACK, p.seq, p.cnp, p.nhop, (unsigned long long)p.hop[0], (unsigned long long)p.hop[1],
               (unsigned long long)p.hop[2], (unsigned long long)p.hop[3], (unsigned long long)p.hop[4], (unsigned long long)q.size,
               (unsigned long long)q.snd_una);
        params_json(H.P);
        printf(",");
        state_json("a", q, H.P.cc == 3);
        H.c.now = 5000000;
        rdma::h_ack(H.c, p);
        const unsigned started = (q.t_alpha >= 0 ? 1u : 0u) | (q.t_dec >= 0 ? 2u : 0u) | (q.t_rp >= 0 ? 4u : 0u);
        printf(",\"snd_una_after\":%llu,\"done\":%u,\"fct\":%lld,\"started\":%u,", (unsigned long long)q.snd_una, q.done,
               (long long)fct[0], started);
        state_json("b", q, H.P.cc == 3);
        printf("}\n");
    }
}
// the NIC's dequeue (DequeueAndTransmit): its pick's next data frame goes out onto a one-slot link
// buffer, or, with none ready, the next send is scheduled; and a queue pair's start
void kat_dequeue()
{
    for (int i = 0; i < 400; i++)
    {
        Harness H;
        static rdma::SndQP qps[8];
        static int list[8];
        static rdma::FlowInfo fi[8];
        static rdma::Chain h_tc[1], h_ns[1];
        static rdma::Pkt ackq[4];
        static unsigned long long ev[64];
        static unsigned pend[8];
        static rdma::LFrame msg[4];
        static int64_t first_sent[8];
        for (int k = 0; k < 8; k++)
            first_sent[k] = -1;
        H.s.sent = first_sent;
        H.s.qp = qps;
        H.s.qps = list;
        H.s.qps_cap = 8;
        H.s.fi = fi;
        H.s.h_tc = h_tc;
        H.s.h_ns = h_ns;
        H.s.ackq = ackq;
        H.s.ackq_cap = 4;
        H.s.ev = ev;
        H.s.R = 1;
        H.s.fD = rdma::fdiv_make(1000);
        H.s.fpend = rdma::fdiv_make(8);
        H.s.pend = pend;
        H.s.msg = msg;
        H.P.delay = 1000;
        H.P.simai = (int)below(2);
        H.P.seq_extra = H.P.simai ? 4 : 0;
        H.P.int_size = below(2) ? 42 : 0;
        H.P.mtu = 500 + (uint32_t)below(4000);
        H.P.var_win = (int)below(2);
        H.P.rate_bound = (int)below(2);
        const rdma::FDiv one = rdma::fdiv_make(1);
        rdma::OutBucket &o = H.c.obv[0];
        o = rdma::OutBucket{};
        o.nb = 1;
        o.nb_m = one.m;
        o.nb_sh = (uint8_t)one.sh;
        o.nb_add = (uint8_t)one.add;
        o.cap = 4;
        H.c.ldl[0] = 1000;
        msg[0] = rdma::LFrame{};
        const int64_t now = 5000 + (int64_t)below(3);
        H.c.now = now;
        const int n = 1 + (int)below(8);
        printf("{\"fn\":\"dequeue\",\"simai\":%d,\"int_size\":%d,\"mtu\":%u,\"var_win\":%d,\"rate_bound\":%d,\"now\":%lld,\"qps\":[",
               H.P.simai, H.P.int_size, H.P.mtu, H.P.var_win, H.P.rate_bound, (long long)now);
        for (int k = 0; k < 8; k++)
        {
            rdma::SndQP &q = qps[k];
            q = rdma::SndQP{};
            q.size = 1 + below(20000);
            const int st = (int)below(4); // done / all sent, window-bound, late, ready
            q.snd_una = st == 0 ? (below(2) ? q.size : below(q.size)) : below(q.size);
            q.snd_nxt = st == 0 ? q.size : q.snd_una + below(q.size - q.snd_una);
            q.max_rate = RATES[below(5)];
            q.rate = 1000000000ull + below(q.max_rate - 1000000000ull);
            q.win = st == 1 ? (uint32_t)(q.snd_nxt - q.snd_una + 1 - below(2)) : 0;
            // (at times due exactly now, or one ns later)
            q.next_avail = st == 2 ? now + 1 + (below(3) ? (int64_t)below(1000) : 0) : now - (below(3) ? (int64_t)below(1000) : 0);
            fi[k] = rdma::FlowInfo{};
            printf("%s[%llu,%llu,%llu,%llu,%llu,%u,%lld]", k ? "," : "", (unsigned long long)q.size, (unsigned long long)q.snd_nxt,
                   (unsigned long long)q.snd_una, (unsigned long long)q.rate, (unsigned long long)q.max_rate, q.win, (long long)q.next_avail);
        }
        for (int k = 0; k < 8; k++)
            list[k] = k;
        rdma::Host &h = H.c.stv[0];
        h.tc_at = -1;
        h.ns_at = below(3) == 0 ? now + 5000 : -1;
        h.qp_n = n;
        h.rr = (int)below(16);
        printf("],\"n\":%d,\"rr\":%d,\"ns_at\":%lld,", n, h.rr, (long long)h.ns_at);
        rdma::h_dequeue(H.c);
        const rdma::Pkt &f = msg[0].p;
        const bool sent = f.size != 0;
        printf("\"sent\":%d,\"flow\":%u,\"seq\":%u,\"size\":%u,\"rr_after\":%d,\"ns_at_after\":%lld,\"n_after\":%d,\"after\":[", (int)sent,
               sent ? f.flow : 0, sent ? f.seq : 0, f.size, h.rr, (long long)h.ns_at, h.qp_n);
        for (int k = 0; k < 8; k++)
            printf("%s[%llu,%u,%lld]", k ? "," : "", (unsigned long long)qps[k].snd_nxt, qps[k].last_pkt, (long long)qps[k].next_avail);
        printf("]}\n");
    }
    // a queue pair's start (the NIC busy: nothing is sent)
    for (int i = 0; i < 60; i++)
    {
        Harness H;
        static rdma::SndQP qps[1];
        static int list[4];
        static rdma::FlowInfo fi[1];
        static rdma::LinkInfo li[2];
        static unsigned long long ev[64];
        H.s.qp = qps;
        H.s.qps = list;
        H.s.qps_cap = 4;
        H.s.fi = fi;
        H.s.li = li;
        H.s.ev = ev;
        H.P.cc = i % 3 == 0 ? 1 : i % 3 == 1 ? 3 : 8;
        fi[0] = rdma::FlowInfo{};
        fi[0].size = 1 + below(1u << 30);
        fi[0].win = (uint32_t)below(1u << 20);
        fi[0].base_rtt = below(100000);
        li[1].bps = RATES[below(5)];
        H.c.lk[0] = 1;
        H.c.stv[0].tc_at = 1;
        H.c.now = (int64_t)below(1ull << 30);
        qps[0] = rdma::SndQP{};
        qps[0].snd_nxt = 77; // (overwritten)
        rdma::h_start(H.c, 0);
        const rdma::SndQP &q = qps[0];
        char a[24], b[24];
        printf("{\"fn\":\"qp_start\",\"cc\":%d,\"size\":%llu,\"win\":%u,\"base_rtt\":%llu,\"bps\":%llu,\"now\":%lld,\"rate\":%llu,"
               "\"max_rate\":%llu,\"target\":%llu,\"q_win\":%u,\"q_base_rtt\":%llu,\"alpha\":\"%s\",\"first_cnp\":%u,\"cur_rate\":%llu,"
               "\"u\":\"%s\",\"next_avail\":%lld,\"snd_nxt\":%llu,\"listed\":%d}\n",
               H.P.cc, (unsigned long long)fi[0].size, fi[0].win, (unsigned long long)fi[0].base_rtt, (unsigned long long)li[1].bps,
               (long long)H.c.now, (unsigned long long)q.rate, (unsigned long long)q.max_rate, (unsigned long long)q.target, q.win,
               (unsigned long long)q.base_rtt, hx(q.alpha, a), q.first_cnp, (unsigned long long)q.cur_rate, hx(q.u, b), (long long)q.next_avail,
               (unsigned long long)q.snd_nxt, H.c.stv[0].qp_n);
    }
}

// a switch of 4 ports for the buffer rules: every port busy transmitting unless a case frees one
struct SwHarness
{
    rdma::Sim s{};
    rdma::Params P{};
    rdma::SCtx c{};
    rdma::SwPortLds w[4]{};
    rdma::Chain tc[4]{}, zero{};
    rdma::PortCfg pc[4]{};
    int pbase[1] = {0};
    rdma::Pkt q0[32]{}, q3[32]{};
    unsigned long long ev[64]{};
    unsigned pend[8]{};
    rdma::LFrame msg[4]{};
    SwHarness()
    {
        s.pc = pc;
        s.pbase = pbase;
        s.q0 = q0;
        s.q3 = q3;
        s.q0_cap = s.q3_cap = 8;
        s.ev = ev;
        s.R = 1; // (one link rate: tx times from the table, all 0 here)
        s.fD = rdma::fdiv_make(1000);
        s.fpend = rdma::fdiv_make(8);
        s.pend = pend;
        s.msg = msg;
        P.delay = 1000;
        c.s = &s;
        c.P = &P;
        c.x = 0;
        c.node = 10;
        c.w = w;
        c.tc = tc;
        c.cur_src = &zero;
        c.now = 5000;
        const rdma::FDiv one = rdma::fdiv_make(1);
        for (int k = 0; k < 4; k++)
        {
            w[k].pt.tc_at = 1;
            w[k].out_delay = 1000;
            w[k].ob.nb = 1;
            w[k].ob.nb_m = one.m;
            w[k].ob.nb_sh = (uint8_t)one.sh;
            w[k].ob.nb_add = (uint8_t)one.add;
            w[k].ob.cap = 4;
        }
    }
};

void random_switch(SwHarness &S)
{
    S.P.buffer_size = (uint32_t)((1 + below(32)) << 20);
    S.c.sw.total_rsrv = 4 * 4096;
    S.c.sw.total_hdrm = (uint32_t)below(S.P.buffer_size / 4);
    S.c.sw.shared_used = (uint32_t)below(S.P.buffer_size - S.c.sw.total_hdrm - S.c.sw.total_rsrv + 1);
    S.c.nvs = below(8) == 0;
    for (int k = 0; k < 4; k++)
    {
        rdma::PortCfg &pc = S.pc[k];
        pc.bps = RATES[below(5)];
        pc.hdrm_cap = (uint32_t)(10000 + below(200000));
        pc.shift = (uint32_t)below(4);
        pc.kmin = (uint32_t)below(100000);
        pc.kmax = pc.kmin + 1 + (uint32_t)below(400000);
        pc.pmax = unit();
        S.w[k].kmin = pc.kmin;
        S.w[k].kmax = pc.kmax;
        rdma::Port &pt = S.w[k].pt;
        const int shape = (int)below(3); // in the reserve, in the shared pool, in the headroom
        pt.ing = shape == 0 ? (uint32_t)below(4097) : 4096 + (uint32_t)below(400000);
        pt.hdrm = shape == 2 ? (uint32_t)below(pc.hdrm_cap + 1) : 0;
        pt.egr = (uint32_t)below(600000);
        pt.mmu_paused = (uint32_t)below(2);
        pt.tx_bytes = below(1ull << 40);
        pt.bytes_total = (uint32_t)below(1u << 22);
        for (int i = 0; i < 6; i++)
            pt.rng.s[i] = (double)(1 + below(4294944000ull));
    }
}

void port_json(const char *key, const rdma::Port &pt)
{
    printf("\"%s\":[%u,%u,%u,%u,%llu,%u,%d]", key, pt.ing, pt.hdrm, pt.egr, pt.mmu_paused, (unsigned long long)pt.tx_bytes, pt.bytes_total,
           pt.q0_n);
}

void switch_json(const SwHarness &S)
{
    printf("\"buffer\":%u,\"sw\":[%u,%u,%u],\"nvs\":%d,\"cfg\":[", S.P.buffer_size, S.c.sw.shared_used, S.c.sw.total_hdrm, S.c.sw.total_rsrv,
           (int)S.c.nvs);
    char a[24];
    for (int k = 0; k < 4; k++)
        printf("%s[%llu,%u,%u,%u,%u,\"%s\"]", k ? "," : "", (unsigned long long)S.pc[k].bps, S.pc[k].hdrm_cap, S.pc[k].shift, S.pc[k].kmin,
               S.pc[k].kmax, hx(S.pc[k].pmax, a));
    printf("]");
}

// the buffer rules: admission (SwitchNode's forwarding with the egress busy, so the frame queues),
// release at dequeue (the frame goes out onto its link), and the ECMP choice
void kat_mmu()
{
    for (int i = 0; i < 500; i++)
    {
        SwHarness S;
        random_switch(S);
        const int in = (int)below(4), out = (in + 1 + (int)below(3)) % 4;
        rdma::Pkt p{};
        p.kind = rdma::K_DATA;
        p.size = (uint16_t)(64 + below(9000));
        rdma::Port &pi = S.w[in].pt;
        const int edge = (int)below(8);
        const uint32_t free_b = S.P.buffer_size - S.c.sw.total_hdrm - S.c.sw.total_rsrv;
        if (edge == 0) // (a nearly full buffer and headroom: the frame may be dropped)
        {
            pi.hdrm = S.pc[in].hdrm_cap - (uint32_t)below(p.size);
            pi.ing = 4096 + (uint32_t)below(100000);
            S.c.sw.shared_used = free_b - (uint32_t)below(1u << 16);
        }
        else if (edge == 1) // (the headroom exactly full with the frame, the shared part above the threshold)
        {
            const uint32_t th = (free_b - S.c.sw.shared_used) >> S.pc[in].shift;
            pi.hdrm = S.pc[in].hdrm_cap - p.size;
            pi.ing = 4096 + th + (uint32_t)below(2);
        }
        else if (edge == 2) // (the frame fills the shared part exactly to the threshold)
        {
            const uint32_t th = (free_b - S.c.sw.shared_used) >> S.pc[in].shift;
            pi.hdrm = 0;
            pi.mmu_paused = 0;
            if (th >= p.size)
                pi.ing = 4096 + th - p.size;
        }
        else if (edge == 3) // (a threshold of 0 and the frame in the reserve)
        {
            pi.hdrm = 0;
            pi.mmu_paused = 0;
            pi.ing = (uint32_t)below(4096 - p.size + 1);
            S.c.sw.shared_used = free_b - (uint32_t)below(1u << S.pc[in].shift);
        }
        printf("{\"fn\":\"admit\",\"in\":%d,\"out\":%d,\"size\":%u,", in, out, p.size);
        switch_json(S);
        printf(",");
        port_json("pin", S.w[in].pt);
        printf(",");
        port_json("pout", S.w[out].pt);
        const unsigned long long drop0 = S.ev[0], pause0 = S.ev[2];
        rdma::s_forward(S.c, in, p, out, rdma::PG);
        printf(",\"shared_after\":%u,\"drop\":%llu,\"pause\":%llu,", S.c.sw.shared_used, S.ev[0] - drop0, S.ev[2] - pause0);
        port_json("pin_after", S.w[in].pt);
        printf(",");
        port_json("pout_after", S.w[out].pt);
        printf("}\n");
    }
    for (int i = 0; i < 500; i++)
    {
        SwHarness S;
        random_switch(S);
        S.P.ecn = (int)below(4) != 0;
        S.P.cc = below(2) ? 3 : 1;
        S.P.int_multi = (uint32_t)(1 + below(4));
        const int in = (int)below(4), out = (in + 1 + (int)below(3)) % 4;
        rdma::Pkt p{};
        p.kind = below(4) ? rdma::K_DATA : rdma::K_ACK;
        p.size = (uint16_t)(64 + below(9000));
        p.inport = (uint8_t)in;
        p.nhop = (uint16_t)(below(10) == 0 ? 0xFFFF : below(8));
        for (int k = 0; k < 5; k++)
            p.hop[k] = next64();
        // (the frame's bytes are in the counters it leaves: at least its size)
        rdma::Port &pi = S.w[in].pt, &po = S.w[out].pt;
        if (pi.hdrm + pi.ing < p.size)
            pi.ing += p.size;
        if (po.egr < p.size)
            po.egr += p.size;
        const int edge = (int)below(6);
        if (edge == 0) // (the ingress counters near the resume condition)
        {
            pi.hdrm = below(2) ? 0 : (uint32_t)below(p.size + 1);
            pi.ing = 4096 + (uint32_t)below(2 * 4096) + (pi.hdrm < p.size ? p.size - pi.hdrm : 0);
            pi.mmu_paused = 1;
        }
        else if (edge == 1) // (after it leaves, the shared part exactly RESUME_OFFSET below the threshold)
        {
            const uint32_t x = (uint32_t)below(1000);
            S.pc[in].shift = 0;
            pi.hdrm = 0;
            pi.mmu_paused = 1;
            pi.ing = 4096 + x + p.size;
            S.c.sw.shared_used = S.P.buffer_size - S.c.sw.total_hdrm - S.c.sw.total_rsrv + p.size - x - 3072 - (uint32_t)below(2);
        }
        else if (edge == 2) // (after it leaves, the egress queue exactly at kmax)
            po.egr = S.w[out].kmax + p.size;
        else if (edge == 3) // (after it leaves, the egress queue exactly at kmin)
            po.egr = S.w[out].kmin + p.size;
        po.tc_at = -1;
        nsm_rng::State probe = po.rng;
        const double u = nsm_rng::rand_u01(probe);
        const nsm_rng::State rng0 = po.rng;
        char a[24];
        printf("{\"fn\":\"release\",\"in\":%d,\"out\":%d,\"size\":%u,\"kind\":%u,\"ecn\":%d,\"cc\":%d,\"multi\":%u,\"nhop\":%u,"
               "\"hops\":[%llu,%llu,%llu,%llu,%llu],\"now\":%lld,\"u\":\"%s\",",
               in, out, p.size, p.kind, S.P.ecn, S.P.cc, S.P.int_multi, p.nhop, (unsigned long long)p.hop[0], (unsigned long long)p.hop[1],
               (unsigned long long)p.hop[2], (unsigned long long)p.hop[3], (unsigned long long)p.hop[4], (long long)S.c.now, hx(u, a));
        switch_json(S);
        printf(",");
        port_json("pin", pi);
        printf(",");
        port_json("pout", po);
        const unsigned long long mark0 = S.ev[1], resume0 = S.ev[3];
        rdma::s_start_q3(S.c, out, p);
        const int drawn = memcmp(&rng0, &po.rng, sizeof rng0) != 0;
        const rdma::Pkt &f = S.msg[0].p;
        printf(",\"shared_after\":%u,\"mark\":%llu,\"resume\":%llu,\"drawn\":%d,\"sent_ecn\":%u,\"sent_nhop\":%u,"
               "\"sent_hops\":[%llu,%llu,%llu,%llu,%llu],",
               S.c.sw.shared_used, S.ev[1] - mark0, S.ev[3] - resume0, drawn, f.ecn, f.nhop, (unsigned long long)f.hop[0],
               (unsigned long long)f.hop[1], (unsigned long long)f.hop[2], (unsigned long long)f.hop[3], (unsigned long long)f.hop[4]);
        port_json("pin_after", pi);
        printf(",");
        port_json("pout_after", po);
        printf("}\n");
    }
    // ECMP: a switch's equal-cost ports towards each host
    for (int i = 0; i < 300; i++)
    {
        rdma::Sim s{};
        rdma::Params P{};
        rdma::SwInfo si{};
        rdma::Route rt[16];
        uint8_t rtp[64];
        si.seed = (uint32_t)below(3000);
        si.hbase = (int)below(100);
        si.rt_off = 0;
        int off = 0;
        for (int h = 0; h < 16; h++)
        {
            rt[h].off = (uint32_t)off;
            rt[h].n = (uint32_t)(below(8) == 0 ? 0 : 1 + below(4));
            for (uint32_t k = 0; k < rt[h].n; k++)
                rtp[off++] = (uint8_t)below(32);
        }
        s.si = &si;
        s.rt = rt;
        s.rtp = rtp;
        P.ack_high_prio = (int)below(2);
        rdma::Pkt p{};
        p.kind = below(2) ? rdma::K_DATA : rdma::K_ACK;
        p.src = (uint16_t)(si.hbase + below(16));
        p.dst = (uint16_t)(si.hbase + below(16));
        p.sport = (uint16_t)(10000 + below(50000));
        int q = -1;
        const int port = rdma::s_route(s, P, 0, p, &q);
        const int d = (p.kind == rdma::K_DATA ? p.dst : p.src) - si.hbase;
        printf("{\"fn\":\"route\",\"data\":%d,\"src\":%d,\"dst\":%d,\"sport\":%u,\"seed\":%u,\"ack_high_prio\":%d,\"n\":%u,"
               "\"ports\":[",
               p.kind == rdma::K_DATA, p.src - si.hbase, p.dst - si.hbase, p.sport, si.seed, P.ack_high_prio, rt[d].n);
        for (uint32_t k = 0; k < rt[d].n; k++)
            printf("%s%u", k ? "," : "", rtp[rt[d].off + k]);
        printf("],\"port\":%d,\"q\":%d}\n", port, q);
    }
}
// the event order: chains grown with the reference's cpush from flows' start chains, compared by its
// ccmp (with and without a virtual push on either side); each case prints both chains' runs as
// the cursor reads them, newest first
void runs_json(const char *key, const rdma::Chain &c, uint32_t code0)
{
    rdma::RunCursor cur;
    cur.init(c, code0);
    printf("\"%s\":[", key);
    for (int k = 0; cur.code; k++)
    {
        printf("%s[%u,%u]", k ? "," : "", cur.code, cur.left);
        cur.left = 0;
        cur.next();
    }
    printf("]");
}

void kat_chain()
{
    static rdma::TailNode tail[1 << 16];
    static unsigned long long tail_cnt;
    static unsigned long long memo_t[1 << 16], memo_walk[1 << 12];
    rdma::g_tail.n = tail;
    rdma::g_tail.cnt = &tail_cnt;
    rdma::g_tail.mask = (1 << 16) - 1;
    rdma::g_memo.t = memo_t;
    rdma::g_memo.mask = (1 << 16) - 1;
    rdma::g_memo.walk = memo_walk;
    rdma::g_memo.walk_mask = (1 << 12) - 1;
    for (int world = 0; world < 6; world++)
    {
        memset(memo_t, 0, sizeof memo_t);
        memset(memo_walk, 0, sizeof memo_walk);
        // flows' start chains as the reference's driver makes them: the gap since the previous
        // start time, the flow's place among those starting together, StartApplication; their
        // hashes 0 (a chain's hash covers what follows its start)
        const int F = 12;
        std::vector<rdma::Chain> pool;
        int64_t prev_t = 0;
        int prev_n = 0;
        for (int f = 0; f < F;)
        {
            const int together = 1 + (int)below(3);
            const int64_t t = prev_t + (int64_t)below(3) * 1000;
            for (int m = 0; m < together && f < F; m++, f++)
            {
                rdma::Chain c{}, c2, c3;
                rdma::cpush(&c2, rdma::ccode(t - prev_t, prev_n), c);
                rdma::cpush(&c3, rdma::ccode(0, m), c2);
                rdma::cpush(&c, rdma::ccode(0, 0), c3);
                c.root = (uint32_t)(f + 1);
                c.hash = 0;
                for (int k = 0; k < rdma::NANC; k++)
                    c.anc[k] = 0;
                pool.push_back(c);
            }
            prev_n = together;
            prev_t = t;
        }
        // the rank of the start chains (the reference's driver's rule): their leads newest first,
        // the first differing one larger first, a shorter chain first, then the root
        std::vector<uint32_t> rank(F);
        {
            auto leads = [](const rdma::Chain &c) {
                std::vector<uint32_t> v;
                for (int i = 0; i < rdma::RUNS && c.r[i].code; i++)
                    for (uint32_t k = 0; k < c.r[i].cnt; k++)
                        v.push_back(c.r[i].code >> rdma::CODE_ORD_BITS);
                return v;
            };
            std::vector<int> idx(F);
            for (int f = 0; f < F; f++)
                idx[f] = f;
            std::sort(idx.begin(), idx.end(), [&](int x, int y) {
                const std::vector<uint32_t> lx = leads(pool[x]), ly = leads(pool[y]);
                for (size_t i = 0; i < lx.size() && i < ly.size(); i++)
                    if (lx[i] != ly[i])
                        return lx[i] > ly[i];
                if (lx.size() != ly.size())
                    return lx.size() < ly.size();
                return pool[x].root < pool[y].root;
            });
            for (int i = 0; i < F; i++)
                rank[idx[i]] = (uint32_t)i;
        }
        rdma::Sim s{};
        s.root_rank = rank.data();
        printf("{\"fn\":\"chain_rank\",\"world\":%d,\"rank\":[", world);
        for (int f = 0; f < F; f++)
            printf("%s%u", f ? "," : "", rank[f]);
        printf("]}\n");
        // events: a child of a random event, with a lead from a small set (ties are common) and
        // a small ordinal; lockstep lineages: the same pushes on two chains
        const int64_t leads[6] = {0, 1, 80, 1000, 2048 + 1000, 4096};
        for (int e = 0; e < 400; e++)
        {
            const size_t at = pool.size() < 40 || below(3) ? pool.size() - 1 - below(pool.size() < 40 ? pool.size() : 40) : below(pool.size());
            const uint32_t code = rdma::ccode(leads[below(6)], (int)below(3));
            rdma::Chain c;
            rdma::cpush(&c, code, pool[at]);
            pool.push_back(c);
            if (below(4) == 0)
            {
                const size_t other = below(pool.size());
                rdma::Chain d;
                rdma::cpush(&d, code, pool[other]);
                pool.push_back(d);
            }
        }
        // lineages in lockstep: the same pushes on two flows' start chains (equal hashes where the
        // starts' leads are equal)
        std::vector<std::pair<size_t, size_t>> lock;
        for (int i = 0; i < 30; i++)
        {
            const int f1 = (int)below(F), f2 = (f1 + 1 + (int)below(F - 1)) % F;
            rdma::Chain a = pool[f1], b = pool[f2];
            const int depth = 1 + (int)below(25);
            for (int k = 0; k < depth; k++)
            {
                const uint32_t code = rdma::ccode(leads[below(6)], (int)below(3));
                rdma::Chain a2, b2;
                rdma::cpush(&a2, code, a);
                rdma::cpush(&b2, below(8) ? code : rdma::ccode(leads[below(6)], (int)below(3)), b);
                a = a2, b = b2;
            }
            pool.push_back(a);
            pool.push_back(b);
            lock.push_back({pool.size() - 2, pool.size() - 1});
        }
        // siblings at two depths: equal leads from a common ancestor, ordinals that differ at both
        // (the deeper difference decides)
        for (int i = 0; i < 30; i++)
        {
            const rdma::Chain &anc = pool[below(pool.size())];
            const int64_t l1 = leads[below(6)], l2 = leads[below(6)];
            const int o1 = (int)below(3), o2 = (int)below(3);
            rdma::Chain a1, a2, b1, b2;
            rdma::cpush(&a1, rdma::ccode(l1, o1), anc);
            rdma::cpush(&a2, rdma::ccode(l2, o2), a1);
            rdma::cpush(&b1, rdma::ccode(l1, (o1 + 1 + (int)below(2)) % 3), anc);
            rdma::cpush(&b2, rdma::ccode(l2, (o2 + 1 + (int)below(2)) % 3), b1);
            pool.push_back(a2);
            pool.push_back(b2);
            lock.push_back({pool.size() - 2, pool.size() - 1});
        }
        for (int i = 0; i < 200; i++)
        {
            size_t x = below(pool.size()), y = below(3) == 0 ? x : below(pool.size());
            if (i < (int)lock.size())
                x = lock[i].first, y = lock[i].second;
            const uint32_t pa = below(3) == 0 ? rdma::ccode(leads[below(6)], (int)below(3)) : 0;
            const uint32_t pb = below(3) == 0 ? (below(2) ? pa : rdma::ccode(leads[below(6)], (int)below(3))) : 0;
            bool inexact = false, inexact_walk = false;
            const int r = rdma::ccmp(s, pa, pool[x], pb, pool[y], &inexact);
            const uint64_t ha = pa ? rdma::chash(pool[x].hash, pa) : pool[x].hash, hb = pb ? rdma::chash(pool[y].hash, pb) : pool[y].hash;
            // the same comparison without the memo of decisions: the root-rank rule, else the walk
            // (a memo key made of ancestors' hashes can be 0 for every chain that starts at a flow's
            // start, whose hash is 0: there an unrelated decision answers)
            const uint32_t ra = pool[x].root, rb = pool[y].root;
            const int walk = ra && rb && ra != rb && ha == hb ? (rank[ra - 1] < rank[rb - 1] ? -1 : 1)
                                                             : rdma::ccmp_walk(pa, pool[x], pb, pool[y], &inexact_walk);
            printf("{\"fn\":\"chain\",\"world\":%d,\"root\":[%u,%u],\"hash\":[\"0x%016llx\",\"0x%016llx\"],", world, pool[x].root,
                   pool[y].root, (unsigned long long)ha, (unsigned long long)hb);
            runs_json("a", pool[x], pa);
            printf(",");
            runs_json("b", pool[y], pb);
            printf(",\"order\":%d,\"walk\":%d,\"inexact\":%d}\n", r, walk, (int)(inexact || inexact_walk));
        }
    }
}
} // namespace

int main()
{
    kat_time();
    kat_hash();
    kat_hops();
    kat_dcqcn();
    kat_dctcp();
    kat_hpcc();
    kat_single();
    kat_nic();
    kat_mmu();
    kat_chain();
    kat_dequeue();
    return 0;
}
