// A C shim over the RDMA arithmetic (twins_b200/csrc/tr_cc.cuh), built by tests/test_rdma_cc.py
// with g++ (no floating-point contraction: the rules' fma() calls are explicit) and checked there
// against the reference's known answers.
#include "tr_cc.cuh"

using namespace tr;

extern "C" {

int rc_failed() { return 0; }

void rc_sizes(int *out)
{
    out[0] = (int)sizeof(QpRate);
    out[1] = (int)sizeof(CcParams);
}

long long rc_ns_seconds(double x) { return ns_seconds(x); }
long long rc_tx(unsigned long long bps, unsigned bytes, int ns336) { return tx_time(ns336 != 0, bps, bytes); }
unsigned rc_node_ip(int id) { return node_ip(id); }
unsigned rc_ecmp(unsigned a, unsigned b, unsigned c, unsigned seed) { return ecmp_hash(a, b, c, seed); }

unsigned long long rc_hop_make(unsigned long long t, unsigned long long b, unsigned q, unsigned long long rate, unsigned multi)
{
    return hop_make(t, b, q, rate, multi);
}
unsigned long long rc_hop_time_delta(unsigned long long now, unsigned long long was) { return hop_time_delta(now, was); }
unsigned long long rc_hop_bytes_delta(unsigned long long now, unsigned long long was, unsigned multi) { return hop_bytes_delta(now, was, multi); }
double rc_hop_u(unsigned long long now, unsigned long long was, unsigned multi, unsigned long long max_rate, unsigned win, unsigned long long *tau)
{
    uint64_t t;
    const double u = hpcc_hop_u(now, was, multi, max_rate, win, &t);
    *tau = t;
    return u;
}

// DCQCN events: 0 a CNP, 1 the alpha timer, 2 the decrease check, 3 the increase timer
unsigned rc_dcqcn(QpRate *q, const CcParams *P, int ev)
{
    switch (ev)
    {
    case 0:
        return dcqcn_cnp(*q, *P);
    case 1:
        return dcqcn_alpha(*q, *P);
    case 2:
        return dcqcn_decrease(*q, *P);
    default:
        return dcqcn_increase(*q, *P);
    }
}

void rc_dctcp(QpRate *q, const CcParams *P, unsigned seq, int cnp) { dctcp_ack(*q, *P, seq, cnp != 0); }

int rc_hpcc(QpRate *q, const CcParams *P, const unsigned long long *hops, int nhop, int fast)
{
    uint64_t h[MAX_HOP];
    for (int i = 0; i < MAX_HOP; i++)
        h[i] = hops[i];
    return hpcc_ack(*q, *P, h, nhop, fast != 0);
}

long long rc_paced(long long next_avail, int ns336, unsigned long long old_rate, unsigned long long new_rate, unsigned last_pkt)
{
    return paced_after_change(next_avail, ns336 != 0, old_rate, new_rate, last_pkt);
}
}

// ------------------------------------------------------------------ the NIC rules (tr_nic.cuh)
#include "tr_nic.cuh"

extern "C" {

void rc_nic_sizes(int *out)
{
    out[0] = (int)sizeof(NicParams);
    out[1] = (int)sizeof(QpSend);
    out[2] = (int)sizeof(RxQp);
}

void rc_frame_sizes(const NicParams *P, unsigned payload, unsigned *out)
{
    out[0] = data_size(*P, payload);
    out[1] = ack_size(*P);
}

int rc_next_qindex(const NicParams *P, unsigned paused, int ackq_n, int *list, int *n, int rr, long long now, const QpRate *rates,
                   const QpSend *sends)
{
    return next_qindex(*P, paused, ackq_n, list, n, rr, now, [rates, sends](int f) { return QpView{rates[f], sends[f]}; });
}

int rc_rx_check(const NicParams *P, RxQp *r, unsigned seq, unsigned payload, long long now) { return rx_check(*P, *r, seq, payload, now); }

unsigned rc_ack_received(const NicParams *P, const CcParams *C, QpRate *r, QpSend *q, unsigned seq, int nack, int cnp,
                         const unsigned long long *hops, int nhop)
{
    uint64_t h[MAX_HOP];
    for (int i = 0; i < MAX_HOP; i++)
        h[i] = hops[i];
    return ack_received(*P, *C, *r, *q, seq, nack != 0, cnp != 0, h, nhop);
}
}

// ------------------------------------------------------------------ the buffer rules (tr_mmu.cuh)
#include "tr_mmu.cuh"

extern "C" {

unsigned rc_mmu_admit(unsigned buffer, MmuSwitch *sw, MmuPort *in, unsigned hdrm_cap, unsigned shift, MmuPort *out, unsigned size, int nvs)
{
    return mmu_admit(buffer, *sw, *in, hdrm_cap, shift, *out, size, nvs != 0);
}

// (u: the stream's next uniform number; *drawn: whether the rule took it)
unsigned rc_mmu_release(unsigned buffer, MmuSwitch *sw, MmuPort *in, unsigned in_shift, MmuPort *out, unsigned size, int ecn, unsigned kmin,
                        unsigned kmax, double pmax, int nvs, double u, int *drawn)
{
    *drawn = 0;
    return mmu_release(buffer, *sw, *in, in_shift, *out, size, ecn != 0, kmin, kmax, pmax, nvs != 0, [u, drawn]() {
        *drawn = 1;
        return u;
    });
}

void rc_int_stamp(unsigned long long *hops, unsigned short *nhop, long long now, unsigned long long tx_bytes, unsigned queue_bytes,
                  unsigned long long bps, unsigned multi)
{
    uint64_t h[MAX_HOP];
    for (int i = 0; i < MAX_HOP; i++)
        h[i] = hops[i];
    uint16_t n = *nhop;
    int_stamp(h, n, now, tx_bytes, queue_bytes, bps, multi);
    for (int i = 0; i < MAX_HOP; i++)
        hops[i] = h[i];
    *nhop = n;
}

int rc_ecmp_choice(int src, int dst, unsigned sport, int data, unsigned seed, int n) { return ecmp_choice(src, dst, sport, data != 0, seed, n); }
}

// ------------------------------------------------------------------ the event order (tr_chain.cuh)
#include "tr_chain.cuh"

extern "C" {

unsigned rc_event_code(long long lead, int ord) { return event_code(lead, ord); }
unsigned long long rc_chain_hash(unsigned long long h, unsigned code) { return chain_hash(h, code); }

// runs as (code, count) pairs, newest first
int rc_chain_order(const unsigned *ra, int na, unsigned root_a, unsigned long long hash_a, const unsigned *rb, int nb, unsigned root_b,
                   unsigned long long hash_b, const unsigned *root_rank)
{
    const ChainView a{(const ChainRun *)ra, na, root_a, hash_a}, b{(const ChainRun *)rb, nb, root_b, hash_b};
    return chain_order(a, b, root_rank);
}
}

// (the NIC's start, next frame and next send: tr_nic.cuh)
extern "C" {

void rc_qp_start(const NicParams *P, QpRate *r, QpSend *q, unsigned long long size, unsigned long long bps, unsigned win, unsigned long long base_rtt,
                 long long now)
{
    qp_start(*P, *r, *q, size, bps, win, base_rtt, now);
}

unsigned rc_next_data(const NicParams *P, QpRate *r, QpSend *q, long long now, int rate_bound, unsigned *seq)
{
    return next_data(*P, *r, *q, now, rate_bound != 0, seq);
}

long long rc_next_send_at(const NicParams *P, const int *list, int n, long long now, const QpRate *rates, const QpSend *sends)
{
    return next_send_at(*P, list, n, now, [rates, sends](int f) { return QpView{rates[f], sends[f]}; });
}
}
