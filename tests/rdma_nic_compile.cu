// Built by tests/test_rdma_nic.py with nvcc for sm_100a (compiled, not run): every NIC rule of
// twins_b200/csrc/tr_nic.cuh instantiated in a kernel.
#include "tr_nic.cuh"

using namespace tr;

struct NicCase
{
    NicParams P;
    CcParams C;
    QpRate rate[4];
    QpSend send[4];
    RxQp rx;
    int list[4], n;
    uint64_t hops[MAX_HOP];
    unsigned out[4];
};

__global__ void nic_rules(NicCase *c)
{
    c->out[0] = data_size(c->P, 1000) + ack_size(c->P);
    const QpRate *r = c->rate;
    const QpSend *s = c->send;
    c->out[1] = (unsigned)next_qindex(c->P, 0, 0, c->list, &c->n, 0, 0, [r, s](int f) { return QpView{r[f], s[f]}; });
    c->out[2] = (unsigned)rx_check(c->P, c->rx, 0, 1000, 0);
    c->out[3] = ack_received(c->P, c->C, c->rate[0], c->send[0], 1000, false, true, c->hops, 1);
    uint32_t seq;
    c->out[0] += next_data(c->P, c->rate[1], c->send[1], 0, true, &seq) + seq;
    c->out[1] += (unsigned)next_send_at(c->P, c->list, c->n, 0, [r, s](int f) { return QpView{r[f], s[f]}; });
    qp_start(c->P, c->rate[2], c->send[2], 1000, 100000000000ull, 1 << 20, 10000, 0);
}

// (and the buffer rules of tr_mmu.cuh)
#include "tr_mmu.cuh"

__global__ void mmu_rules(MmuSwitch *sw, MmuPort *p, uint64_t *hops, unsigned *out)
{
    out[0] = mmu_admit(1 << 20, *sw, p[0], 100000, 2, p[1], 1000, false);
    out[1] = mmu_release(1 << 20, *sw, p[0], 2, p[1], 1000, true, 100, 1000, 0.5, false, [] { return 0.25; });
    uint16_t n = 0;
    int_stamp(hops, n, 5000, 1 << 20, 4096, 100000000000ull, 1);
    out[2] = (unsigned)ecmp_choice(1, 2, 10000, true, 7, 4) + n;
}

// (and the event order of tr_chain.cuh)
#include "tr_chain.cuh"

__global__ void chain_rules(const ChainRun *ra, const ChainRun *rb, const uint32_t *rank, int *out)
{
    out[0] = chain_order(ChainView{ra, 3, 1, chain_hash(0, event_code(1000, 0))}, ChainView{rb, 2, 2, 7}, rank);
}
