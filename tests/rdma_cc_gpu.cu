// The C shim of tests/rdma_cc.cpp with every function run on the GPU: each call copies its
// arguments to the device, runs the function of twins_b200/csrc/tr_cc.cuh in one thread and copies
// the results back. Built by tests/test_rdma_cc.py with nvcc for sm_100a (--fmad=false: the rules'
// fma() calls are explicit), so that the same known answers check the device code.
#include <cuda_runtime.h>

#include "tr_cc.cuh"

using namespace tr;

namespace
{
struct Args
{
    QpRate q;
    CcParams P;
    uint64_t u64[8];
    uint32_t u32[8];
    double d[2];
    int64_t i64[2];
    int i32[4];
};

Args *dev = nullptr;
int failed = 0;

__global__ void run(Args *a, int fn)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    switch (fn)
    {
    case 0:
        a->i64[0] = ns_seconds(a->d[0]);
        break;
    case 1:
        a->i64[0] = tx_time(a->i32[0] != 0, a->u64[0], a->u32[0]);
        break;
    case 2:
        a->u32[0] = node_ip(a->i32[0]);
        break;
    case 3:
        a->u32[4] = ecmp_hash(a->u32[0], a->u32[1], a->u32[2], a->u32[3]);
        break;
    case 4:
        a->u64[4] = hop_make(a->u64[0], a->u64[1], a->u32[0], a->u64[2], a->u32[1]);
        break;
    case 5:
        a->u64[4] = hop_time_delta(a->u64[0], a->u64[1]);
        a->u64[5] = hop_bytes_delta(a->u64[0], a->u64[1], a->u32[0]);
        break;
    case 6:
    {
        uint64_t tau;
        a->d[0] = hpcc_hop_u(a->u64[0], a->u64[1], a->u32[0], a->u64[2], a->u32[1], &tau);
        a->u64[4] = tau;
        break;
    }
    case 7:
        switch (a->i32[0])
        {
        case 0:
            a->u32[4] = dcqcn_cnp(a->q, a->P);
            break;
        case 1:
            a->u32[4] = dcqcn_alpha(a->q, a->P);
            break;
        case 2:
            a->u32[4] = dcqcn_decrease(a->q, a->P);
            break;
        default:
            a->u32[4] = dcqcn_increase(a->q, a->P);
        }
        break;
    case 8:
        dctcp_ack(a->q, a->P, a->u32[0], a->i32[0] != 0);
        break;
    case 9:
        a->i32[2] = hpcc_ack(a->q, a->P, a->u64, a->i32[0], a->i32[1] != 0);
        break;
    case 10:
        a->i64[0] = paced_after_change(a->i64[0], a->i32[0] != 0, a->u64[0], a->u64[1], a->u32[0]);
        break;
    }
}

// runs fn on the device over *a (a stays the host copy, updated in place)
void call(Args &a, int fn)
{
    if (failed)
        return;
    if ((!dev && cudaMalloc(&dev, sizeof(Args)) != cudaSuccess) || cudaMemcpy(dev, &a, sizeof a, cudaMemcpyHostToDevice) != cudaSuccess)
    {
        failed = 1;
        return;
    }
    run<<<1, 32>>>(dev, fn);
    if (cudaGetLastError() != cudaSuccess || cudaMemcpy(&a, dev, sizeof a, cudaMemcpyDeviceToHost) != cudaSuccess)
        failed = 1;
}
} // namespace

extern "C" {

int rc_failed() { return failed; }

void rc_sizes(int *out)
{
    out[0] = (int)sizeof(QpRate);
    out[1] = (int)sizeof(CcParams);
}

long long rc_ns_seconds(double x)
{
    Args a{};
    a.d[0] = x;
    call(a, 0);
    return a.i64[0];
}

long long rc_tx(unsigned long long bps, unsigned bytes, int ns336)
{
    Args a{};
    a.u64[0] = bps;
    a.u32[0] = bytes;
    a.i32[0] = ns336;
    call(a, 1);
    return a.i64[0];
}

unsigned rc_node_ip(int id)
{
    Args a{};
    a.i32[0] = id;
    call(a, 2);
    return a.u32[0];
}

unsigned rc_ecmp(unsigned w0, unsigned w1, unsigned w2, unsigned seed)
{
    Args a{};
    a.u32[0] = w0, a.u32[1] = w1, a.u32[2] = w2, a.u32[3] = seed;
    call(a, 3);
    return a.u32[4];
}

unsigned long long rc_hop_make(unsigned long long t, unsigned long long b, unsigned q, unsigned long long rate, unsigned multi)
{
    Args a{};
    a.u64[0] = t, a.u64[1] = b, a.u64[2] = rate;
    a.u32[0] = q, a.u32[1] = multi;
    call(a, 4);
    return a.u64[4];
}

unsigned long long rc_hop_time_delta(unsigned long long now, unsigned long long was)
{
    Args a{};
    a.u64[0] = now, a.u64[1] = was;
    a.u32[0] = 1;
    call(a, 5);
    return a.u64[4];
}

unsigned long long rc_hop_bytes_delta(unsigned long long now, unsigned long long was, unsigned multi)
{
    Args a{};
    a.u64[0] = now, a.u64[1] = was;
    a.u32[0] = multi;
    call(a, 5);
    return a.u64[5];
}

double rc_hop_u(unsigned long long now, unsigned long long was, unsigned multi, unsigned long long max_rate, unsigned win, unsigned long long *tau)
{
    Args a{};
    a.u64[0] = now, a.u64[1] = was, a.u64[2] = max_rate;
    a.u32[0] = multi, a.u32[1] = win;
    call(a, 6);
    *tau = a.u64[4];
    return a.d[0];
}

unsigned rc_dcqcn(QpRate *q, const CcParams *P, int ev)
{
    Args a{};
    a.q = *q, a.P = *P;
    a.i32[0] = ev;
    call(a, 7);
    *q = a.q;
    return a.u32[4];
}

void rc_dctcp(QpRate *q, const CcParams *P, unsigned seq, int cnp)
{
    Args a{};
    a.q = *q, a.P = *P;
    a.u32[0] = seq;
    a.i32[0] = cnp;
    call(a, 8);
    *q = a.q;
}

int rc_hpcc(QpRate *q, const CcParams *P, const unsigned long long *hops, int nhop, int fast)
{
    Args a{};
    a.q = *q, a.P = *P;
    for (int i = 0; i < MAX_HOP; i++)
        a.u64[i] = hops[i];
    a.i32[0] = nhop, a.i32[1] = fast;
    call(a, 9);
    *q = a.q;
    return a.i32[2];
}

long long rc_paced(long long next_avail, int ns336, unsigned long long old_rate, unsigned long long new_rate, unsigned last_pkt)
{
    Args a{};
    a.i64[0] = next_avail;
    a.i32[0] = ns336;
    a.u64[0] = old_rate, a.u64[1] = new_rate;
    a.u32[0] = last_pkt;
    call(a, 10);
    return a.i64[0];
}
}
