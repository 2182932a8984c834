// twins-b200: an RDMA run on the device behind the C ABI (include/twinsb200.h: tb_world_add_rdma,
// tb_run, tb_rdma_results, tb_counters, tb_get_stats): its worlds built on the host (tr_world.h),
// laid out side by side (tr_layout.h), copied to the device, run by the slot kernel (tr_kernel.cu)
// until every flow is done, the stop time or quiescence, and read back.
// (reference: the driver of src/rdma/rmain.cu:1023-2373)
#include "tr_capi.h"
#include "tr_kernel.h"
#include "tr_layout.h"

#include <algorithm>
#include <chrono>
#include <cstring>

namespace tr
{

namespace
{
// the run's arrays that start as set-up images, the ones that start zeroed, and the tail ring
struct DevArrays
{
    std::vector<void *> mem;
    size_t bytes = 0;
    ~DevArrays() { release(); }
    void release()
    {
        for (void *p : mem)
            cudaFree(p);
        mem.clear();
        bytes = 0;
    }
    template <class T>
    bool zeroed(T **p, size_t n)
    {
        const size_t b = sizeof(T) * (n ? n : 1);
        if (cudaMalloc((void **)p, b) != cudaSuccess)
            return false;
        mem.push_back(*p);
        bytes += b;
        return cudaMemset(*p, 0, b) == cudaSuccess;
    }
    template <class T>
    bool copy(T **p, const std::vector<T> &v)
    {
        if (!zeroed(p, v.size()))
            return false;
        return v.empty() || cudaMemcpy(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    }
};
} // namespace

struct RdmaRun
{
    int device = 0;
    std::vector<RdmaWorld> worlds;
    RLayout L;
    DevArrays d;
    RSim s{};
    bool prepared = false, ran = false;
    int tail_log2 = 0; // the tail ring's size (0: by the flows), doubled on a run that lost tails
    int q3_cap = 4096; // frames a switch port's data queue holds
    long long tx_cap = 0, tx_from = 0, tx_until = 0; // the transmission trace (0: none)
    std::vector<TxRec> tx;
    unsigned long long tx_total = 0;
    int grid = 0;
    size_t smem = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<int64_t> fct;
    std::vector<unsigned long long> ev;
    RStats st{};
    unsigned long long h2d = 0, d2h = 0;

    ~RdmaRun()
    {
        d.release();
        if (e0)
            cudaEventDestroy(e0);
        if (e1)
            cudaEventDestroy(e1);
        if (stream)
            cudaStreamDestroy(stream);
    }

    // the initial state on the device: set-up images copied, the rest zeroed
    bool upload(std::string *err)
    {
        d.release();
        const RLayout &l = L;
        RSim x{};
        x.H = l.H, x.S = l.S, x.F = l.F, x.W = l.W, x.P = l.P;
        x.D = l.D;
        x.max_slots = l.max_slots;
        x.ackq_cap = l.ackq_cap;
        x.qps_cap = l.qps_cap;
        x.q0_cap = l.q0_cap;
        x.q3_cap = l.q3_cap;
        x.pend_n = l.pend_n;
        const int tl = tail_log2 ? tail_log2 : (l.F >= 20000 ? 24 : 22);
        tail_log2 = tl;
        x.tail_mask = (1ull << tl) - 1;
        std::vector<int64_t> minus1(l.F, -1);
        std::vector<long long> tags(l.n_tags, -(1ll << 16));
        RCtl c{};
        c.next_wake = ~0ull;
        std::vector<RCtl> ctl(1, c);
        bool ok = d.copy((RWorld **)&x.world, l.world) && d.copy((HostInfo **)&x.hinfo, l.hinfo) && d.copy(&x.nic, l.nic) &&
                  d.zeroed(&x.h_tc, l.H) && d.zeroed(&x.h_ns, l.H) && d.zeroed(&x.ackq, (size_t)l.H * l.ackq_cap) &&
                  d.zeroed(&x.qps, (size_t)l.H * l.qps_cap) && d.copy((SwInfo **)&x.sinfo, l.sinfo) && d.copy(&x.sw, l.sw) &&
                  d.copy((PortInfo **)&x.pinfo, l.pinfo) && d.copy(&x.port, l.port) && d.zeroed(&x.p_tc, l.P) &&
                  d.zeroed(&x.q0, (size_t)l.P * l.q0_cap) && d.zeroed(&x.q3, (size_t)l.P * l.q3_cap) &&
                  d.copy((uint32_t **)&x.rt, l.rt) && d.copy((uint8_t **)&x.rtp, l.rtp) && d.copy((FlowInfo **)&x.flow, l.flow) &&
                  d.copy((int **)&x.start_list, l.start_list) && d.copy((uint32_t **)&x.root_rank, l.root_rank) && d.zeroed(&x.qp, l.F) &&
                  d.zeroed(&x.qc, l.F) && d.zeroed(&x.rx, l.F) && d.copy(&x.fct, minus1) && d.copy((LinkInfo **)&x.link, l.link) && d.copy((int32_t **)&x.txt, l.txt) &&
                  d.zeroed(&x.msg, l.n_frames) && d.copy(&x.msg_cnt, tags) && d.zeroed(&x.pend, (size_t)l.pend_n) &&
                  d.zeroed(&x.tail, (size_t)1 << tl) && d.zeroed(&x.tail_cnt, 1) && d.zeroed(&x.ev, EV_N) && d.copy(&x.ctl, ctl) &&
                  (!tx_cap || (d.zeroed(&x.tx, (size_t)tx_cap) && d.zeroed(&x.tx_cnt, 1)));
        if (!ok)
        {
            *err = std::string("device memory for the RDMA run: ") + cudaGetErrorString(cudaGetLastError());
            d.release();
            return false;
        }
        x.tx_cap = tx_cap;
        x.tx_from = tx_from;
        x.tx_until = tx_until;
        // (the zeroing and copies above run on the legacy default stream, which the run's own
        // non-blocking stream does not wait for: all of it must be done before the first launch)
        if (cudaDeviceSynchronize() != cudaSuccess)
        {
            *err = std::string("device memory for the RDMA run: ") + cudaGetErrorString(cudaGetLastError());
            d.release();
            return false;
        }
        s = x;
        h2d = sizeof(RWorld) * l.world.size() + sizeof(HostInfo) * l.hinfo.size() + sizeof(Nic) * l.nic.size() +
              sizeof(SwInfo) * l.sinfo.size() + sizeof(SwState) * l.sw.size() + sizeof(PortInfo) * l.pinfo.size() +
              sizeof(Port) * l.port.size() + 4 * l.rt.size() + l.rtp.size() + sizeof(FlowInfo) * l.flow.size() + 4 * l.start_list.size() +
              4 * l.root_rank.size() + 8 * l.F + sizeof(LinkInfo) * l.link.size() + 8 * l.n_tags + sizeof(RCtl);
        return true;
    }
};

RdmaRun *rdma_new(int device)
{
    RdmaRun *r = new RdmaRun();
    r->device = device;
    return r;
}

void rdma_delete(RdmaRun *r) { delete r; }

int rdma_worlds(const RdmaRun *r) { return (int)r->worlds.size(); }

int rdma_add_world(RdmaRun *r, const char *config, const char *topology, int n, const int *src, const int *dst, const long long *size,
                   const long long *start_ns, unsigned long long bps, long long delay_ns, std::string *err)
{
    if (r->prepared)
        return *err = "worlds are added before the first run", -4;
    if (!config || !topology || n < 0 || (n > 0 && (!src || !dst || !size || !start_ns)) || bps == 0 || delay_ns <= 0)
        return *err = "bad argument", -1;
    RdmaWorld w;
    if (!build_rdma_world(w, parse_rdma_config(config), topology, bps, delay_ns) || !build_rdma_flows(w, n, src, dst, size, start_ns))
        return *err = w.error, -1;
    r->worlds.push_back(std::move(w));
    return (int)r->worlds.size() - 1;
}

int rdma_prepare(RdmaRun *r, std::string *err)
{
    if (r->prepared)
        return 0;
    if (r->worlds.empty())
        return *err = "no worlds", -4;
    if (r->tx_cap && r->worlds.size() > 1)
        return *err = "--txtrace traces one world (no --batch)", -1;
    if (cudaSetDevice(r->device) != cudaSuccess)
        return *err = "cudaSetDevice failed", -2;
    std::vector<const RdmaWorld *> wp;
    for (const RdmaWorld &w : r->worlds)
        wp.push_back(&w);
    if (!layout_rdma(r->L, wp, r->q3_cap))
        return *err = r->L.error, -1;
    if (!r->stream && cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess)
        return *err = "cudaStreamCreate failed", -2;
    if (!r->e0)
    {
        cudaEventCreate(&r->e0);
        cudaEventCreate(&r->e1);
    }
    if (int e = rdma_launch_shape(r->L.max_deg, (r->L.H + RDMA_WARPS - 1) / RDMA_WARPS + r->L.S, &r->grid, &r->smem))
        return *err = std::string("the RDMA slot kernel does not fit: ") + cudaGetErrorString((cudaError_t)e), -2;
    r->prepared = true;
    return 0;
}

int rdma_set_queue_cap(RdmaRun *r, int frames)
{
    if (r->prepared || frames < 1)
        return -4;
    r->q3_cap = frames;
    return 0;
}

int rdma_run(RdmaRun *r, long long max_slots, std::string *err)
{
    if (int e = rdma_prepare(r, err))
        return e;
    for (int attempt = 0;; attempt++)
    {
        const auto t0 = std::chrono::steady_clock::now();
        if (!r->upload(err))
            return -3;
        RSim s = r->s;
        if (max_slots > 0 && max_slots < s.max_slots)
            s.max_slots = max_slots;
        r->st = RStats{};
        r->st.upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        RCtl ctl{};
        float ms_total = 0;
        for (;;)
        {
            cudaEventRecord(r->e0, r->stream);
            const int slots = 4096;
            if (int e = rdma_launch(s, r->grid, r->smem, slots, r->L.max_deg, r->stream))
                return *err = std::string("RDMA slot kernel launch: ") + cudaGetErrorString((cudaError_t)e), -2;
            cudaEventRecord(r->e1, r->stream);
            if (cudaMemcpyAsync(&ctl, s.ctl, sizeof ctl, cudaMemcpyDeviceToHost, r->stream) != cudaSuccess ||
                cudaStreamSynchronize(r->stream) != cudaSuccess)
                return *err = std::string("RDMA slot kernel: ") + cudaGetErrorString(cudaGetLastError()), -2;
            float ms = 0;
            cudaEventElapsedTime(&ms, r->e0, r->e1);
            ms_total += ms;
            r->st.launches++;
            if (ctl.finished || ctl.error)
                break;
        }
        r->fct.assign(r->L.F, -1);
        r->ev.assign(EV_N, 0);
        if (cudaMemcpy(r->fct.data(), s.fct, 8 * (size_t)r->L.F, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(r->ev.data(), s.ev, 8 * EV_N, cudaMemcpyDeviceToHost) != cudaSuccess)
            return *err = "cudaMemcpy failed", -2;
        r->st.kernel_ms = ms_total;
        r->st.slots = ctl.slot;
        r->st.slots_run = ctl.slots_run;
        r->st.flows_done = ctl.flows_done;
        r->st.host_events = r->ev[EV_HOST_ARRIVALS];
        r->st.switch_events = r->ev[EV_SWITCH_ARRIVALS];
        r->st.host_ack_events = r->ev[EV_HOST_ACKS];
        r->st.host_data_events = r->ev[EV_HOST_DATA];
        r->st.frames_sent = r->ev[EV_HOST_FRAMES];
        r->st.grid = r->grid;
        r->st.bytes_h2d = r->h2d;
        r->st.bytes_d2h = 8 * (size_t)r->L.F + 8 * EV_N + sizeof(RCtl) * r->st.launches;
        r->st.device_bytes = r->d.bytes;
        r->tx.clear();
        r->tx_total = 0;
        if (s.tx)
        {
            if (cudaMemcpy(&r->tx_total, s.tx_cnt, sizeof r->tx_total, cudaMemcpyDeviceToHost) != cudaSuccess)
                return *err = "cudaMemcpy failed", -2;
            r->tx.resize((size_t)std::min<unsigned long long>(r->tx_total, (unsigned long long)r->tx_cap));
            if (!r->tx.empty() && cudaMemcpy(r->tx.data(), s.tx, sizeof(TxRec) * r->tx.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
                return *err = "cudaMemcpy failed", -2;
            std::sort(r->tx.begin(), r->tx.end(), [](const TxRec &a, const TxRec &b) {
                return a.ts != b.ts ? a.ts < b.ts : a.node != b.node ? a.node < b.node : a.dev < b.dev;
            });
            r->st.bytes_d2h += sizeof(TxRec) * r->tx.size();
        }
        r->ran = true;
        if (ctl.error)
            return *err = "a device-side barrier wait ran out; the run was abandoned", -5;
        // a decision met a tail node the ring had reused: the run again with a ring twice as large
        if (r->ev[EV_LOST_TAIL] && r->tail_log2 < 27)
        {
            r->tail_log2++;
            continue;
        }
        break;
    }
    const unsigned long long *e = r->ev.data();
    const bool inexact = e[EV_OVF_TX] || e[EV_OVF_QUEUE] || e[EV_OVF_ACKQ] || e[EV_OVF_QPS] || e[EV_OVF_DUE] || e[EV_UNDECIDED] ||
                         e[EV_LOST_TAIL];
    if (inexact)
        *err = "a capacity overflowed or a tie was not decided exactly; results may differ from the reference";
    return inexact ? 1 : 0;
}

int rdma_results(RdmaRun *r, int world, long long *start_ns, long long *fct_ns)
{
    if (!r->ran)
        return -4;
    if (world < 0 || world >= (int)r->worlds.size())
        return -1;
    const int f0 = r->L.world_fbase[world], n = (int)r->worlds[world].flows.size();
    for (int i = 0; i < n; i++)
    {
        if (start_ns)
            start_ns[i] = r->L.flow[f0 + i].start;
        if (fct_ns)
            fct_ns[i] = r->fct[f0 + i];
    }
    return 0;
}

int rdma_counters(RdmaRun *r, unsigned long long *out, int n)
{
    if (!r->ran)
        return -4;
    for (int i = 0; i < n && i < EV_N; i++)
        out[i] = r->ev[i];
    return 0;
}

int rdma_stats(RdmaRun *r, RStats *out)
{
    *out = r->st;
    return r->ran ? 0 : -4;
}

int rdma_set_txtrace(RdmaRun *r, long long cap, long long from_ns, long long until_ns)
{
    if (r->prepared || cap < 0 || until_ns < from_ns)
        return -1;
    r->tx_cap = cap;
    r->tx_from = from_ns;
    r->tx_until = until_ns;
    return 0;
}

int rdma_txtrace(RdmaRun *r, void *out, long long cap, long long *n, long long *total)
{
    if (!r->ran)
        return -4;
    const size_t k = (size_t)std::max(0LL, std::min<long long>(cap, (long long)r->tx.size()));
    if (k && out)
        memcpy(out, r->tx.data(), sizeof(TxRec) * k);
    if (n)
        *n = (long long)k;
    if (total)
        *total = (long long)r->tx_total;
    return 0;
}

int rdma_world_flows(RdmaRun *r, int world) { return world >= 0 && world < (int)r->worlds.size() ? (int)r->worlds[world].flows.size() : -1; }

} // namespace tr
