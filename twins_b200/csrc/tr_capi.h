// twins-b200: an RDMA run behind the C ABI (tr_capi.cu), for tb_capi.cu's entry points.
#pragma once
#include <string>

namespace tr
{

struct RdmaRun;

struct RStats
{
    long long slots, slots_run, launches;
    double kernel_ms, upload_ms;
    unsigned long long host_events, switch_events, host_ack_events, host_data_events, frames_sent, flows_done;
    unsigned long long bytes_h2d, bytes_d2h, device_bytes;
    int grid;
};

RdmaRun *rdma_new(int device);
void rdma_delete(RdmaRun *r);
int rdma_worlds(const RdmaRun *r);
int rdma_world_flows(RdmaRun *r, int world);
// the world's index, or a negative status (*err: why)
int rdma_add_world(RdmaRun *r, const char *config, const char *topology, int n, const int *src, const int *dst, const long long *size,
                   const long long *start_ns, unsigned long long bps, long long delay_ns, std::string *err);
int rdma_prepare(RdmaRun *r, std::string *err);
// frames a switch port's data queue holds (before the first run)
int rdma_set_queue_cap(RdmaRun *r, int frames);
// 0, 1 (inexact: a capacity overflowed or a tie was not decided exactly), or a negative status
int rdma_run(RdmaRun *r, long long max_slots, std::string *err);
int rdma_results(RdmaRun *r, int world, long long *start_ns, long long *fct_ns);
int rdma_counters(RdmaRun *r, unsigned long long *out, int n);
int rdma_stats(RdmaRun *r, RStats *out);
// the transmission trace: set before the first run (one world); read after it (records of the
// reference's TxRec layout, sorted by start, node, device)
int rdma_set_txtrace(RdmaRun *r, long long cap, long long from_ns, long long until_ns);
int rdma_txtrace(RdmaRun *r, void *out, long long cap, long long *n, long long *total);

} // namespace tr
