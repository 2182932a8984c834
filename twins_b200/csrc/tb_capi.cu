// twins-b200: the C ABI (include/twinsb200.h): batches of worlds, their device state, the run.
// World set-up restates the reference's driver (src/main.cu:223-1015): topologies and routes,
// messages over connections, ns-3's ECMP hashes, the order of application events, link wiring.
#include "tb_kernel.h"
#include "tb_state.cuh"
#include "tb_rng_host.h"
#include "tr_capi.h"
#include "tr_kernel.h"
#include "../../include/twinsb200.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <mutex>
#include <vector>

using namespace tb;

namespace
{

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

// ------------------------------------------------------------------ a world on the host
struct FlowRow
{
    int src, dst;
    long long size, start_ns, conn;
};

struct HostWorld
{
    // inputs
    tb_topology topo;
    std::vector<int> link_a, link_b, fail_a, fail_b, fail_up;
    std::vector<long long> fail_t;
    std::vector<FlowRow> rows;
    std::vector<uint32_t> given_hd, given_ha;
    tb_tcp_params p;
    // derived
    int kind = 0, k = 0, hk = 0, H1 = 0, S1 = 0, ecmp_n = 1, leaves = 0, spines = 0, hpl = 0;
    std::vector<int> host_sw, host_port;
    std::vector<uint32_t> rt_off;
    std::vector<uint8_t> rt_n, rt_ports, port_dn;
    std::vector<int64_t> fail_ps;
    std::vector<int> host_in_port;  // world-local: the port (switch*k + p) the host hangs off
    std::vector<int> port_in;       // [S1*k]: the arriving link: host h (>= 0) or -2 - (switch*k + p), -1 unused
    // connections and messages (world-local)
    std::vector<std::vector<int>> conn_rows;
    std::vector<int> row_conn, row_msg;
    std::vector<uint32_t> hash_data, hash_ack; // per connection
    std::vector<int> pend;                     // messages in each host's event order
    std::vector<int> pend_first;               // [H1 + 1]
    std::vector<int> msg_row;                  // message -> row
    std::vector<uint64_t> conn_bytes;
    // global offsets
    int host0 = 0, sw0 = 0, port0 = 0, conn0 = 0, msg0 = 0;
};

bool build_topology(HostWorld &w, std::string &err)
{
    const tb_topology &T = w.topo;
    w.kind = T.kind;
    std::vector<std::vector<std::pair<int, int>>> adj;
    if (T.kind == TB_TOPO_GRAPH)
    {
        w.H1 = T.n_hosts;
        w.S1 = T.n_switches;
        if (w.H1 < 1 || w.S1 < 1)
        {
            err = "a topology file needs hosts and switches";
            return false;
        }
        std::vector<int> deg(w.S1, 0);
        w.host_sw.assign(w.H1, -1);
        w.host_port.assign(w.H1, 0);
        adj.assign(w.S1, {});
        for (size_t i = 0; i < w.link_a.size(); i++)
        {
            int a = w.link_a[i], b = w.link_b[i];
            if (b >= 0 || (a >= 0 && (a >= w.H1 || w.host_sw[a] >= 0)) || -1 - b >= w.S1 || (a < 0 && -1 - a >= w.S1))
            {
                err = "hosts need exactly one link, as its first endpoint";
                return false;
            }
            int sb = -1 - b, pb = deg[sb]++;
            if (a >= 0)
            {
                w.host_sw[a] = sb;
                w.host_port[a] = pb;
            }
            else
            {
                int sa = -1 - a, pa = deg[sa]++;
                adj[sa].push_back({pa, sb});
                adj[sb].push_back({pb, sa});
            }
        }
        for (int h = 0; h < w.H1; h++)
            if (w.host_sw[h] < 0)
            {
                err = "host " + std::to_string(h) + " has no link";
                return false;
            }
        w.k = 0;
        for (int d : deg)
            w.k = std::max(w.k, d);
        if (w.k > 32)
        {
            err = "a switch has more than 32 ports";
            return false;
        }
        struct F
        {
            int64_t t;
            int a, pa, b, pb;
            bool up;
        };
        std::vector<F> fails;
        for (size_t i = 0; i < w.fail_t.size(); i++)
        {
            F x{(int64_t)w.fail_t[i] * 1000, w.fail_a[i], -1, w.fail_b[i], -1, w.fail_up[i] != 0};
            if (x.a < 0 || x.a >= w.S1 || x.b < 0 || x.b >= w.S1)
            {
                err = "--fail: no such switch";
                return false;
            }
            for (auto &pn : adj[x.a])
                if (pn.second == x.b && x.pa < 0)
                    x.pa = pn.first;
            for (auto &pn : adj[x.b])
                if (pn.second == x.a && x.pb < 0)
                    x.pb = pn.first;
            if (x.pa < 0)
            {
                err = "--fail: no link between the switches";
                return false;
            }
            fails.push_back(x);
        }
        std::stable_sort(fails.begin(), fails.end(), [](const F &x, const F &y) { return x.t < y.t; });
        const int NE = (int)fails.size() + 1, S = w.S1, k = w.k;
        for (auto &x : fails)
            w.fail_ps.push_back(x.t);
        w.rt_off.assign((size_t)NE * S * S, 0);
        w.rt_n.assign((size_t)NE * S * S, 0);
        w.port_dn.assign((size_t)NE * S * k, 0);
        std::vector<uint8_t> dn((size_t)S * k, 0);
        for (int ep = 0; ep < NE; ep++)
        {
            if (ep > 0)
            {
                const F &x = fails[ep - 1];
                dn[(size_t)x.a * k + x.pa] = dn[(size_t)x.b * k + x.pb] = x.up ? 0 : 1;
            }
            std::copy(dn.begin(), dn.end(), w.port_dn.begin() + (size_t)ep * S * k);
            // shortest paths (hops) to each switch; equal-cost ports towards a closer neighbour
            // in interface order, as Ipv4GlobalRouting installs them (src/main.cu:420-456)
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
                        err = "switch " + std::to_string(x) + " cannot reach switch " + std::to_string(e);
                        return false;
                    }
                    std::vector<int> pts;
                    for (auto &pn : adj[x])
                        if (!dn[(size_t)x * k + pn.first] && dist[pn.second] == dist[x] - 1)
                            pts.push_back(pn.first);
                    std::sort(pts.begin(), pts.end());
                    size_t r = ((size_t)ep * S + x) * S + e;
                    w.rt_off[r] = (uint32_t)w.rt_ports.size();
                    w.rt_n[r] = (uint8_t)pts.size();
                    for (int q : pts)
                        w.rt_ports.push_back((uint8_t)q);
                }
            }
        }
        w.ecmp_n = 1;
    }
    else if (T.kind == TB_TOPO_LEAFSPINE)
    {
        w.leaves = T.leaves, w.spines = T.spines, w.hpl = T.hpl;
        if (w.leaves < 1 || w.spines < 1 || w.hpl < 1 || std::max(w.hpl + w.spines, w.leaves) > 32 || w.leaves * w.hpl > 65535)
        {
            err = "leaf-spine: max(hpl + spines, leaves) <= 32";
            return false;
        }
        w.k = std::max(w.hpl + w.spines, w.leaves);
        w.H1 = w.leaves * w.hpl;
        w.S1 = w.leaves + w.spines;
        w.ecmp_n = w.spines;
    }
    else if (T.kind == TB_TOPO_FATTREE)
    {
        int k = T.k;
        if (k < 4 || k > 32 || (k & (k - 1)))
        {
            err = "FatTree k: a power of two, 4..32";
            return false;
        }
        w.k = k;
        w.H1 = k * k * k / 4;
        w.S1 = k * k + k * k / 4;
        w.ecmp_n = k / 2;
    }
    else
    {
        err = "unknown topology kind";
        return false;
    }
    if (w.H1 > 65535)
    {
        err = "a world has more than 65535 hosts";
        return false;
    }
    w.hk = w.k / 2;
    // wiring (src/main.cu:870-945): which link arrives at each host and port
    const int k = w.k, hk = w.hk;
    w.host_in_port.assign(w.H1, -1);
    w.port_in.assign((size_t)w.S1 * k, -1);
    auto port_of = [&](int sw, int p) { return sw * k + p; };
    auto from_port = [&](int sw, int p) { return -2 - port_of(sw, p); };
    if (w.kind == TB_TOPO_GRAPH)
    {
        for (int h = 0; h < w.H1; h++)
        {
            w.host_in_port[h] = port_of(w.host_sw[h], w.host_port[h]);
            w.port_in[port_of(w.host_sw[h], w.host_port[h])] = h;
        }
        for (int x = 0; x < w.S1; x++)
            for (auto &pn : adj[x])
            {
                int y = pn.second, nth = 0;
                for (auto &q : adj[x])
                    if (q.second == y && q.first < pn.first)
                        nth++;
                for (auto &q : adj[y])
                    if (q.second == x && nth-- == 0)
                    {
                        w.port_in[port_of(x, pn.first)] = from_port(y, q.first);
                        break;
                    }
            }
    }
    else if (w.kind == TB_TOPO_LEAFSPINE)
    {
        for (int h = 0; h < w.H1; h++)
        {
            int l = h / w.hpl, q = h % w.hpl;
            w.host_in_port[h] = port_of(l, q);
            w.port_in[port_of(l, q)] = h;
        }
        for (int l = 0; l < w.leaves; l++)
            for (int j = 0; j < w.spines; j++)
            {
                int sp = w.leaves + j;
                w.port_in[port_of(l, w.hpl + j)] = from_port(sp, l);
                w.port_in[port_of(sp, l)] = from_port(l, w.hpl + j);
            }
    }
    else
    {
        const int E = k * hk;
        for (int h = 0; h < w.H1; h++)
        {
            int e = h / hk, q = h % hk;
            w.host_in_port[h] = port_of(e, q);
            w.port_in[port_of(e, q)] = h;
        }
        for (int pod = 0; pod < k; pod++)
            for (int j = 0; j < hk; j++)
            {
                int agg = E + pod * hk + j;
                for (int x = 0; x < hk; x++)
                {
                    int e2 = pod * hk + x;
                    w.port_in[port_of(agg, x)] = from_port(e2, j + hk);
                    w.port_in[port_of(e2, j + hk)] = from_port(agg, x);
                }
            }
        for (int i = 0; i < hk; i++)
            for (int j = 0; j < hk; j++)
            {
                int core = k * k + i * hk + j;
                for (int pod = 0; pod < k; pod++)
                {
                    int agg = E + pod * hk + i;
                    w.port_in[port_of(core, pod)] = from_port(agg, j + hk);
                    w.port_in[port_of(agg, j + hk)] = from_port(core, pod);
                }
            }
    }
    return true;
}

bool build_flows(HostWorld &w, std::string &err)
{
    const int M = (int)w.rows.size(), H = w.H1;
    std::map<long long, int> by_id;
    w.row_conn.assign(M, -1);
    for (int i = 0; i < M; i++)
    {
        const FlowRow &r = w.rows[i];
        if (r.src < 0 || r.src >= H || r.dst < 0 || r.dst >= H || r.src == r.dst || r.size < 0)
        {
            err = "flow row " + std::to_string(i) + ": hosts out of range";
            return false;
        }
        int c;
        if (r.conn < 0 || !by_id.count(r.conn))
        {
            c = (int)w.conn_rows.size();
            w.conn_rows.push_back({});
            if (r.conn >= 0)
                by_id[r.conn] = c;
        }
        else
        {
            c = by_id[r.conn];
            const FlowRow &first = w.rows[w.conn_rows[c][0]];
            if (first.src != r.src || first.dst != r.dst || r.start_ns < w.rows[w.conn_rows[c].back()].start_ns)
            {
                err = "the flows of connection " + std::to_string(r.conn) + " need the same hosts and later starts";
                return false;
            }
        }
        w.conn_rows[c].push_back(i);
        w.row_conn[i] = c;
    }
    const int F = (int)w.conn_rows.size();
    w.row_msg.assign(M, -1);
    w.msg_row.clear();
    w.conn_bytes.assign(F, 0);
    for (int c = 0; c < F; c++)
        for (int i : w.conn_rows[c])
        {
            w.row_msg[i] = (int)w.msg_row.size();
            w.msg_row.push_back(i);
            w.conn_bytes[c] += (uint64_t)w.rows[i].size;
            if (w.conn_bytes[c] >= 0xFFFFFFFFull)
            {
                err = "a connection carries 4 GB or more";
                return false;
            }
        }
    // application events per host in ns-3's order: message writes before starts at equal times
    // (src/main.cu:590-612)
    std::vector<int> byrow(M);
    for (int i = 0; i < M; i++)
        byrow[i] = i;
    auto is_first = [&](int i) { return w.conn_rows[w.row_conn[i]][0] == i; };
    std::stable_sort(byrow.begin(), byrow.end(), [&](int a, int b) {
        const FlowRow &x = w.rows[a], &y = w.rows[b];
        if (x.src != y.src)
            return x.src < y.src;
        if (x.start_ns != y.start_ns)
            return x.start_ns < y.start_ns;
        bool fa = is_first(a), fb = is_first(b);
        if (fa != fb)
            return !fa;
        return fa ? w.row_conn[a] < w.row_conn[b] : a < b;
    });
    w.pend.resize(M);
    w.pend_first.assign(H + 1, 0);
    for (int i = 0; i < M; i++)
        w.pend[i] = w.row_msg[byrow[i]];
    {
        int i = 0;
        for (int h = 0; h < H; h++)
        {
            w.pend_first[h] = i;
            while (i < M && w.rows[byrow[i]].src == h)
                i++;
        }
        w.pend_first[H] = i;
    }
    // ECMP hashes (src/main.cu:674-723)
    std::vector<int> hsub(H);
    for (int h = 0; h < H; h++)
        hsub[h] = h;
    if (w.kind == TB_TOPO_GRAPH)
        for (size_t i = 0; i < w.link_a.size(); i++)
            if (w.link_a[i] >= 0)
                hsub[w.link_a[i]] = (int)i;
    auto ip = [&](int h) { return 0x0a000001u | (uint32_t)(hsub[h] & 0xFFFF) << 8; };
    std::vector<int> byhost(F);
    for (int c = 0; c < F; c++)
        byhost[c] = c;
    std::stable_sort(byhost.begin(), byhost.end(), [&](int a, int b) {
        const FlowRow &x = w.rows[w.conn_rows[a][0]], &y = w.rows[w.conn_rows[b][0]];
        return x.src != y.src ? x.src < y.src : x.start_ns < y.start_ns;
    });
    w.hash_data.assign(F, 0);
    w.hash_ack.assign(F, 0);
    const bool given = !w.given_hd.empty();
    for (int i = 0, n = 0; i < F; i++, n++)
    {
        const int c = byhost[i];
        const int src = w.rows[w.conn_rows[c][0]].src, dst = w.rows[w.conn_rows[c][0]].dst;
        if (i > 0 && w.rows[w.conn_rows[byhost[i - 1]][0]].src != src)
            n = 0;
        if (n > 65535 - 49153 && !given)
        {
            err = "a host binds more than 16382 connections: give the hashes";
            return false;
        }
        const uint16_t sport = (uint16_t)(49153 + n), dport = 1000;
        w.hash_data[c] = flow_hash(ip(src), ip(dst), sport, dport);
        w.hash_ack[c] = flow_hash(ip(dst), ip(src), dport, sport);
    }
    if (given)
        for (int i = 0; i < M; i++)
            if (is_first(i))
            {
                w.hash_data[w.row_conn[i]] = w.given_hd[i];
                w.hash_ack[w.row_conn[i]] = w.given_ha[i];
            }
    return true;
}

template <typename T>
struct DevBuf
{
    T *p = nullptr;
    size_t n = 0;
};

} // namespace

// ------------------------------------------------------------------ the context
struct tb_ctx
{
    int device = 0;
    unsigned long long budget = 0;
    std::vector<HostWorld> worlds;
    bool prepared = false, ran = false;
    int host_lanes = 1, grid_req = 0, grid = 0;
    int stage_cap = SW_STAGE;     // frames staged per warp
    int *d_units = nullptr;       // the running units' list (tb_run)
    int64_t *d_unit_done = nullptr; // batches without a grid barrier: per list entry its last slot
    unsigned *d_wunits = nullptr;   // and per world its units in the list
    bool free_batches = true;       // batches run each world on its own barrier
    unsigned long long qtrace_cap = 0; // the enqueue trace (trace build): records kept, window (ps)
    long long qtrace_from = 0, qtrace_until = 0;
    bool autotune = true;         // pick the launch shape per launch by measured throughput
    bool port_local = false;      // a fixed shape's switch egress (tb_set_port_local)
    int dev_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, la = nullptr, lb = nullptr;
    Sim sim{};
    std::vector<void *> allocs;
    size_t dev_bytes = 0;
    // pristine copies of the mutable state, for tb_reset
    struct Snap
    {
        void *dst, *src;
        size_t bytes;
    };
    std::vector<Snap> snaps;
    std::vector<MsgRec> host_msgs;
    std::vector<unsigned long long> ev_w;
    tb_stats stats{};
    int max_slots_per_launch = 4096;
    // tb_run_static: device state carved from a fixed area instead of allocated
    unsigned char *arena = nullptr;
    size_t arena_cap = 0, arena_used = 0;
    // RDMA worlds (tb_world_add_rdma): a context holds TCP worlds or RDMA worlds
    tr::RdmaRun *rdma = nullptr;

    ~tb_ctx()
    {
        release();
        if (rdma)
            tr::rdma_delete(rdma);
    }
    void release()
    {
        for (void *p : allocs)
            cudaFree(p);
        allocs.clear();
        snaps.clear();
        dev_bytes = 0;
        prepared = false;
    }
    template <typename T>
    int alloc(T **p, size_t n, bool snapshot)
    {
        size_t bytes = sizeof(T) * std::max<size_t>(n, 1);
        if (arena)
        {
            // a piece of the fixed area, 256-byte aligned and zeroed (no snapshot: no tb_reset)
            size_t at = (arena_used + 255) & ~(size_t)255;
            if (at + bytes > arena_cap)
                return fail(TB_ERR_MEMORY, "the world needs more device memory than tb_run_static's fixed area (" +
                                               std::to_string(arena_cap >> 20) + " MiB) holds");
            if (cudaMemset(arena + at, 0, bytes) != cudaSuccess)
                return fail(TB_ERR_CUDA, "cudaMemset failed");
            arena_used = at + bytes;
            dev_bytes = arena_used;
            *p = (T *)(arena + at);
            return TB_OK;
        }
        if (budget && dev_bytes + bytes * (snapshot ? 2 : 1) > budget)
            return fail(TB_ERR_MEMORY, "the batch needs more than the context's HBM budget");
        void *d = nullptr;
        if (cudaMalloc(&d, bytes) != cudaSuccess)
            return fail(TB_ERR_CUDA, "cudaMalloc failed");
        allocs.push_back(d);
        dev_bytes += bytes;
        cudaMemset(d, 0, bytes);
        *p = (T *)d;
        if (snapshot)
        {
            void *s = nullptr;
            if (cudaMalloc(&s, bytes) != cudaSuccess)
                return fail(TB_ERR_CUDA, "cudaMalloc failed");
            allocs.push_back(s);
            dev_bytes += bytes;
            snaps.push_back({d, s, bytes});
        }
        return TB_OK;
    }
    template <typename T>
    int upload(T **p, const std::vector<T> &v, bool snapshot)
    {
        int r = alloc(p, v.size(), snapshot);
        if (r)
            return r;
        if (!v.empty() && cudaMemcpy(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(TB_ERR_CUDA, "cudaMemcpy failed");
        stats.bytes_h2d += sizeof(T) * v.size();
        return TB_OK;
    }
};

namespace
{
// Where a world's entities sit in the device arrays (global ids), and where the ports' links
// start: host h sends on link h, port p on link port_links + p.
struct Place
{
    int world = 0, host0 = 0, sw0 = 0, port0 = 0, conn0 = 0, msg0 = 0;
    uint64_t it0 = 0, oo0 = 0;
    int port_links = 0;
};

// A world's initial device records for a place (reference src/model.h:124-277 for the initial
// socket values, src/main.cu:327-1015 for the wiring and the per-host application order)
struct WorldImage
{
    WorldDesc desc;
    std::vector<HostRec> hosts;
    std::vector<SwRec> sws;
    std::vector<PortRec> ports;
    std::vector<int> pend;
    std::vector<SndRec> snd;
    std::vector<RcvRec> rcv;
    std::vector<MsgRec> msgs;
    std::vector<Rng> rng;
    uint64_t it_n = 0, oo_n = 0; // sent-list / RTT-history and out-of-order ring entries it uses
    int active = 1;              // the most connections one host holds on one side
};

void build_image(const HostWorld &w, const Place &pl, WorldImage &img)
{
    WorldDesc &d = img.desc;
    memset(&d, 0, sizeof d);
    d.kind = w.kind;
    d.k = w.k;
    d.hk = w.hk;
    d.leaves = w.leaves;
    d.spines = w.spines;
    d.hpl = w.hpl;
    d.ecmp_n = w.ecmp_n;
    d.H1 = w.H1;
    d.S1 = w.S1;
    d.host0 = pl.host0;
    d.sw0 = pl.sw0;
    d.conn0 = pl.conn0;
    d.msg0 = pl.msg0;
    d.n_msgs = (int)w.rows.size();
    d.cc = (uint8_t)w.p.tcp;
    d.fin = (uint8_t)(w.p.fin != 0);
    d.spray = (uint8_t)(w.p.spray != 0);
    d.red_k = w.p.ecn_k;
    d.qcap = w.p.queue;
    // hosts, switches, ports
    img.hosts.assign(w.H1, HostRec{});
    img.sws.assign(w.S1, SwRec{});
    img.ports.assign((size_t)w.S1 * w.k, PortRec{});
    img.pend.assign(w.rows.size(), 0);
    std::vector<int> nsnd(w.H1, 0), nrcv(w.H1, 0);
    for (auto &cr : w.conn_rows)
    {
        nsnd[w.rows[cr[0]].src]++;
        nrcv[w.rows[cr[0]].dst]++;
    }
    for (int h = 0; h < w.H1; h++)
    {
        img.active = std::max(img.active, std::max(nsnd[h], nrcv[h]));
        HostRec &hr = img.hosts[h];
        memset(&hr, 0, sizeof hr);
        hr.world = pl.world;
        hr.local = h;
        hr.wake = 0; // every host runs the first slot
        hr.pend_next = pl.msg0 + w.pend_first[h];
        hr.pend_end = pl.msg0 + w.pend_first[h + 1];
        hr.in_link = pl.port_links + pl.port0 + w.host_in_port[h];
    }
    for (size_t j = 0; j < w.pend.size(); j++)
        img.pend[j] = pl.msg0 + w.pend[j];
    for (int x = 0; x < w.S1; x++)
    {
        SwRec &sr = img.sws[x];
        sr.world = pl.world;
        sr.local = x;
        sr.port0 = pl.port0 + x * w.k;
        sr.k = w.k;
        for (int q = 0; q < w.k; q++)
        {
            PortRec &pr = img.ports[(size_t)x * w.k + q];
            memset(&pr, 0, sizeof pr);
            pr.red_k = w.p.ecn_k;
            pr.qcap = w.p.queue;
            int src = w.port_in[(size_t)x * w.k + q];
            pr.in_link = src >= 0 ? pl.host0 + src : src == -1 ? -1 : pl.port_links + pl.port0 + (-2 - src);
        }
    }
    // connections and messages
    const int F = (int)w.conn_rows.size();
    img.snd.assign(F, SndRec{});
    img.rcv.assign(F, RcvRec{});
    img.msgs.assign(w.rows.size(), MsgRec{});
    uint64_t it_n = 0, oo_n = 0;
    for (int cc = 0; cc < F; cc++)
    {
        const auto &cr = w.conn_rows[cc];
        const FlowRow &first = w.rows[cr[0]];
        SndRec &S_ = img.snd[cc];
        RcvRec &R = img.rcv[cc];
        memset(&S_, 0, sizeof S_);
        memset(&R, 0, sizeof R);
        S_.world = R.world = pl.world;
        S_.src_local = R.src_local = first.src;
        S_.dst_local = R.dst_local = first.dst;
        S_.hash_data = w.hash_data[cc];
        S_.hash_ack = R.hash_ack = w.hash_ack[cc];
        S_.m_first = pl.msg0 + w.row_msg[cr[0]];
        S_.m_cnt = (int)cr.size();
        S_.fin_on = R.fin_on = (uint8_t)(w.p.fin != 0);
        uint64_t segs = (w.conn_bytes[cc] + MSS - 1) / MSS + cr.size() + 1;
        S_.it_cap = sent_list_cap(segs);
        S_.it_off = pl.it0 + it_n;
        it_n += S_.it_cap;
        R.oo_cap = (uint32_t)std::min<uint64_t>(segs / 2 + 2, 4096);
        R.oo_off = pl.oo0 + oo_n;
        oo_n += R.oo_cap;
        R.bytes = (uint32_t)w.conn_bytes[cc];
        // initial values (reference src/model.h:124-277)
        S_.cwnd = INIT_CWND;
        S_.ssthresh = 0xFFFFFFFFu;
        S_.first_partial = 1;
        S_.cub_delaymin = S_.cub_epoch = S_.cub_roundstart = S_.cub_lastack = S_.cub_currrtt = INT64_MIN;
        S_.ecn_echo_seq = S_.ecn_cwr_seq = -1;
        S_.alpha = 1.0;
        S_.srtt = -1;
        S_.rto = MIN_RTO_PS;
        S_.rto_at = -1;
        S_.syn_at = -1;
        R.fin_seq = R.synack_t = R.srtt = R.last_at = R.frx_at = R.syn_at = R.delack_at = R.ecn_ce_seq = -1;
        for (int r : cr)
        {
            MsgRec &m = img.msgs[w.row_msg[r]];
            m.conn = pl.conn0 + cc;
            m.start = w.rows[r].start_ns * 1000;
            m.est = m.done = -1;
        }
        uint64_t off = 0;
        for (int r : cr)
        {
            off += (uint64_t)w.rows[r].size;
            img.msgs[w.row_msg[r]].end = (uint32_t)off;
        }
    }
    img.it_n = it_n;
    img.oo_n = oo_n;
    // per-packet spraying: node i's Ipv4GlobalRouting draws from stream i; switches are nodes
    // H1.. of the world
    img.rng.assign(w.S1, Rng{});
    if (w.p.spray)
        for (int x = 0; x < w.S1; x++)
            img.rng[x] = stream_state(w.p.rng_seed, (uint64_t)(w.H1 + x), w.p.rng_run);
}

// a graph world's routing tables, uploaded into the context (pointers into d)
int upload_graph(tb_ctx *c, const HostWorld &w, WorldDesc &d)
{
    if (w.kind != TB_TOPO_GRAPH)
        return TB_OK;
    int *hsw;
    uint8_t *hp, *rn, *rp, *pd;
    uint32_t *ro;
    int64_t *ft;
    std::vector<uint8_t> hport(w.host_port.begin(), w.host_port.end());
    int r;
    if ((r = c->upload(&hsw, w.host_sw, false)) || (r = c->upload(&hp, hport, false)) || (r = c->upload(&ro, w.rt_off, false)) ||
        (r = c->upload(&rn, w.rt_n, false)) || (r = c->upload(&rp, w.rt_ports, false)) || (r = c->upload(&pd, w.port_dn, false)) ||
        (r = c->upload(&ft, w.fail_ps, false)))
        return r;
    d.host_sw = hsw;
    d.host_port = hp;
    d.rt_off = ro;
    d.rt_n = rn;
    d.rt_ports = rp;
    d.port_dn = pd;
    d.fail_t = ft;
    d.n_fail = (int)w.fail_ps.size();
    return TB_OK;
}

// A world from the caller's arrays: topology, flow rows (reference src/main.cu:110-137,
// 531-648), parameters; validated, wired and hashed.
int make_world(const tb_topology *topo, int n_flows, const int *src, const int *dst, const long long *size, const long long *start_ns,
               const long long *conn, const unsigned *hash_data, const unsigned *hash_ack, const tb_tcp_params *params, HostWorld &w)
{
    if (!topo || !params || n_flows < 0 || (n_flows > 0 && (!src || !dst || !size || !start_ns)))
        return fail(TB_ERR_ARG, "tb_world_add_tcp: missing argument");
    if (params->tcp < 0 || params->tcp > 2 || params->ecn_k < 0 || params->queue < 1 || params->queue > 65000)
        return fail(TB_ERR_ARG, "bad TCP parameters");
    w.topo = *topo;
    w.p = *params;
    if (topo->kind == TB_TOPO_GRAPH)
    {
        if (topo->n_links < 0 || (topo->n_links && (!topo->link_a || !topo->link_b)))
            return fail(TB_ERR_ARG, "graph links missing");
        w.link_a.assign(topo->link_a, topo->link_a + topo->n_links);
        w.link_b.assign(topo->link_b, topo->link_b + topo->n_links);
        for (int i = 0; i < topo->n_fails; i++)
        {
            w.fail_t.push_back(topo->fail_t_ns[i]);
            w.fail_a.push_back(topo->fail_a[i]);
            w.fail_b.push_back(topo->fail_b[i]);
            w.fail_up.push_back(topo->fail_up ? topo->fail_up[i] : 0);
        }
    }
    else if (topo->n_fails)
        return fail(TB_ERR_ARG, "link failures need a topology file");
    w.topo.link_a = w.topo.link_b = nullptr;
    w.topo.fail_t_ns = nullptr;
    w.topo.fail_a = w.topo.fail_b = w.topo.fail_up = nullptr;
    w.rows.resize(n_flows);
    for (int i = 0; i < n_flows; i++)
        w.rows[i] = {src[i], dst[i], size[i], start_ns[i], conn ? conn[i] : -1};
    if (hash_data && hash_ack)
    {
        w.given_hd.assign(hash_data, hash_data + n_flows);
        w.given_ha.assign(hash_ack, hash_ack + n_flows);
    }
    std::string err;
    if (!build_topology(w, err) || !build_flows(w, err))
        return fail(TB_ERR_ARG, err);
    return TB_OK;
}

// the grid of a launch shape: a warp per unit, at most what is co-resident (0: does not fit)
int grid_for(const tb_ctx *c, int host_lanes, int stage, int units = -1, bool port_local = false, bool free = false)
{
    if (units < 0)
        units = (c->sim.H + host_lanes - 1) / host_lanes + c->sim.S;
    return grid_of(units, TB_WARPS_PER_BLOCK, tb::slot_kernel_blocks_per_sm(stage, port_local, host_lanes, free), c->dev_sms, c->grid_req);
}

// the launch-shape tuner's start, on this context's device: the candidates that fit, and the warps
// co-resident at one host per warp and the default staging
void tuner_init(ShapeTuner &tu, const tb_ctx *c, bool autotune, int lanes, int stage, long long entities, int kmax = 0)
{
    const long long resident = (long long)c->dev_sms * std::max(1, tb::slot_kernel_blocks_per_sm(SW_STAGE, false, 1)) * TB_WARPS_PER_BLOCK;
    tu.init(autotune, lanes, stage, c->port_local, entities, kmax, resident,
            [c](int l, int st, bool pl) { return grid_for(c, l, st, -1, pl) > 0; });
}

int prepare(tb_ctx *c)
{
    if (c->prepared)
        return TB_OK;
    if (c->worlds.empty())
        return fail(TB_ERR_STATE, "no worlds");
    if (c->device < 0)
        return fail(TB_ERR_STATE, "a host-only context (device -1) cannot run");
    if (cudaSetDevice(c->device) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaSetDevice failed");
    auto t0 = std::chrono::steady_clock::now();
    c->stats.bytes_h2d = 0;
    const int W = (int)c->worlds.size();
    int H = 0, S = 0, P = 0, C = 0, M = 0, kmax = 0, ring = 0;
    for (HostWorld &w : c->worlds)
    {
        w.host0 = H;
        w.sw0 = S;
        w.port0 = P;
        w.conn0 = C;
        w.msg0 = M;
        H += w.H1;
        S += w.S1;
        P += w.S1 * w.k;
        C += (int)w.conn_rows.size();
        M += (int)w.rows.size();
        kmax = std::max(kmax, w.k);
        ring = std::max(ring, w.p.queue + 2);
    }
    Sim &s = c->sim;
    s = Sim{};
    s.W = W;
    s.H = H;
    s.S = S;
    s.P = P;
    s.L = H + P;
    s.C = C;
    s.M = M;
    s.ring = ring;
    s.kmax = kmax;
    // worlds: each one's records for its place in the batch (graph tables uploaded per world)
    std::vector<WorldDesc> wd(W);
    std::vector<HostRec> hosts(H);
    std::vector<SwRec> sws(S);
    std::vector<PortRec> ports(P);
    std::vector<int> pend(M);
    std::vector<SndRec> snd(C);
    std::vector<RcvRec> rcv(C);
    std::vector<MsgRec> msgs(M);
    std::vector<Rng> rng(S);
    uint64_t it_total = 0, oo_total = 0;
    int active = 1;
    for (int i = 0; i < W; i++)
    {
        HostWorld &w = c->worlds[i];
        Place pl;
        pl.world = i;
        pl.host0 = w.host0;
        pl.sw0 = w.sw0;
        pl.port0 = w.port0;
        pl.conn0 = w.conn0;
        pl.msg0 = w.msg0;
        pl.it0 = it_total; // (a multiple of 8: every capacity is)
        pl.oo0 = oo_total;
        pl.port_links = H;
        WorldImage img;
        build_image(w, pl, img);
        int r;
        if ((r = upload_graph(c, w, img.desc)))
            return r;
        wd[i] = img.desc;
        std::copy(img.hosts.begin(), img.hosts.end(), hosts.begin() + w.host0);
        std::copy(img.sws.begin(), img.sws.end(), sws.begin() + w.sw0);
        std::copy(img.ports.begin(), img.ports.end(), ports.begin() + w.port0);
        std::copy(img.pend.begin(), img.pend.end(), pend.begin() + w.msg0);
        std::copy(img.snd.begin(), img.snd.end(), snd.begin() + w.conn0);
        std::copy(img.rcv.begin(), img.rcv.end(), rcv.begin() + w.conn0);
        std::copy(img.msgs.begin(), img.msgs.end(), msgs.begin() + w.msg0);
        std::copy(img.rng.begin(), img.rng.end(), rng.begin() + w.sw0);
        it_total += img.it_n;
        oo_total += img.oo_n;
        active = std::max(active, img.active);
    }
    s.act_cap = active;
    c->host_msgs = msgs;
    int r;
    WorldDesc *dwd;
    if ((r = c->upload(&dwd, wd, false)))
        return r;
    s.worlds = dwd;
    if ((r = c->upload(&s.hosts, hosts, true)) || (r = c->upload(&s.sws, sws, false)) || (r = c->upload(&s.ports, ports, true)))
        return r;
    int *dpend;
    if ((r = c->upload(&dpend, pend, false)))
        return r;
    s.pend_msg = dpend;
    if ((r = c->upload(&s.snd, snd, true)) || (r = c->upload(&s.rcv, rcv, true)) || (r = c->upload(&s.msgs, msgs, true)))
        return r;
    // rings and scratch (zero; nothing in them matters before it is written)
    if ((r = c->alloc(&s.host_ring, (size_t)H * ring, false)) || (r = c->alloc(&s.port_ring, (size_t)P * ring, false)) ||
        (r = c->alloc(&s.act_snd, (size_t)H * s.act_cap, false)) || (r = c->alloc(&s.act_rcv, (size_t)H * s.act_cap, false)) ||
        (r = c->alloc(&s.it_start, it_total, false)) || (r = c->alloc(&s.it_fl, it_total, false)) ||
        (r = c->alloc(&s.h_seq, it_total, false)) || (r = c->alloc(&s.h_end, it_total, false)) || (r = c->alloc(&s.h_t, it_total, false)) ||
        (r = c->alloc(&s.oo_s, oo_total, false)) || (r = c->alloc(&s.oo_e, oo_total, false)) ||
        (r = c->alloc(&s.msg, (size_t)NB * s.L * MAX_TX, false)))
        return r;
    {
        std::vector<int64_t> tags((size_t)NB * s.L, -(1ll << 16)); // no slot
        if ((r = c->upload(&s.msg_tag, tags, true)))
            return r;
    }
    size_t per_sw = (size_t)kmax * 2 * MAX_TX;
    if ((r = c->alloc(&s.sw_ts, (size_t)S * per_sw, false)) || (r = c->alloc(&s.sw_ref, (size_t)S * per_sw, false)) ||
        (r = c->alloc(&s.sw_up, (size_t)S * per_sw, false)))
        return r;
    if ((r = c->upload(&s.sw_rng, rng, true)))
        return r;
    {
        // TcpCubic's K = pow(n / 0.4, 1/3) for window differences n, from the host libm (the
        // function ns-3 calls), so that every K equals ns-3's
        bool any_cubic = false;
        for (auto &w : c->worlds)
            any_cubic |= w.p.tcp == TB_TCP_CUBIC;
        std::vector<double> tab(any_cubic ? 65536 : 1);
        for (size_t n = 0; n < tab.size(); n++)
            tab[n] = std::pow((double)n / 0.4, 1 / 3.);
        double *dt;
        if ((r = c->upload(&dt, tab, false)))
            return r;
        s.cub_k_tab = dt;
        s.cub_k_n = (int)tab.size();
    }
    if ((r = c->alloc(&s.ev, EV_N, true)) || (r = c->alloc(&s.ev_w, (size_t)W * EV_N, true)))
        return r;
    {
        std::vector<SlotCtl> ctl(1);
        memset(&ctl[0], 0, sizeof(SlotCtl));
        ctl[0].act_cur = 1; // no skip before the first slots have run
        ctl[0].act_prev = 1;
        ctl[0].next_wake = ~0ull;
        ctl[0].finished = M == 0;
        if ((r = c->upload(&s.ctl, ctl, true)))
            return r;
        std::vector<WorldCtl> wctl(W);
        for (auto &x : wctl)
        {
            memset(&x, 0, sizeof x);
            x.next = 0;
            x.wake = (unsigned long long)INT64_MAX;
            x.act = x.prev = 1; // (as the ticket block's: no skip before the first slots have run)
        }
        if ((r = c->upload(&s.wctl, wctl, true)))
            return r;
    }
    if (!c->arena && ((r = c->alloc(&c->d_units, (size_t)H + S, false)) || (r = c->alloc(&c->d_unit_done, (size_t)H + S, false)) ||
                      (r = c->alloc(&c->d_wunits, (size_t)W, false))))
        return r;
    if (c->qtrace_cap)
    {
        if ((r = c->alloc(&s.qtrace, c->qtrace_cap, false)) || (r = c->alloc(&s.qtrace_cnt, 1, true)))
            return r;
        s.qtrace_n = c->qtrace_cap;
        s.qtrace_from = c->qtrace_from;
        s.qtrace_until = c->qtrace_until;
    }
    // snapshots of the initial state
    for (auto &sn : c->snaps)
        if (cudaMemcpy(sn.src, sn.dst, sn.bytes, cudaMemcpyDeviceToDevice) != cudaSuccess)
            return fail(TB_ERR_CUDA, "snapshot copy failed");
    if (!c->arena && !c->stream && cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaStreamCreate failed");
    if (!c->arena && !c->ev0)
    {
        cudaEventCreate(&c->ev0);
        cudaEventCreate(&c->ev1);
        cudaEventCreate(&c->la);
        cudaEventCreate(&c->lb);
    }
    cudaDeviceGetAttribute(&c->dev_sms, cudaDevAttrMultiProcessorCount, c->device);
    if ((c->grid = grid_for(c, c->host_lanes, c->stage_cap)) <= 0)
        return fail(TB_ERR_CUDA, "the slot kernel does not fit on the device");
    c->prepared = true;
    // (tb_run_static: its own work only, on the legacy default stream, not every stream of the device)
    if (c->arena)
        cudaStreamSynchronize(0);
    else
        cudaDeviceSynchronize();
    c->stats.upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return TB_OK;
}
} // namespace

// ------------------------------------------------------------------ the C ABI
extern "C" {

const char *tb_last_error(void) { return g_err.c_str(); }

int tb_ctx_create(int device, unsigned long long hbm_budget_bytes, tb_ctx **out)
{
    if (!out)
        return fail(TB_ERR_ARG, "out is NULL");
    int n = 0;
    if (device >= 0 && (cudaGetDeviceCount(&n) != cudaSuccess || device >= n))
        return fail(TB_ERR_CUDA, "no such CUDA device");
    tb_ctx *c = new tb_ctx;
    c->device = device;
    c->budget = hbm_budget_bytes;
    *out = c;
    return TB_OK;
}

int tb_ctx_destroy(tb_ctx *ctx)
{
    if (!ctx)
        return TB_OK;
    if (ctx->device >= 0)
        cudaSetDevice(ctx->device);
    if (ctx->stream)
        cudaStreamDestroy(ctx->stream);
    if (ctx->ev0)
    {
        cudaEventDestroy(ctx->ev0);
        cudaEventDestroy(ctx->ev1);
        cudaEventDestroy(ctx->la);
        cudaEventDestroy(ctx->lb);
    }
    delete ctx;
    return TB_OK;
}

int tb_world_add_tcp(tb_ctx *ctx, const tb_topology *topo, int n_flows, const int *src, const int *dst, const long long *size,
                     const long long *start_ns, const long long *conn, const unsigned *hash_data, const unsigned *hash_ack,
                     const tb_tcp_params *params, int *world)
{
    if (!ctx)
        return fail(TB_ERR_ARG, "tb_world_add_tcp: missing argument");
    if (ctx->prepared)
        return fail(TB_ERR_STATE, "the batch is already prepared");
    if (ctx->rdma)
        return fail(TB_ERR_STATE, "a context holds TCP worlds or RDMA worlds, not both");
    HostWorld w;
    int r = make_world(topo, n_flows, src, dst, size, start_ns, conn, hash_data, hash_ack, params, w);
    if (r)
        return r;
    int H = 0;
    for (auto &x : ctx->worlds)
        H += x.H1;
    if ((long long)H + w.H1 > (1ll << 30))
        return fail(TB_ERR_ARG, "too many hosts in the batch");
    ctx->worlds.push_back(std::move(w));
    if (world)
        *world = (int)ctx->worlds.size() - 1;
    return TB_OK;
}

int tb_world_add_rdma(tb_ctx *ctx, const char *config, const char *topology, int n_flows, const int *src, const int *dst,
                      const long long *size, const long long *start_ns, unsigned long long link_bps, long long link_delay_ns, int *world)
{
    if (!ctx)
        return fail(TB_ERR_ARG, "tb_world_add_rdma: missing argument");
    if (!ctx->worlds.empty() || ctx->prepared)
        return fail(TB_ERR_STATE, "a context holds TCP worlds or RDMA worlds, not both");
    if (!ctx->rdma)
        ctx->rdma = tr::rdma_new(ctx->device < 0 ? 0 : ctx->device);
    std::string err;
    const int r = tr::rdma_add_world(ctx->rdma, config, topology, n_flows, src, dst, size, start_ns, link_bps, link_delay_ns, &err);
    if (r < 0)
        return fail(r, err);
    if (world)
        *world = r;
    return TB_OK;
}

int tb_rdma_set_queue_cap(tb_ctx *ctx, int frames)
{
    if (!ctx || frames < 1)
        return fail(TB_ERR_ARG, "frames >= 1");
    if (!ctx->rdma)
        ctx->rdma = tr::rdma_new(ctx->device < 0 ? 0 : ctx->device);
    return tr::rdma_set_queue_cap(ctx->rdma, frames) ? fail(TB_ERR_STATE, "set before the first run") : TB_OK;
}

static_assert(sizeof(tb_tx_record) == sizeof(tr::TxRec) && offsetof(tb_tx_record, seq) == offsetof(tr::TxRec, seq) &&
                  offsetof(tb_tx_record, size) == offsetof(tr::TxRec, size) && offsetof(tb_tx_record, ecn) == offsetof(tr::TxRec, ecn),
              "tb_tx_record is the device's TxRec");

int tb_rdma_set_txtrace(tb_ctx *ctx, long long cap, long long from_ns, long long until_ns)
{
    if (!ctx || cap < 0 || until_ns < from_ns)
        return fail(TB_ERR_ARG, "cap >= 0, from_ns <= until_ns");
    if (!ctx->rdma)
        ctx->rdma = tr::rdma_new(ctx->device < 0 ? 0 : ctx->device);
    return tr::rdma_set_txtrace(ctx->rdma, cap, from_ns, until_ns) ? fail(TB_ERR_STATE, "set before the first run") : TB_OK;
}

int tb_rdma_txtrace(tb_ctx *ctx, tb_tx_record *out, long long cap, long long *n, long long *total)
{
    if (!ctx || !ctx->rdma)
        return fail(TB_ERR_STATE, "no RDMA worlds");
    if (cap < 0)
        return fail(TB_ERR_ARG, "cap >= 0");
    return tr::rdma_txtrace(ctx->rdma, out, cap, n, total) ? fail(TB_ERR_STATE, "not run yet") : TB_OK;
}

int tb_rdma_results(tb_ctx *ctx, int world, long long *start_ns, long long *fct_ns)
{
    if (!ctx || !ctx->rdma)
        return fail(TB_ERR_STATE, "no RDMA worlds");
    const int r = tr::rdma_results(ctx->rdma, world, start_ns, fct_ns);
    return r ? fail(r, r == TB_ERR_STATE ? "not run yet" : "no such world") : TB_OK;
}

int tb_prepare(tb_ctx *ctx)
{
    if (!ctx)
        return fail(TB_ERR_ARG, "ctx is NULL");
    if (ctx->rdma)
    {
        std::string err;
        const int r = tr::rdma_prepare(ctx->rdma, &err);
        return r ? fail(r, err) : TB_OK;
    }
    return prepare(ctx);
}

int tb_reset(tb_ctx *ctx)
{
    if (!ctx || !ctx->prepared)
        return fail(TB_ERR_STATE, "nothing prepared");
    cudaSetDevice(ctx->device);
    for (auto &sn : ctx->snaps)
        if (cudaMemcpyAsync(sn.dst, sn.src, sn.bytes, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
            return fail(TB_ERR_CUDA, "reset copy failed");
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return fail(TB_ERR_CUDA, "reset failed");
    ctx->ran = false;
    return TB_OK;
}

int tb_set_launch_shape(tb_ctx *ctx, int host_lanes, int stage_frames, int grid)
{
    if (!ctx || host_lanes < 1 || host_lanes > 32 || grid < 0 || stage_frames < 1 || stage_frames > SW_STAGE_MAX)
        return fail(TB_ERR_ARG, "host_lanes 1..32, stage_frames 1.." + std::to_string(SW_STAGE_MAX) + ", grid >= 0");
    ctx->host_lanes = host_lanes;
    ctx->stage_cap = stage_frames;
    ctx->grid_req = grid;
    ctx->autotune = false;
    if (ctx->prepared && (ctx->grid = grid_for(ctx, host_lanes, stage_frames)) <= 0)
        return fail(TB_ERR_CUDA, "the slot kernel does not fit on the device with this shape");
    return TB_OK;
}

int tb_set_launch(tb_ctx *ctx, int host_lanes, int grid) { return tb_set_launch_shape(ctx, host_lanes, SW_STAGE, grid); }

int tb_set_port_local(tb_ctx *ctx, int on)
{
    if (!ctx)
        return fail(TB_ERR_ARG, "ctx is NULL");
    ctx->port_local = on != 0;
    if (ctx->prepared && !ctx->autotune && (ctx->grid = grid_for(ctx, ctx->host_lanes, ctx->stage_cap, -1, ctx->port_local)) <= 0)
        return fail(TB_ERR_CUDA, "the slot kernel does not fit on the device with this shape");
    return TB_OK;
}

int tb_set_free_batches(tb_ctx *ctx, int on)
{
    if (!ctx)
        return fail(TB_ERR_ARG, "ctx is NULL");
    ctx->free_batches = on != 0;
    return TB_OK;
}

int tb_set_autotune(tb_ctx *ctx, int on)
{
    if (!ctx)
        return fail(TB_ERR_ARG, "ctx is NULL");
    ctx->autotune = on != 0;
    return TB_OK;
}

int tb_run(tb_ctx *ctx, long long max_slots)
{
    if (!ctx)
        return fail(TB_ERR_ARG, "ctx is NULL");
    if (ctx->rdma)
    {
        std::string err;
        const int r = tr::rdma_run(ctx->rdma, max_slots, &err);
        if (r)
            g_err = err;
        return r;
    }
    int r = prepare(ctx);
    if (r)
        return r;
    if (ctx->ran && (r = tb_reset(ctx)))
        return r;
    cudaSetDevice(ctx->device);
    Sim s = ctx->sim;
    s.max_slots = max_slots > 0 ? max_slots : 2000000;
    SlotCtl ctl{};
    ShapeTuner tu;
    tuner_init(tu, ctx, ctx->autotune, ctx->host_lanes, ctx->stage_cap, (long long)s.H + s.S, s.kmax);
    tu.backoff(96);
    const int run_slots = tu.shapes.size() > 1 ? std::min(ctx->max_slots_per_launch, 1024) : ctx->max_slots_per_launch;
    long long launches = 0;
    // the running worlds' units: rebuilt when a world finishes (or the shape changes), so that a
    // finished world's entities cost a launch nothing and the grid shrinks with the work
    std::vector<std::array<int, 4>> wr(s.W);
    for (int i = 0; i < s.W; i++)
        wr[i] = {ctx->worlds[i].host0, ctx->worlds[i].H1, ctx->worlds[i].sw0, ctx->worlds[i].S1};
    std::vector<WorldCtl> wc(s.W);
    std::vector<int> ulist;
    std::vector<unsigned> wunits;
    int alive = s.W, list_alive = s.W, list_lanes = 0, tuned_alive = s.W;
    s.unit_list = nullptr;
    s.n_list = 0;
    // a batch runs each world on its own barrier (free_kernel), over a world-aligned unit list
    const bool free = ctx->free_batches && s.W > 1 && ctx->d_units && ctx->d_unit_done && ctx->d_wunits;
    if (free)
    {
        s.unit_done = ctx->d_unit_done;
        s.w_units = ctx->d_wunits;
        list_alive = -1;
    }
    bool finished = false;
    tb::SlotGraph graph;
    struct GraphRelease
    {
        tb::SlotGraph &g;
        ~GraphRelease() { tb::release_graph(g); }
    } graph_release{graph};
    cudaEventRecord(ctx->ev0, ctx->stream);
    for (;;)
    {
        const bool explore = tu.explore();
        std::vector<double> per_slot(tu.shapes.size(), -1);
        for (size_t k = 0; k < tu.shapes.size(); k++)
        {
            if (explore ? !tu.probes(k) : k != tu.best)
                continue;
            ShapeTuner::Shape &sh = tu.shapes[k];
            int grid = ctx->grid_req > 0 && !ctx->autotune ? ctx->grid : grid_for(ctx, sh.lanes, sh.stage, -1, sh.port_local);
            if (free)
            {
                if (alive != list_alive || sh.lanes != list_lanes)
                {
                    world_units([&wc](size_t w) { return wc[w].next != INT64_MAX; }, wr, sh.lanes, s.H, ulist, wunits);
                    if ((!ulist.empty() &&
                         cudaMemcpyAsync(ctx->d_units, ulist.data(), sizeof(int) * ulist.size(), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) ||
                        cudaMemcpyAsync(ctx->d_wunits, wunits.data(), sizeof(unsigned) * s.W, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
                        return fail(TB_ERR_CUDA, "cudaMemcpyAsync failed");
                    list_alive = alive;
                    list_lanes = sh.lanes;
                }
                s.unit_list = ctx->d_units;
                s.n_list = (int)ulist.size();
                grid = grid_for(ctx, sh.lanes, sh.stage, s.n_list, sh.port_local, true);
                if (ctx->grid_req > 0 && !ctx->autotune)
                    grid = std::min(grid, ctx->grid);
            }
            else if (ctx->d_units && alive < s.W)
            {
                if (alive != list_alive || sh.lanes != list_lanes)
                {
                    running_units([&wc](size_t w) { return wc[w].next != INT64_MAX; }, wr, sh.lanes, s.H, ulist);
                    if (!ulist.empty() &&
                        cudaMemcpyAsync(ctx->d_units, ulist.data(), sizeof(int) * ulist.size(), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
                        return fail(TB_ERR_CUDA, "cudaMemcpyAsync failed");
                    list_alive = alive;
                    list_lanes = sh.lanes;
                }
                s.unit_list = ctx->d_units;
                s.n_list = (int)ulist.size();
                grid = grid_for(ctx, sh.lanes, sh.stage, s.n_list, sh.port_local);
            }
            const long long slots_before = ctl.slots_run;
            cudaEventRecord(ctx->la, ctx->stream);
            // (the steady launches replay a captured graph; the short probes launch directly)
            int e = explore ? (free ? tb::launch_free(s, grid, tu.probe, sh.lanes, sh.stage, sh.port_local, ctx->stream)
                                    : tb::launch_slots(s, grid, tu.probe, sh.lanes, sh.stage, sh.port_local, ctx->stream))
                            : tb::launch_slots_graph(graph, s, grid, run_slots, sh.lanes, sh.stage, sh.port_local, ctx->stream, free);
            if (e)
                return fail(TB_ERR_CUDA, std::string("slot kernel launch: ") + cudaGetErrorString((cudaError_t)e));
            cudaEventRecord(ctx->lb, ctx->stream);
            launches++;
            if (cudaMemcpyAsync(&ctl, s.ctl, sizeof ctl, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
                (s.W > 1 && cudaMemcpyAsync(wc.data(), s.wctl, sizeof(WorldCtl) * s.W, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) ||
                cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                return fail(TB_ERR_CUDA, std::string("slot kernel: ") + cudaGetErrorString(cudaGetLastError()));
            if (s.W > 1)
            {
                alive = 0;
                for (const WorldCtl &x : wc)
                    alive += x.next != INT64_MAX;
            }
            finished = ctl.error || (free ? alive == 0 : ctl.finished != 0);
            const long long ran = ctl.slots_run - slots_before;
            sh.slots += ran;
            float lms = 0;
            cudaEventElapsedTime(&lms, ctx->la, ctx->lb);
            if (ran >= tu.probe / 2)
                per_slot[k] = lms / (double)ran;
            if (finished)
                break;
        }
        if (explore)
            tu.decide(per_slot);
        else
            tu.since++;
        if (finished)
            break;
        if (4 * (tuned_alive - alive) > tuned_alive)
        {
            tu.load_changed();
            tuned_alive = alive;
        }
    }
    cudaEventRecord(ctx->ev1, ctx->stream);
    cudaEventSynchronize(ctx->ev1);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->ran = true;
    const ShapeTuner::Shape &most = tu.shapes[tu.most()];
    const int most_grid = grid_for(ctx, most.lanes, most.stage, -1, most.port_local);
#ifdef TB_PROFILE
    if (ctl.slots_run > 1)
    {
        const double n = (double)ctl.slots_run;
        fprintf(stderr, "profile: %lld slots; per slot: %.2f us, slowest host unit %.2f us, slowest switch unit %.2f us\n",
                ctl.slots_run, ctl.prof_slot_sum / 1e3 / (n - 1), ctl.prof_host_sum / 1e3 / n, ctl.prof_sw_sum / 1e3 / n);
        fprintf(stderr, "profile: per slot, summed over units (us): host setup %.2f timers %.2f events %.2f flush %.2f "
                        "prune %.2f counters %.2f | switch ingress %.2f egress %.2f\n",
                ctl.prof_phase[0] / 1e3 / n, ctl.prof_phase[1] / 1e3 / n, ctl.prof_phase[2] / 1e3 / n, ctl.prof_phase[3] / 1e3 / n,
                ctl.prof_phase[4] / 1e3 / n, ctl.prof_phase[5] / 1e3 / n, ctl.prof_phase[6] / 1e3 / n, ctl.prof_phase[7] / 1e3 / n);
        fprintf(stderr, "profile: host events split (us per slot, summed): egress advance %.2f arrivals %.2f timers+starts %.2f\n",
                ctl.prof_phase[8] / 1e3 / n, ctl.prof_phase[9] / 1e3 / n, ctl.prof_phase[10] / 1e3 / n);
        fprintf(stderr, "profile: switch ingress split (us per slot, summed): staging %.2f spraying draws %.2f; "
                        "switch slots merged by keys %.0f, by the argmin %.0f\n",
                ctl.prof_phase[11] / 1e3 / n, ctl.prof_phase[12] / 1e3 / n, ctl.prof_phase[13] / 1e3, ctl.prof_phase[14] / 1e3);
    }
#endif
    std::vector<unsigned long long> ev(EV_N);
    ctx->ev_w.assign((size_t)s.W * EV_N, 0);
    cudaMemcpy(ev.data(), s.ev, 8 * EV_N, cudaMemcpyDeviceToHost);
    cudaMemcpy(ctx->ev_w.data(), s.ev_w, 8 * ctx->ev_w.size(), cudaMemcpyDeviceToHost);
    tb_stats &st = ctx->stats;
    st.slots = ctl.slot;
    if (free)
    {
        // (each world's own last slot; the batch's is the latest)
        st.slots = 0;
        for (const WorldCtl &x : wc)
            st.slots = std::max<long long>(st.slots, x.last + 1);
    }
    st.slots_run = ctl.slots_run;
    st.launches = launches;
    st.kernel_ms = ms;
    st.host_events = ev[EV_HOST_PKT];
    st.host_sender_events = ev[EV_HOST_SND];
    st.host_frames = ev[EV_HOST_FRAMES];
    st.switch_events = ev[EV_SW_PKT];
    st.packet_events = st.host_events + st.switch_events;
    st.grid = ctx->grid_req > 0 && !ctx->autotune ? ctx->grid : most_grid;
    st.host_lanes = most.lanes;
    st.warps_per_block = TB_WARPS_PER_BLOCK;
    st.stage_frames = most.stage;
    st.autotuned = tu.shapes.size() > 1;
    st.port_local = most.port_local && most.lanes == 1;
    st.graph_launches = graph.replays;
    st.bytes_d2h = 0;
    if (ctl.error)
        return fail(TB_ERR_TIMEOUT, "a device-side barrier wait ran out; the run was abandoned");
    if (ev[EV_OVF_ACT] || ev[EV_OVF_DUE] || ev[EV_OVF_RING] || ev[EV_OVF_OOO] || ev[EV_OVF_TX])
    {
        g_err = "a capacity overflowed; results may differ from the reference";
        return TB_WARN_INEXACT;
    }
    return TB_OK;
}

int tb_results(tb_ctx *ctx, int world, long long *established_ns, long long *completed_ns)
{
    if (!ctx || world < 0 || world >= (int)ctx->worlds.size())
        return fail(TB_ERR_ARG, "no such world");
    if (!ctx->ran)
        return fail(TB_ERR_STATE, "no run yet");
    HostWorld &w = ctx->worlds[world];
    const int M = (int)w.rows.size();
    std::vector<MsgRec> m(M);
    if (M && cudaMemcpy(m.data(), ctx->sim.msgs + w.msg0, sizeof(MsgRec) * M, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaMemcpy failed");
    ctx->stats.bytes_d2h += sizeof(MsgRec) * M;
    for (int i = 0; i < M; i++)
    {
        const MsgRec &x = m[w.row_msg[i]];
        if (established_ns)
            established_ns[i] = x.est >= 0 ? x.est / 1000 : -1;
        if (completed_ns)
            completed_ns[i] = x.done >= 0 ? x.done / 1000 : -1;
    }
    return TB_OK;
}

int tb_counters(tb_ctx *ctx, int world, unsigned long long *out, int n)
{
    if (ctx && ctx->rdma && out && n >= 0)
    {
        if (world < 0 || world >= tr::rdma_worlds(ctx->rdma))
            return fail(TB_ERR_ARG, "no such world");
        return tr::rdma_counters(ctx->rdma, out, n) ? fail(TB_ERR_STATE, "no run yet") : TB_OK;
    }
    if (!ctx || !out || n < 0 || world < 0 || world >= (int)ctx->worlds.size())
        return fail(TB_ERR_ARG, "bad arguments");
    if (!ctx->ran)
        return fail(TB_ERR_STATE, "no run yet");
    for (int i = 0; i < n && i < EV_N; i++)
        out[i] = ctx->ev_w[(size_t)world * EV_N + i];
    return TB_OK;
}

int tb_hashes(tb_ctx *ctx, int world, unsigned *hash_data, unsigned *hash_ack)
{
    if (!ctx || world < 0 || world >= (int)ctx->worlds.size())
        return fail(TB_ERR_ARG, "no such world");
    HostWorld &w = ctx->worlds[world];
    for (size_t i = 0; i < w.rows.size(); i++)
    {
        if (hash_data)
            hash_data[i] = w.hash_data[w.row_conn[i]];
        if (hash_ack)
            hash_ack[i] = w.hash_ack[w.row_conn[i]];
    }
    return TB_OK;
}

int tb_abi_sizes(unsigned long long *out, int n)
{
    const unsigned long long v[8] = {sizeof(tb_topology),     sizeof(tb_tcp_params),  sizeof(tb_stats), sizeof(tb_serve_caps),
                                     sizeof(tb_request_info), sizeof(tb_serve_stats), sizeof(tb_qrec),  sizeof(tb_tx_record)};
    for (int i = 0; i < n && i < 8; i++)
        out[i] = v[i];
    return TB_OK;
}

int tb_has_qtrace(void)
{
#ifdef TB_QTRACE
    return 1;
#else
    return 0;
#endif
}

int tb_set_qtrace(tb_ctx *ctx, unsigned long long capacity, long long from_ps, long long until_ps)
{
    if (!ctx)
        return fail(TB_ERR_ARG, "ctx is NULL");
    if (!tb_has_qtrace())
        return fail(TB_ERR_STATE, "this library records no enqueue trace: load libtwinsb200_trace.so (or run twins-trace)");
    if (ctx->prepared)
        return fail(TB_ERR_STATE, "set the trace before tb_prepare");
    ctx->qtrace_cap = capacity;
    ctx->qtrace_from = from_ps;
    ctx->qtrace_until = until_ps;
    return TB_OK;
}

int tb_qtrace(tb_ctx *ctx, tb_qrec *out, unsigned long long cap, unsigned long long *n)
{
    static_assert(sizeof(tb_qrec) == sizeof(QRec), "tb_qrec is QRec's public twin");
    if (!ctx || !n)
        return fail(TB_ERR_ARG, "ctx and n are required");
    if (!ctx->ran || !ctx->sim.qtrace)
        return fail(TB_ERR_STATE, "no traced run");
    unsigned long long cnt = 0;
    if (cudaMemcpy(&cnt, ctx->sim.qtrace_cnt, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaMemcpy failed");
    cnt = std::min<unsigned long long>(cnt, ctx->sim.qtrace_n);
    *n = cnt;
    if (out && cap && cudaMemcpy(out, ctx->sim.qtrace, sizeof(QRec) * std::min(cnt, cap), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaMemcpy failed");
    return TB_OK;
}

int tb_get_stats(tb_ctx *ctx, tb_stats *out)
{
    if (!ctx || !out)
        return fail(TB_ERR_ARG, "bad arguments");
    if (ctx->rdma)
    {
        // an RDMA run: host arrivals split by side (ACKs at senders), frames the NICs sent
        tr::RStats r{};
        tr::rdma_stats(ctx->rdma, &r);
        tb_stats o{};
        o.slots = r.slots;
        o.slots_run = r.slots_run;
        o.launches = r.launches;
        o.kernel_ms = r.kernel_ms;
        o.upload_ms = r.upload_ms;
        o.host_events = r.host_events;
        o.switch_events = r.switch_events;
        o.packet_events = r.host_events + r.switch_events;
        o.host_sender_events = r.host_ack_events;
        o.host_frames = r.frames_sent;
        o.bytes_h2d = r.bytes_h2d;
        o.bytes_d2h = r.bytes_d2h;
        o.grid = r.grid;
        o.host_lanes = 1;
        o.warps_per_block = tr::RDMA_WARPS;
        *out = o;
        return TB_OK;
    }
    *out = ctx->stats;
    return TB_OK;
}

} // extern "C"

// ------------------------------------------------------------------ a run that allocates nothing
// Some callers may not allocate device memory: a host program whose memory is managed by a
// framework's pool (the caching allocator of a training or serving process, which owns the
// device's free memory), code running where cudaMalloc is not allowed at that moment, or a
// process under a hard memory cap. tb_run_static serves them: one world's whole device state
// lives in this fixed area, which every process that loads the library holds on each device it
// uses until it exits.
#define TB_STATIC_AREA_BYTES (48ull << 20)
static __device__ __align__(256) unsigned char tb_static_area[TB_STATIC_AREA_BYTES];

namespace
{
std::mutex g_static_mu; // calls of this process take turns
} // namespace

extern "C" int tb_run_static(int device, const tb_topology *topo, int n_flows, const int *src, const int *dst,
                             const long long *size, const long long *start_ns, const long long *conn,
                             const tb_tcp_params *params, long long max_slots, long long *established_ns,
                             long long *completed_ns)
{
    std::lock_guard<std::mutex> lock(g_static_mu);
    int n = 0;
    if (device < 0 || device >= 64 || cudaGetDeviceCount(&n) != cudaSuccess || device >= n)
        return fail(TB_ERR_CUDA, "no such CUDA device");
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaSetDevice failed");
    struct Restore
    {
        int d;
        ~Restore()
        {
            if (d >= 0)
                cudaSetDevice(d);
        }
    } restore{prev};
    // with the device current: the host-side name of the area is not a device address; the runtime
    // gives the address. Asked on every call (it is cheap), so that a context made anew after a
    // cudaDeviceReset, which may load the module at another address, is never given a stale one.
    void *area = nullptr;
    cudaError_t e0 = cudaGetSymbolAddress(&area, tb_static_area);
    if (e0 != cudaSuccess || !area)
        return fail(TB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e0));
    tb_ctx c;
    c.device = device;
    c.arena = (unsigned char *)area;
    c.arena_cap = TB_STATIC_AREA_BYTES;
    int r = tb_world_add_tcp(&c, topo, n_flows, src, dst, size, start_ns, conn, nullptr, nullptr, params, nullptr);
    if (r)
        return r;
    if ((r = prepare(&c)))
        return r;
    Sim s = c.sim;
    s.max_slots = max_slots > 0 ? max_slots : 2000000;
    SlotCtl ctl{};
    for (;;)
    {
        int e = tb::launch_slots(s, c.grid, c.max_slots_per_launch, c.host_lanes, c.stage_cap, false, 0);
        if (e)
            return fail(TB_ERR_CUDA, std::string("slot kernel launch: ") + cudaGetErrorString((cudaError_t)e));
        if (cudaMemcpy(&ctl, s.ctl, sizeof ctl, cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(TB_ERR_CUDA, std::string("slot kernel: ") + cudaGetErrorString(cudaGetLastError()));
        if (ctl.finished || ctl.error)
            break;
    }
    if (ctl.error)
        return fail(TB_ERR_TIMEOUT, "a device-side barrier wait ran out; the run was abandoned");
    c.ran = true;
    c.ev_w.assign(EV_N, 0);
    if (cudaMemcpy(c.ev_w.data(), s.ev_w, 8 * EV_N, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaMemcpy failed");
    if ((r = tb_results(&c, 0, established_ns, completed_ns)))
        return r;
    if (c.ev_w[EV_OVF_ACT] || c.ev_w[EV_OVF_DUE] || c.ev_w[EV_OVF_RING] || c.ev_w[EV_OVF_OOO] || c.ev_w[EV_OVF_TX])
    {
        g_err = "a capacity overflowed; results may differ from the reference";
        return TB_WARN_INEXACT;
    }
    return TB_OK;
}

// ------------------------------------------------------------------ serving
#include "tb_serve.cuh"
