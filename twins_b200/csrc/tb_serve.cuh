// twins-b200: serving. Simulation requests join a running batch as it runs (continuous batching).
//
// A server owns one set of device arrays sized by its capacities (world slots, hosts, switches,
// ports, connections, messages, ring entries) and runs the slot kernel over all of them in
// launches of a few hundred slots. Between two launches it retires the worlds whose messages are
// all done (their results are read back and their ranges freed) and admits queued requests into
// free ranges (first fit in every pool): a request's records are built for its place and copied
// in, its link messages are cleared, and its time starts at the launch slot it joins (its world
// origin t0), so it runs exactly as it would alone while the worlds already in the batch go on.
// Free entities belong to a world slot that never runs. Requests are admitted in arrival order;
// one that does not fit yet waits, and later ones that fit may pass it (a bounded look-ahead).
//
// There is no counterpart in the reference, which runs one batch of worlds fixed at start
// (src/main.cu:283-325).
//
// (Included by tb_capi.cu: it shares the world builder.)
#pragma once
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

namespace
{
double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
} // namespace

struct tb_server
{
    enum
    {
        QUEUED,
        RUNNING,
        DONE,
        FAILED
    };
    struct Req
    {
        long long id = 0;
        HostWorld w;
        Place pl;
        uint64_t it_n = 0, oo_n = 0;
        int state = QUEUED;
        std::unique_ptr<tb_ctx> tables; // a graph world's routing tables
        std::vector<long long> est, done;
        std::vector<unsigned long long> ctr;
        double t_submit = 0, t_admit = 0, t_done = 0;
        long long t0 = 0, slots = 0; // launch slot it joined, slots it took
        std::string error;
    };
    int device = 0;
    tb_serve_caps caps{};
    tb_ctx dev;  // the pool's device arrays, stream and events
    Sim sim{};
    int dead = 0; // the world slot of free entities (never runs)
    RangeAlloc a_world, a_host, a_sw, a_port, a_conn, a_msg, a_it, a_oo;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<long long> queue;
    std::map<long long, std::unique_ptr<Req>> reqs;
    std::vector<long long> slot_req; // world slot -> running request (0: none)
    long long next_id = 1;
    int lanes = 1, stage = SW_STAGE, grid = 0;
    int *d_units = nullptr;      // the batch's units (device)
    bool units_stale = true;     // admissions or retirements since the list was built
    int list_lanes = 0;          // the hosts per unit the list was built for
    long long batch_entities = 0;
    ShapeTuner tuner;            // the launch shape, per launch
    // statistics
    long long launches = 0, slots_run = 0, admitted = 0, retired = 0;
    double kernel_ms = 0;
    unsigned long long events = 0;
    // the background loop
    std::thread loop;
    bool stop = false, looping = false;
    int error = 0;
    std::string error_text;

    ~tb_server()
    {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
        }
        cv.notify_all();
        if (loop.joinable())
            loop.join();
        if (dev.stream)
            cudaStreamDestroy(dev.stream);
        for (cudaEvent_t e : {dev.ev0, dev.ev1, dev.la, dev.lb})
            if (e)
                cudaEventDestroy(e);
        dev.stream = nullptr;
        dev.ev0 = dev.ev1 = dev.la = dev.lb = nullptr;
    }
};

namespace
{
// ring entries a world's connections need (as build_image sizes them)
void ring_needs(const HostWorld &w, uint64_t &it_n, uint64_t &oo_n)
{
    it_n = oo_n = 0;
    for (size_t cc = 0; cc < w.conn_rows.size(); cc++)
    {
        uint64_t segs = (w.conn_bytes[cc] + MSS - 1) / MSS + w.conn_rows[cc].size() + 1;
        it_n += sent_list_cap(segs);
        oo_n += std::min<uint64_t>(segs / 2 + 2, 4096);
    }
}

int most_active(const HostWorld &w)
{
    std::vector<int> nsnd(w.H1, 0), nrcv(w.H1, 0);
    int a = 1;
    for (auto &cr : w.conn_rows)
    {
        a = std::max(a, ++nsnd[w.rows[cr[0]].src]);
        a = std::max(a, ++nrcv[w.rows[cr[0]].dst]);
    }
    return a;
}

template <typename T>
int put(tb_server *v, T *dst, const std::vector<T> &src)
{
    if (src.empty())
        return TB_OK;
    if (cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, v->dev.stream) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaMemcpyAsync failed");
    return TB_OK;
}

// records that park a range of entities in the dead world
int park(tb_server *v, int host0, int n_hosts, int sw0, int n_sws)
{
    std::vector<HostRec> hosts(n_hosts);
    for (auto &h : hosts)
    {
        memset(&h, 0, sizeof h);
        h.world = v->dead;
        h.wake = INT64_MAX;
    }
    std::vector<SwRec> sws(n_sws);
    for (auto &x : sws)
    {
        memset(&x, 0, sizeof x);
        x.world = v->dead;
    }
    int r;
    if ((r = put(v, v->sim.hosts + host0, hosts)) || (r = put(v, v->sim.sws + sw0, sws)))
        return r;
    return TB_OK;
}

// places a queued request and copies its records in (the device is idle between launches)
// returns 1 when it was admitted, 0 when it does not fit now, < 0 on an error
int admit(tb_server *v, tb_server::Req &q, long long gslot)
{
    HostWorld &w = q.w;
    const uint64_t P1 = (uint64_t)w.S1 * w.k;
    long long wi = v->a_world.take(1), h0 = v->a_host.take(w.H1), s0 = v->a_sw.take(w.S1), p0 = v->a_port.take(P1),
              c0 = v->a_conn.take(w.conn_rows.size()), m0 = v->a_msg.take(w.rows.size()), i0 = v->a_it.take(q.it_n),
              o0 = v->a_oo.take(q.oo_n);
    if (wi < 0 || h0 < 0 || s0 < 0 || p0 < 0 || c0 < 0 || m0 < 0 || i0 < 0 || o0 < 0)
    {
        if (wi >= 0)
            v->a_world.give(wi, 1);
        if (h0 >= 0)
            v->a_host.give(h0, w.H1);
        if (s0 >= 0)
            v->a_sw.give(s0, w.S1);
        if (p0 >= 0)
            v->a_port.give(p0, P1);
        if (c0 >= 0)
            v->a_conn.give(c0, w.conn_rows.size());
        if (m0 >= 0)
            v->a_msg.give(m0, w.rows.size());
        if (i0 >= 0)
            v->a_it.give(i0, q.it_n);
        if (o0 >= 0)
            v->a_oo.give(o0, q.oo_n);
        return 0;
    }
    if (i0 & 7)
    {
        // (sent-list ranges are multiples of 8 entries from 0, so that their flag words are aligned)
        g_err = "internal: a sent-list range off the 8-entry grid";
        return -1;
    }
    Place &pl = q.pl;
    pl.world = (int)wi;
    pl.host0 = (int)h0;
    pl.sw0 = (int)s0;
    pl.port0 = (int)p0;
    pl.conn0 = (int)c0;
    pl.msg0 = (int)m0;
    pl.it0 = (uint64_t)i0;
    pl.oo0 = (uint64_t)o0;
    pl.port_links = v->sim.H;
    w.host0 = pl.host0;
    w.sw0 = pl.sw0;
    w.port0 = pl.port0;
    w.conn0 = pl.conn0;
    w.msg0 = pl.msg0;
    WorldImage img;
    build_image(w, pl, img);
    int r;
    if (w.kind == TB_TOPO_GRAPH)
    {
        q.tables.reset(new tb_ctx);
        q.tables->device = v->device;
        if ((r = upload_graph(q.tables.get(), w, img.desc)))
            return r;
    }
    Sim &s = v->sim;
    std::vector<WorldDesc> desc(1, img.desc);
    std::vector<WorldCtl> wc(1);
    memset(&wc[0], 0, sizeof wc[0]);
    wc[0].next = gslot;
    wc[0].t0 = gslot;
    wc[0].wake = (unsigned long long)INT64_MAX;
    wc[0].act = wc[0].prev = 1;
    std::vector<unsigned long long> zero(EV_N, 0);
    if ((r = put(v, const_cast<WorldDesc *>(s.worlds) + wi, desc)) || (r = put(v, s.hosts + h0, img.hosts)) ||
        (r = put(v, s.sws + s0, img.sws)) || (r = put(v, s.ports + p0, img.ports)) || (r = put(v, const_cast<int *>(s.pend_msg) + m0, img.pend)) ||
        (r = put(v, s.snd + c0, img.snd)) || (r = put(v, s.rcv + c0, img.rcv)) || (r = put(v, s.msgs + m0, img.msgs)) ||
        (r = put(v, s.sw_rng + s0, img.rng)) || (r = put(v, s.ev_w + (size_t)wi * EV_N, zero)))
        return r;
    // its links' messages: no slot yet (host links, then port links)
    std::vector<int64_t> none_h(w.H1, -(1ll << 16)), none_p(P1, -(1ll << 16));
    for (int b = 0; b < NB; b++)
        if ((r = put(v, s.msg_tag + (size_t)b * s.L + h0, none_h)) || (r = put(v, s.msg_tag + (size_t)b * s.L + s.H + p0, none_p)))
            return r;
    if ((r = put(v, s.wctl + wi, wc)))
        return r;
    v->slot_req[wi] = q.id;
    v->units_stale = true;
    q.t0 = gslot;
    q.state = tb_server::RUNNING;
    q.t_admit = now_s();
    v->admitted++;
    return 1;
}

// reads a finished world's results and frees its place
int retire(tb_server *v, tb_server::Req &q, long long gslot)
{
    HostWorld &w = q.w;
    const Place &pl = q.pl;
    const int M = (int)w.rows.size();
    std::vector<MsgRec> m(M);
    q.ctr.assign(EV_N, 0);
    if ((M && cudaMemcpy(m.data(), v->sim.msgs + pl.msg0, sizeof(MsgRec) * M, cudaMemcpyDeviceToHost) != cudaSuccess) ||
        cudaMemcpy(q.ctr.data(), v->sim.ev_w + (size_t)pl.world * EV_N, 8 * EV_N, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaMemcpy failed");
    q.est.resize(M);
    q.done.resize(M);
    for (int i = 0; i < M; i++)
    {
        const MsgRec &x = m[w.row_msg[i]];
        q.est[i] = x.est >= 0 ? x.est / 1000 : -1;
        q.done[i] = x.done >= 0 ? x.done / 1000 : -1;
    }
    int r;
    if ((r = park(v, pl.host0, w.H1, pl.sw0, w.S1)))
        return r;
    const uint64_t P1 = (uint64_t)w.S1 * w.k;
    v->a_world.give(pl.world, 1);
    v->a_host.give(pl.host0, w.H1);
    v->a_sw.give(pl.sw0, w.S1);
    v->a_port.give(pl.port0, P1);
    v->a_conn.give(pl.conn0, w.conn_rows.size());
    v->a_msg.give(pl.msg0, w.rows.size());
    v->a_it.give(pl.it0, q.it_n);
    v->a_oo.give(pl.oo0, q.oo_n);
    v->slot_req[pl.world] = 0;
    v->units_stale = true;
    q.tables.reset();
    q.slots = gslot - q.t0;
    q.state = tb_server::DONE;
    q.t_done = now_s();
    v->retired++;
    return TB_OK;
}

// one round: admit what fits, run one launch, retire what finished. *running: requests in the
// batch afterwards. Called with the lock not held.
int serve_round(tb_server *v, int *running)
{
    Sim &s = v->sim;
    SlotCtl ctl{};
    if (cudaMemcpy(&ctl, s.ctl, sizeof ctl, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaMemcpy failed");
    const long long gslot = ctl.slot;
    int r = 0, in_batch = 0;
    {
        std::lock_guard<std::mutex> g(v->mu);
        // admissions, in arrival order with a bounded look-ahead past requests that do not fit
        int passed = 0;
        for (auto it = v->queue.begin(); it != v->queue.end() && passed < 64;)
        {
            tb_server::Req &q = *v->reqs[*it];
            int a = admit(v, q, gslot);
            if (a < 0)
            {
                q.state = tb_server::FAILED;
                q.error = g_err;
                it = v->queue.erase(it);
                continue;
            }
            if (a == 0)
            {
                passed++;
                ++it;
                continue;
            }
            it = v->queue.erase(it);
        }
        for (long long id : v->slot_req)
            in_batch += id != 0;
    }
    if (in_batch)
    {
        // the units of the worlds in the batch (free entities are not visited), for a shape's
        // hosts per warp; world slots in place order, so that host units come out ascending
        auto build_list = [&](int lanes) -> int {
            std::vector<std::array<int, 4>> wr(s.W, std::array<int, 4>{0, 0, 0, 0});
            std::vector<WorldCtl> live(s.W);
            {
                std::lock_guard<std::mutex> g(v->mu);
                for (int wi = 0; wi < s.W; wi++)
                {
                    live[wi].next = v->slot_req[wi] ? 0 : INT64_MAX;
                    if (v->slot_req[wi])
                    {
                        const tb_server::Req &q = *v->reqs[v->slot_req[wi]];
                        wr[wi] = {q.pl.host0, q.w.H1, q.pl.sw0, q.w.S1};
                    }
                }
            }
            std::vector<int> order(s.W);
            for (int i = 0; i < s.W; i++)
                order[i] = i;
            std::sort(order.begin(), order.end(), [&](int a, int b) { return wr[a][0] < wr[b][0]; });
            std::vector<std::array<int, 4>> wr2(s.W);
            std::vector<WorldCtl> live2(s.W);
            long long entities = 0;
            for (int i = 0; i < s.W; i++)
            {
                wr2[i] = wr[order[i]];
                live2[i] = live[order[i]];
                entities += wr2[i][1] + wr2[i][3];
            }
            v->batch_entities = entities;
            std::vector<int> ulist;
            running_units([&live2](size_t w) { return live2[w].next != INT64_MAX; }, wr2, lanes, s.H, ulist);
            if (!ulist.empty() &&
                cudaMemcpyAsync(v->d_units, ulist.data(), sizeof(int) * ulist.size(), cudaMemcpyHostToDevice, v->dev.stream) != cudaSuccess)
                return fail(TB_ERR_CUDA, "cudaMemcpyAsync failed");
            s.unit_list = v->d_units;
            s.n_list = (int)ulist.size();
            v->list_lanes = lanes;
            v->units_stale = false;
            return TB_OK;
        };
        // one launch of `slots` slots with shape k; *per_slot: its device ms per slot run
        long long before_all = ctl.slots_run;
        auto launch = [&](size_t k, int slots, double *per_slot) -> int {
            ShapeTuner::Shape &sh = v->tuner.shapes[k];
            if (v->units_stale || v->list_lanes != sh.lanes)
            {
                int rr = build_list(sh.lanes);
                if (rr)
                    return rr;
            }
            v->lanes = sh.lanes;
            v->stage = sh.stage;
            v->grid = grid_for(&v->dev, sh.lanes, sh.stage, s.n_list, sh.port_local);
            // the kernel stops early when every world in the batch is done
            ctl.finished = 0;
            if (cudaMemcpyAsync(&s.ctl->finished, &ctl.finished, sizeof(int), cudaMemcpyHostToDevice, v->dev.stream) != cudaSuccess)
                return fail(TB_ERR_CUDA, "cudaMemcpyAsync failed");
            const long long before = ctl.slots_run;
            cudaEventRecord(v->dev.la, v->dev.stream);
            int e = tb::launch_slots(s, v->grid, slots, sh.lanes, sh.stage, sh.port_local, v->dev.stream);
            if (e)
                return fail(TB_ERR_CUDA, std::string("slot kernel launch: ") + cudaGetErrorString((cudaError_t)e));
            cudaEventRecord(v->dev.lb, v->dev.stream);
            if (cudaMemcpyAsync(&ctl, s.ctl, sizeof ctl, cudaMemcpyDeviceToHost, v->dev.stream) != cudaSuccess ||
                cudaStreamSynchronize(v->dev.stream) != cudaSuccess)
                return fail(TB_ERR_CUDA, std::string("slot kernel: ") + cudaGetErrorString(cudaGetLastError()));
            if (ctl.error)
                return fail(TB_ERR_TIMEOUT, "a device-side barrier wait ran out");
            float ms = 0;
            cudaEventElapsedTime(&ms, v->dev.la, v->dev.lb);
            const long long ran = ctl.slots_run - before;
            sh.slots += ran;
            v->kernel_ms += ms;
            v->launches++;
            if (per_slot)
                *per_slot = ran >= v->tuner.probe / 2 ? ms / (double)ran : -1;
            return TB_OK;
        };
        if (v->tuner.explore())
        {
            std::vector<double> per_slot(v->tuner.shapes.size(), -1);
            for (size_t k = 0; k < v->tuner.shapes.size() && !ctl.finished; k++)
                if (v->tuner.probes(k) && (r = launch(k, v->tuner.probe, &per_slot[k])))
                    return r;
            v->tuner.decide(per_slot);
        }
        else
        {
            if ((r = launch(v->tuner.best, v->caps.slots_per_launch, nullptr)))
                return r;
            v->tuner.since++;
        }
        std::vector<WorldCtl> wc(s.W);
        std::vector<unsigned long long> ev(EV_N);
        if (cudaMemcpy(wc.data(), s.wctl, sizeof(WorldCtl) * s.W, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(ev.data(), s.ev, 8 * EV_N, cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(TB_ERR_CUDA, "cudaMemcpy failed");
        std::lock_guard<std::mutex> g(v->mu);
        v->slots_run += ctl.slots_run - before_all;
        v->events = ev[EV_HOST_PKT] + ev[EV_SW_PKT];
        for (int wi = 0; wi < s.W; wi++)
            if (v->slot_req[wi] && wc[wi].next == INT64_MAX)
            {
                tb_server::Req &q = *v->reqs[v->slot_req[wi]];
                if ((r = retire(v, q, ctl.slot)))
                    return r;
            }
        in_batch = 0;
        for (long long id : v->slot_req)
            in_batch += id != 0;
    }
    v->cv.notify_all();
    if (running)
        *running = in_batch;
    return TB_OK;
}

int server_alloc(tb_server *v)
{
    tb_ctx &c = v->dev;
    Sim &s = v->sim;
    const tb_serve_caps &k = v->caps;
    s = Sim{};
    s.W = k.worlds + 1;
    s.H = k.hosts;
    s.S = k.switches;
    s.P = k.ports;
    s.L = s.H + s.P;
    s.C = k.connections;
    s.M = k.messages;
    s.ring = k.max_queue + 2;
    s.kmax = k.max_ports;
    s.act_cap = k.active_per_host;
    s.max_slots = 1ll << 60;
    v->dead = k.worlds;
    int r;
    WorldDesc *wd;
    int *pend;
    if ((r = c.alloc(&wd, s.W, false)) || (r = c.alloc(&s.hosts, s.H, false)) || (r = c.alloc(&s.sws, s.S, false)) ||
        (r = c.alloc(&s.ports, s.P, false)) || (r = c.alloc(&pend, s.M, false)) || (r = c.alloc(&s.snd, s.C, false)) ||
        (r = c.alloc(&s.rcv, s.C, false)) || (r = c.alloc(&s.msgs, s.M, false)) ||
        (r = c.alloc(&s.host_ring, (size_t)s.H * s.ring, false)) || (r = c.alloc(&s.port_ring, (size_t)s.P * s.ring, false)) ||
        (r = c.alloc(&s.act_snd, (size_t)s.H * s.act_cap, false)) || (r = c.alloc(&s.act_rcv, (size_t)s.H * s.act_cap, false)) ||
        (r = c.alloc(&s.it_start, k.sent_list_entries, false)) || (r = c.alloc(&s.it_fl, k.sent_list_entries, false)) ||
        (r = c.alloc(&s.h_seq, k.sent_list_entries, false)) || (r = c.alloc(&s.h_end, k.sent_list_entries, false)) ||
        (r = c.alloc(&s.h_t, k.sent_list_entries, false)) || (r = c.alloc(&s.oo_s, k.ooo_blocks, false)) ||
        (r = c.alloc(&s.oo_e, k.ooo_blocks, false)) || (r = c.alloc(&s.msg, (size_t)NB * s.L * MAX_TX, false)) ||
        (r = c.alloc(&s.msg_tag, (size_t)NB * s.L, false)) || (r = c.alloc(&s.sw_rng, s.S, false)))
        return r;
    s.worlds = wd;
    s.pend_msg = pend;
    size_t per_sw = (size_t)s.kmax * 2 * MAX_TX;
    if ((r = c.alloc(&s.sw_ts, (size_t)s.S * per_sw, false)) || (r = c.alloc(&s.sw_ref, (size_t)s.S * per_sw, false)) ||
        (r = c.alloc(&s.sw_up, (size_t)s.S * per_sw, false)) || (r = c.alloc(&s.ev, EV_N, false)) ||
        (r = c.alloc(&s.ev_w, (size_t)s.W * EV_N, false)) || (r = c.alloc(&v->d_units, (size_t)s.H + s.S, false)))
        return r;
    {
        std::vector<double> tab(65536);
        for (size_t n = 0; n < tab.size(); n++)
            tab[n] = std::pow((double)n / 0.4, 1 / 3.);
        double *dt;
        if ((r = c.upload(&dt, tab, false)))
            return r;
        s.cub_k_tab = dt;
        s.cub_k_n = (int)tab.size();
    }
    {
        std::vector<SlotCtl> ctl(1);
        memset(&ctl[0], 0, sizeof(SlotCtl));
        ctl[0].next_wake = ~0ull;
        if ((r = c.upload(&s.ctl, ctl, false)))
            return r;
        std::vector<WorldCtl> wc(s.W);
        for (auto &x : wc)
        {
            memset(&x, 0, sizeof x);
            x.next = INT64_MAX; // free slots (and the dead world) never run
            x.wake = (unsigned long long)INT64_MAX;
        }
        if ((r = c.upload(&s.wctl, wc, false)))
            return r;
        std::vector<int64_t> tags((size_t)NB * s.L, -(1ll << 16));
        if (cudaMemcpy(s.msg_tag, tags.data(), 8 * tags.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(TB_ERR_CUDA, "cudaMemcpy failed");
    }
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaStreamCreate failed");
    cudaEventCreate(&c.ev0);
    cudaEventCreate(&c.ev1);
    cudaEventCreate(&c.la);
    cudaEventCreate(&c.lb);
    if ((r = park(v, 0, s.H, 0, s.S)))
        return r;
    cudaStreamSynchronize(c.stream);
    cudaDeviceGetAttribute(&c.dev_sms, cudaDevAttrMultiProcessorCount, v->device);
    c.sim = s;
    tuner_init(v->tuner, &c, true, 1, SW_STAGE, (long long)s.H + s.S);
    v->tuner.period = 8;
    v->tuner.probe = 32;
    v->lanes = v->tuner.shapes[v->tuner.best].lanes;
    v->stage = v->tuner.shapes[v->tuner.best].stage;
    if ((v->grid = grid_for(&c, v->lanes, v->stage)) <= 0)
        return fail(TB_ERR_CUDA, "the slot kernel does not fit on the device");
    v->a_world.init(k.worlds);
    v->a_host.init(k.hosts);
    v->a_sw.init(k.switches);
    v->a_port.init(k.ports);
    v->a_conn.init(k.connections);
    v->a_msg.init(k.messages);
    v->a_it.init(k.sent_list_entries);
    v->a_oo.init(k.ooo_blocks);
    v->slot_req.assign(s.W, 0);
    return TB_OK;
}
} // namespace

extern "C" {

int tb_server_create(int device, const tb_serve_caps *caps, tb_server **out)
{
    if (!caps || !out)
        return fail(TB_ERR_ARG, "caps and out are required");
    const tb_serve_caps &k = *caps;
    if (k.worlds < 1 || k.hosts < 1 || k.switches < 1 || k.ports < 1 || k.connections < 1 || k.messages < 1 || k.sent_list_entries < 1 ||
        k.ooo_blocks < 1 || k.active_per_host < 1 || k.max_queue < 1 || k.max_queue > 65000 || k.max_ports < 1 || k.max_ports > 32 ||
        k.slots_per_launch < 1)
        return fail(TB_ERR_ARG, "bad server capacities");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
        return fail(TB_ERR_CUDA, "no such CUDA device");
    if (cudaSetDevice(device) != cudaSuccess)
        return fail(TB_ERR_CUDA, "cudaSetDevice failed");
    std::unique_ptr<tb_server> v(new tb_server);
    v->device = device;
    v->caps = k;
    v->dev.device = device;
    v->dev.budget = k.hbm_budget_bytes;
    int r = server_alloc(v.get());
    if (r)
        return r;
    *out = v.release();
    return TB_OK;
}

int tb_server_destroy(tb_server *srv)
{
    if (!srv)
        return fail(TB_ERR_ARG, "srv is NULL");
    cudaSetDevice(srv->device);
    delete srv;
    return TB_OK;
}

int tb_server_submit_tcp(tb_server *srv, const tb_topology *topo, int n_flows, const int *src, const int *dst, const long long *size,
                         const long long *start_ns, const long long *conn, const tb_tcp_params *params, long long *request)
{
    if (!srv || !request)
        return fail(TB_ERR_ARG, "srv and request are required");
    std::unique_ptr<tb_server::Req> q(new tb_server::Req);
    q->t_submit = now_s();
    int r = make_world(topo, n_flows, src, dst, size, start_ns, conn, nullptr, nullptr, params, q->w);
    if (r)
        return r;
    ring_needs(q->w, q->it_n, q->oo_n);
    const tb_serve_caps &k = srv->caps;
    if (q->w.H1 > k.hosts || q->w.S1 > k.switches || (long long)q->w.S1 * q->w.k > k.ports ||
        (long long)q->w.conn_rows.size() > k.connections || (long long)q->w.rows.size() > k.messages || q->it_n > k.sent_list_entries ||
        q->oo_n > k.ooo_blocks || q->w.k > k.max_ports || q->w.p.queue > k.max_queue || most_active(q->w) > k.active_per_host)
        return fail(TB_ERR_MEMORY, "the request exceeds the server's capacities");
    std::lock_guard<std::mutex> g(srv->mu);
    q->id = srv->next_id++;
    *request = q->id;
    srv->queue.push_back(q->id);
    srv->reqs[q->id] = std::move(q);
    srv->cv.notify_all();
    return TB_OK;
}

int tb_server_step(tb_server *srv, int *running)
{
    if (!srv)
        return fail(TB_ERR_ARG, "srv is NULL");
    {
        std::lock_guard<std::mutex> g(srv->mu);
        if (srv->looping)
            return fail(TB_ERR_STATE, "the server's own loop is running");
    }
    cudaSetDevice(srv->device);
    return serve_round(srv, running);
}

int tb_server_start(tb_server *srv)
{
    if (!srv)
        return fail(TB_ERR_ARG, "srv is NULL");
    std::lock_guard<std::mutex> g(srv->mu);
    if (srv->looping)
        return TB_OK;
    srv->looping = true;
    srv->loop = std::thread([srv] {
        cudaSetDevice(srv->device);
        for (;;)
        {
            {
                std::unique_lock<std::mutex> l(srv->mu);
                srv->cv.wait(l, [srv] {
                    if (srv->stop)
                        return true;
                    if (!srv->queue.empty())
                        return true;
                    for (long long id : srv->slot_req)
                        if (id)
                            return true;
                    return false;
                });
                if (srv->stop)
                    return;
            }
            int running = 0;
            int r = serve_round(srv, &running);
            if (r)
            {
                std::lock_guard<std::mutex> l(srv->mu);
                srv->error = r;
                srv->error_text = g_err;
                srv->stop = true;
                srv->cv.notify_all();
                return;
            }
        }
    });
    return TB_OK;
}

int tb_server_wait(tb_server *srv, long long request, double timeout_s)
{
    if (!srv)
        return fail(TB_ERR_ARG, "srv is NULL");
    std::unique_lock<std::mutex> l(srv->mu);
    auto it = srv->reqs.find(request);
    if (it == srv->reqs.end())
        return fail(TB_ERR_ARG, "no such request");
    tb_server::Req *q = it->second.get();
    auto finished = [&] { return q->state == tb_server::DONE || q->state == tb_server::FAILED || srv->error; };
    if (timeout_s > 0)
    {
        if (!srv->cv.wait_for(l, std::chrono::duration<double>(timeout_s), finished))
            return fail(TB_ERR_TIMEOUT, "the request is not done yet");
    }
    else
        srv->cv.wait(l, finished);
    if (srv->error)
        return fail(srv->error, srv->error_text);
    if (q->state == tb_server::FAILED)
        return fail(TB_ERR_ARG, q->error);
    return TB_OK;
}

int tb_server_results(tb_server *srv, long long request, long long *established_ns, long long *completed_ns, unsigned long long *counters,
                      int n_counters, tb_request_info *info)
{
    if (!srv)
        return fail(TB_ERR_ARG, "srv is NULL");
    std::lock_guard<std::mutex> g(srv->mu);
    auto it = srv->reqs.find(request);
    if (it == srv->reqs.end())
        return fail(TB_ERR_ARG, "no such request");
    tb_server::Req &q = *it->second;
    if (info)
    {
        info->state = q.state;
        info->t_submit = q.t_submit;
        info->t_admit = q.t_admit;
        info->t_done = q.t_done;
        info->slot0 = q.t0;
        info->slots = q.slots;
        info->n_flows = (int)q.w.rows.size();
    }
    if (q.state != tb_server::DONE)
        return (established_ns || completed_ns || counters) ? fail(TB_ERR_STATE, "the request is not done") : TB_OK;
    for (size_t i = 0; i < q.est.size(); i++)
    {
        if (established_ns)
            established_ns[i] = q.est[i];
        if (completed_ns)
            completed_ns[i] = q.done[i];
    }
    for (int i = 0; counters && i < n_counters && i < EV_N; i++)
        counters[i] = q.ctr[i];
    return TB_OK;
}

int tb_server_release(tb_server *srv, long long request)
{
    if (!srv)
        return fail(TB_ERR_ARG, "srv is NULL");
    std::lock_guard<std::mutex> g(srv->mu);
    auto it = srv->reqs.find(request);
    if (it == srv->reqs.end())
        return fail(TB_ERR_ARG, "no such request");
    if (it->second->state == tb_server::RUNNING)
        return fail(TB_ERR_STATE, "the request is running");
    srv->queue.erase(std::remove(srv->queue.begin(), srv->queue.end(), request), srv->queue.end());
    srv->reqs.erase(it);
    return TB_OK;
}

int tb_server_stats(tb_server *srv, tb_serve_stats *out)
{
    if (!srv || !out)
        return fail(TB_ERR_ARG, "srv and out are required");
    std::lock_guard<std::mutex> g(srv->mu);
    memset(out, 0, sizeof *out);
    out->launches = srv->launches;
    out->slots_run = srv->slots_run;
    out->admitted = srv->admitted;
    out->retired = srv->retired;
    out->queued = (long long)srv->queue.size();
    out->kernel_ms = srv->kernel_ms;
    out->packet_events = srv->events;
    out->hbm_bytes = srv->dev.dev_bytes;
    out->host_lanes = srv->lanes;
    out->stage_frames = srv->stage;
    out->grid = srv->grid;
    for (long long id : srv->slot_req)
        out->running += id != 0;
    return TB_OK;
}

} // extern "C"
