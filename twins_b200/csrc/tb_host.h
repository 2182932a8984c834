// twins-b200: host-side launch logic with no CUDA in it (plain C++17): the launch shapes' staging
// sizes, the grid of a shape, the running units of a batch, the launch-shape tuner, and the
// server's first-fit ranges. The C ABI (tb_capi.cu, tb_serve.cuh) drives these between launches.
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <iterator>
#include <map>
#include <vector>

#ifndef TB_CHAIN_RUNS
#define TB_CHAIN_RUNS 9
#endif

namespace tb
{

// frames a warp stages in shared memory per switch (or host) and slot: the default staging area
// and the largest; a launch may use a smaller one (more resident warps per SM, fewer slots
// staged) or a larger one (big switches' slots staged, fewer resident warps)
constexpr int SW_STAGE = 192;
constexpr int SW_STAGE_MAX = TB_CHAIN_RUNS > 9 ? 256 : 384; // (what four warps' scratch fits in 227 KB)
constexpr int SW_STAGE_SMALL = 96;
constexpr int SW_STAGE_TWO = 288; // the most with which two blocks of four warps fit on an SM

// the grid of a launch: a block per `warps` units, at most what is co-resident (per_sm blocks on
// each of sms SMs; 0: the shape does not fit), or the caller's grid when it asked for one
inline int grid_of(long long units, int warps, int per_sm, int sms, int grid_req)
{
    if (per_sm <= 0 || sms <= 0)
        return 0;
    const long long need = std::max(1LL, (units + warps - 1) / warps);
    const int most = sms * per_sm;
    return grid_req > 0 ? std::min(grid_req, most) : (int)std::min<long long>(need, most);
}

// The units of a batch's running worlds, ascending: host units (`lanes` hosts each; a unit that
// holds hosts of two worlds appears once, while either runs), then one unit per switch after
// all host units. worlds[w] = {first host, hosts, first switch, switches}; alive(w) whether
// world w still runs; H the batch's hosts.
template <class Alive>
void running_units(Alive alive, const std::vector<std::array<int, 4>> &worlds, int lanes, int H, std::vector<int> &out)
{
    out.clear();
    const int host_units = (H + lanes - 1) / lanes;
    for (size_t w = 0; w < worlds.size(); w++)
    {
        if (!alive(w) || worlds[w][1] == 0)
            continue;
        for (int u = worlds[w][0] / lanes; u <= (worlds[w][0] + worlds[w][1] - 1) / lanes; u++)
            if (out.empty() || out.back() < u)
                out.push_back(u);
    }
    for (size_t w = 0; w < worlds.size(); w++)
        if (alive(w))
            for (int x = 0; x < worlds[w][3]; x++)
                out.push_back(host_units + worlds[w][2] + x);
}

// The units of a batch's running worlds for a launch without a grid barrier: per running world
// its host units (the first host of up to `lanes` consecutive hosts of that world, never of two)
// and its switches (H + switch); counts[w] the units of world w (0: it does not run).
template <class Alive>
void world_units(Alive alive, const std::vector<std::array<int, 4>> &worlds, int lanes, int H, std::vector<int> &out,
                 std::vector<unsigned> &counts)
{
    out.clear();
    counts.assign(worlds.size(), 0);
    for (size_t w = 0; w < worlds.size(); w++)
    {
        if (!alive(w))
            continue;
        const size_t first = out.size();
        for (int h = worlds[w][0]; h < worlds[w][0] + worlds[w][1]; h += lanes)
            out.push_back(h);
        for (int x = 0; x < worlds[w][3]; x++)
            out.push_back(H + worlds[w][2] + x);
        counts[w] = (unsigned)(out.size() - first);
    }
}

// Launch-shape autotuning, for tb_run and the server. A shape is the hosts per warp, the frames a
// warp stages per slot and the switch egress variant; no shape changes a result. It starts from
// one host per warp while the entities fit the resident warps about twice (latency-bound: each
// host's serial events are the slot's critical path), else 32 hosts per warp (throughput-bound:
// the lanes' memory accesses overlap). Every `period` launches each shape still in the running
// runs a probe of `probe` slots, and one whose device time per slot beats the current one's by
// more than 5% takes over; a shape that loses a probe by more than 30% twice, or by more than 60%
// once, is not probed again until every fourth round of probes, which probes all shapes (the load changes along a run).
// With backoff, a round that keeps the shape doubles the period (up to a bound: probes of losing
// shapes cost time), and a new shape or a change of the load (load_changed) restores it; a change
// of the load also clears the strikes.
struct ShapeTuner
{
    struct Shape
    {
        int lanes, stage;
        long long slots;
        int strikes;
        bool port_local; // switch ports' slot copies in shared memory (PortEgress)
    };
    std::vector<Shape> shapes;
    size_t best = 0;
    long long since = 0, rounds = 0;
    int period = 12, probe = 128;
    int period0 = 12, most_period = 0; // (backoff: the first period and the bound; 0: none)

    // the candidates: (lanes, stage, port-local)
    static constexpr int N_CAND = 9;
    static constexpr int CAND[N_CAND][3] = {{1, SW_STAGE_TWO, 0},  {1, SW_STAGE, 0},       {4, SW_STAGE, 0},
                                            {32, SW_STAGE, 0},     {1, SW_STAGE_SMALL, 0}, {32, SW_STAGE_SMALL, 0},
                                            {1, SW_STAGE_MAX, 0},  {1, SW_STAGE_MAX, 1},   {1, SW_STAGE_TWO - 32, 1}};

    // autotune: probe the candidates that fit (fits(lanes, stage, port_local) on this device),
    // else run the one shape (lanes, stage, port_local). entities: hosts and switches to run;
    // resident: the warps co-resident on the device at one host per warp and the default
    // staging; kmax: the most ports a switch has.
    template <class Fits>
    void init(bool autotune, int lanes, int stage, bool port_local, long long entities, int kmax, long long resident, Fits fits)
    {
        shapes.clear();
        best = 0;
        since = 0;
        rounds = 0;
        if (autotune)
        {
            for (auto &x : CAND)
                if (fits(x[0], x[1], x[2] != 0))
                    shapes.push_back({x[0], x[1], 0, 0, x[2] != 0});
            // (one host per warp: with big switches (16 ports or more), whose ports' serial
            // enqueues are the critical path, the port-local egress and the largest staging; else
            // the largest staging that keeps two blocks per SM. 32 hosts per warp: the smallest
            // staging, for four blocks per SM)
            const int lanes0 = entities <= 2 * resident ? 1 : 32;
            const bool pl0 = lanes0 == 1 && kmax >= 16;
            const int stage0 = lanes0 == 1 ? (pl0 ? SW_STAGE_MAX : SW_STAGE_TWO) : SW_STAGE_SMALL;
            for (size_t k = 0; k < shapes.size(); k++)
                if (shapes[k].lanes == lanes0 && shapes[k].stage == stage0 && shapes[k].port_local == pl0)
                    best = k;
        }
        if (shapes.empty())
            shapes.push_back({lanes, stage, 0, 0, port_local});
    }
    // the period doubles after each round that keeps the shape, up to `most` launches
    void backoff(int most)
    {
        period0 = period;
        most_period = most;
    }
    // the running worlds' entities changed much: earlier losses say little now; probe every shape
    // again, at the first period
    void load_changed()
    {
        if (most_period > 0)
            period = period0;
        for (auto &x : shapes)
            x.strikes = 0;
    }
    bool explore() const { return shapes.size() > 1 && since >= period; }
    bool probes(size_t k) const { return k == best || shapes[k].strikes < 2; }
    // after a round of probes (per_slot[k]: ms per slot, <= 0 where no probe ran)
    void decide(const std::vector<double> &per_slot)
    {
        size_t b = best;
        for (size_t k = 0; k < shapes.size(); k++)
            if (per_slot[k] > 0 && (per_slot[b] <= 0 || per_slot[k] < 0.95 * per_slot[b]))
                b = k;
        for (size_t k = 0; k < shapes.size(); k++)
            if (per_slot[k] > 0 && per_slot[b] > 0 && per_slot[k] > 1.3 * per_slot[b])
                shapes[k].strikes += per_slot[k] > 1.6 * per_slot[b] ? 2 : 1;
        if (most_period > 0)
            period = b == best ? std::min(2 * period, most_period) : period0;
        best = b;
        since = 0;
        if (++rounds % 4 == 0)
            for (auto &x : shapes)
                x.strikes = 0;
    }
    // the shape that ran the most slots
    size_t most() const
    {
        size_t m = 0;
        for (size_t k = 1; k < shapes.size(); k++)
            if (shapes[k].slots > shapes[m].slots)
                m = k;
        return m;
    }
};

// first-fit ranges of [0, cap): the server's entities, connections, messages and ring entries
struct RangeAlloc
{
    std::map<uint64_t, uint64_t> free_; // start -> length, no two adjacent
    uint64_t cap = 0, used = 0;
    void init(uint64_t n)
    {
        cap = n;
        used = 0;
        free_.clear();
        if (n)
            free_[0] = n;
    }
    // the start of n free entries (the lowest that fits), or -1
    long long take(uint64_t n)
    {
        if (n == 0)
            return 0;
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n)
            {
                uint64_t at = it->first, len = it->second;
                free_.erase(it);
                if (len > n)
                    free_[at + n] = len - n;
                used += n;
                return (long long)at;
            }
        return -1;
    }
    // returns [at, at + n), which take() gave out, merging it with free neighbours
    void give(uint64_t at, uint64_t n)
    {
        if (n == 0)
            return;
        used -= n;
        auto next = free_.lower_bound(at);
        if (next != free_.begin())
        {
            auto prev = std::prev(next);
            if (prev->first + prev->second == at)
            {
                at = prev->first;
                n += prev->second;
                free_.erase(prev);
            }
        }
        next = free_.lower_bound(at);
        if (next != free_.end() && at + n == next->first)
        {
            n += next->second;
            free_.erase(next);
        }
        free_[at] = n;
    }
};

} // namespace tb
