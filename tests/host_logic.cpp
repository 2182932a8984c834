// A C shim over the library's host-side launch logic (twins_b200/csrc/tb_host.h), built by
// tests/test_host_logic.py with g++ so that the tuner, the unit lists, the grid rule and the
// server's ranges are tested on the CPU with ctypes.
#include "tb_host.h"

using namespace tb;

extern "C" {

int hl_stage(int which)
{
    const int v[4] = {SW_STAGE_SMALL, SW_STAGE, SW_STAGE_TWO, SW_STAGE_MAX};
    return v[which];
}

int hl_n_cand() { return ShapeTuner::N_CAND; }

void hl_cand(int k, int *out)
{
    for (int i = 0; i < 3; i++)
        out[i] = ShapeTuner::CAND[k][i];
}

int hl_grid_of(long long units, int warps, int per_sm, int sms, int grid_req) { return grid_of(units, warps, per_sm, sms, grid_req); }

int hl_running_units(const int *alive, const int *worlds, int W, int lanes, int H, int *out, int cap)
{
    std::vector<std::array<int, 4>> wr(W);
    for (int w = 0; w < W; w++)
        wr[w] = {worlds[4 * w], worlds[4 * w + 1], worlds[4 * w + 2], worlds[4 * w + 3]};
    std::vector<int> v;
    running_units([alive](size_t w) { return alive[w] != 0; }, wr, lanes, H, v);
    for (size_t i = 0; i < v.size() && (int)i < cap; i++)
        out[i] = v[i];
    return (int)v.size();
}

void *hl_tuner(int autotune, int lanes, int stage, int port_local, long long entities, int kmax, long long resident, unsigned fits_mask)
{
    auto *t = new ShapeTuner;
    t->init(autotune != 0, lanes, stage, port_local != 0, entities, kmax, resident, [fits_mask](int l, int st, bool pl) {
        for (int k = 0; k < ShapeTuner::N_CAND; k++)
            if (ShapeTuner::CAND[k][0] == l && ShapeTuner::CAND[k][1] == st && (ShapeTuner::CAND[k][2] != 0) == pl)
                return ((fits_mask >> k) & 1) != 0;
        return false;
    });
    return t;
}

void hl_tuner_free(void *t) { delete (ShapeTuner *)t; }
int hl_tuner_n(void *t) { return (int)((ShapeTuner *)t)->shapes.size(); }

// (lanes, stage, port_local, strikes)
void hl_tuner_shape(void *t, int k, int *out)
{
    const ShapeTuner::Shape &s = ((ShapeTuner *)t)->shapes[k];
    out[0] = s.lanes;
    out[1] = s.stage;
    out[2] = s.port_local;
    out[3] = s.strikes;
}

int hl_tuner_best(void *t) { return (int)((ShapeTuner *)t)->best; }
int hl_tuner_explore(void *t) { return ((ShapeTuner *)t)->explore(); }
int hl_tuner_probes(void *t, int k) { return ((ShapeTuner *)t)->probes(k); }
int hl_tuner_period(void *t) { return ((ShapeTuner *)t)->period; }
void hl_tuner_backoff(void *t, int most) { ((ShapeTuner *)t)->backoff(most); }
void hl_tuner_load_changed(void *t) { ((ShapeTuner *)t)->load_changed(); }
void hl_tuner_tick(void *t) { ((ShapeTuner *)t)->since++; }
void hl_tuner_add_slots(void *t, int k, long long n) { ((ShapeTuner *)t)->shapes[k].slots += n; }
int hl_tuner_most(void *t) { return (int)((ShapeTuner *)t)->most(); }

void hl_tuner_decide(void *t, const double *per_slot)
{
    ShapeTuner *u = (ShapeTuner *)t;
    u->decide(std::vector<double>(per_slot, per_slot + u->shapes.size()));
}

void *hl_ranges(unsigned long long cap)
{
    auto *r = new RangeAlloc;
    r->init(cap);
    return r;
}

void hl_ranges_free(void *r) { delete (RangeAlloc *)r; }
long long hl_take(void *r, unsigned long long n) { return ((RangeAlloc *)r)->take(n); }
void hl_give(void *r, unsigned long long at, unsigned long long n) { ((RangeAlloc *)r)->give(at, n); }
unsigned long long hl_used(void *r) { return ((RangeAlloc *)r)->used; }

// the free ranges, ascending: (start, length) pairs
int hl_free_ranges(void *r, unsigned long long *out, int cap)
{
    int n = 0;
    for (auto &x : ((RangeAlloc *)r)->free_)
    {
        if (n < cap)
        {
            out[2 * n] = x.first;
            out[2 * n + 1] = x.second;
        }
        n++;
    }
    return n;
}
}
