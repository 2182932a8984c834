// twins-b200: the state of an ns-3 MRG32k3a random stream (RngStream) at set-up, on the host:
// stream n of run r under seed s is the seed vector advanced by A^((2^63 + n) 2^127 + r 2^76).
// Used by the TCP path (per-switch spraying streams) and the RDMA path (per-port ECN streams).
#pragma once
#include "tb_common.cuh"

#include <cstdint>

namespace tb
{
namespace rng_host
{
typedef unsigned __int128 u128;
struct M3
{
    uint64_t a[3][3];
};
inline M3 mmul(const M3 &x, const M3 &y, uint64_t m)
{
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
        {
            u128 v = 0;
            for (int t = 0; t < 3; t++)
                v += (u128)x.a[i][t] * y.a[t][j] % m;
            r.a[i][j] = (uint64_t)(v % m);
        }
    return r;
}
inline void mvec(const M3 &x, uint64_t v[3], uint64_t m)
{
    uint64_t r[3];
    for (int i = 0; i < 3; i++)
    {
        u128 s = 0;
        for (int t = 0; t < 3; t++)
            s += (u128)x.a[i][t] * v[t] % m;
        r[i] = (uint64_t)(s % m);
    }
    memcpy(v, r, sizeof r);
}
// the state of ns-3 stream SetStream(stream) under RngSeed seed and RngRun run: the seed vector
// advanced by A^((2^63 + stream) 2^127 + run 2^76) (RngStream's AdvanceNthBy)
struct RngPowers
{
    M3 p127[64], p76[64];
    uint64_t m;
    RngPowers(const M3 &a, uint64_t m_) : m(m_)
    {
        M3 x = a;
        for (int i = 0; i < 76; i++)
            x = mmul(x, x, m);
        for (int b = 0; b < 64; b++)
        {
            p76[b] = x;
            x = mmul(x, x, m);
        }
        x = a;
        for (int i = 0; i < 127; i++)
            x = mmul(x, x, m);
        for (int b = 0; b < 64; b++)
        {
            p127[b] = x;
            x = mmul(x, x, m);
        }
    }
    void advance(uint64_t nth, bool by127, uint64_t v[3]) const
    {
        for (int b = 0; b < 64; b++)
            if ((nth >> b) & 1)
                mvec(by127 ? p127[b] : p76[b], v, m);
    }
};
inline Rng stream_state(uint32_t seed, uint64_t stream, uint64_t run)
{
    const uint64_t m1 = 4294967087ull, m2 = 4294944443ull;
    static const RngPowers P1({{{0, 1, 0}, {0, 0, 1}, {m1 - 810728, 1403580, 0}}}, m1);
    static const RngPowers P2({{{0, 1, 0}, {0, 0, 1}, {m2 - 1370589, 0, 527612}}}, m2);
    uint64_t v1[3] = {seed, seed, seed}, v2[3] = {seed, seed, seed};
    uint64_t target = (1ull << 63) + stream;
    P1.advance(target, true, v1);
    P2.advance(target, true, v2);
    P1.advance(run, false, v1);
    P2.advance(run, false, v2);
    Rng r;
    for (int i = 0; i < 3; i++)
    {
        r.s[i] = (double)v1[i];
        r.s[3 + i] = (double)v2[i];
    }
    return r;
}

} // namespace rng_host
using rng_host::stream_state;
} // namespace tb
