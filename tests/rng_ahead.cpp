// The random stream's look-ahead (twins_b200/csrc/tb_common.cuh: make_rng_ahead, rng_ahead_value,
// u01_of), built with g++ by tests/test_sent_list.py: from random states, the m-th draw computed
// from the table must equal the m-th of the draws made one at a time (its output and its integer
// for every route count the switches use), and the state after m draws must equal the stream's, for
// every m of the table. Exit status 0: all agree.
#include <cstdint>
#include <cstdio>
#include <random>

#include "tb_common.cuh"

using namespace tb;

int main()
{
    static constexpr RngAhead T = make_rng_ahead();
    std::mt19937_64 g(11);
    for (int trial = 0; trial < 200; trial++)
    {
        Rng st;
        for (int c = 0; c < 6; c++)
            st.s[c] = (double)(g() % (c < 3 ? RNG_M1 : RNG_M2));
        if (trial == 0)
            for (int c = 0; c < 6; c++)
                st.s[c] = 12345.0; // ns-3's default seed
        Rng seq = st;
        for (int m = 1; m <= RNG_AHEAD; m++)
        {
            const double u = rand_u01(seq);
            const double p1 = rng_ahead_value<RNG_M1>(T.r[m], st.s), p2 = rng_ahead_value<RNG_M2>(T.r[m] + 3, st.s + 3);
            if (p1 != seq.s[2] || p2 != seq.s[5] || u01_of(p1, p2) != u)
            {
                printf("trial %d draw %d: %.0f %.0f, stream %.0f %.0f\n", trial, m, p1, p2, seq.s[2], seq.s[5]);
                return 1;
            }
            for (uint32_t n = 1; n <= 8; n++)
                if (int_of_u01(u01_of(p1, p2), n) != int_of_u01(u, n))
                    return 1;
            // the state after m draws: x_{m-2}, x_{m-1}, x_m of each component
            for (int c = 0; c < 6; c++)
            {
                const int e = m - 2 + c % 3;
                const double v = e <= 0 ? st.s[(c / 3) * 3 + e + 2]
                                        : (c < 3 ? rng_ahead_value<RNG_M1>(T.r[e], st.s) : rng_ahead_value<RNG_M2>(T.r[e] + 3, st.s + 3));
                if (v != seq.s[c])
                {
                    printf("trial %d after %d draws: state %d differs\n", trial, m, c);
                    return 1;
                }
            }
        }
    }
    puts("look-ahead: all agree");
    return 0;
}
