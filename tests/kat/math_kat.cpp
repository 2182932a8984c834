// Known-answer checks of the product's arithmetic (twins_b200/csrc/tb_common.cuh, built for the
// host) against independent forms: ns-3's GetSeconds through x87 long double, RngStream's
// division-based recurrence, the host libm's pow (the function ns-3 calls). Prints one line of
// counts; tests/test_math_kat.py asserts on them.
#include "../../twins_b200/csrc/tb_common.cuh"
#include <cmath>
#include <cstdio>
#include <random>
using namespace tb;

static double seconds_x87(int64_t ps)
{
    if (ps == 0)
        return 0.0;
    bool neg = ps < 0;
    u128 a = neg ? (u128)(-(__int128)ps) : (u128)ps;
    u128 v = a * INV_1E12_HI + ((a * INV_1E12_LO) >> 64);
    long double hi = (long double)(uint64_t)(v >> 64), lo = (long double)(uint64_t)v / 18446744073709551616.0L;
    long double r = hi;
    r += lo;
    return (double)(neg ? -r : r);
}

// RngStream::RandU01 with its divisions (L'Ecuyer's published form)
static double u01_div(double *s)
{
    const double m1 = 4294967087.0, m2 = 4294944443.0, norm = 1.0 / (4294967087.0 + 1.0);
    double p1 = 1403580.0 * s[1] - 810728.0 * s[0];
    int32_t k = (int32_t)(p1 / m1);
    p1 -= k * m1;
    if (p1 < 0.0)
        p1 += m1;
    s[0] = s[1], s[1] = s[2], s[2] = p1;
    double p2 = 527612.0 * s[5] - 1370589.0 * s[3];
    k = (int32_t)(p2 / m2);
    p2 -= k * m2;
    if (p2 < 0.0)
        p2 += m2;
    s[3] = s[4], s[4] = s[5], s[5] = p2;
    return p1 > p2 ? (p1 - p2) * norm : (p1 - p2 + m1) * norm;
}

int main()
{
    std::mt19937_64 g(12345);
    long sec_bad = 0, sec_n = 2000000;
    for (long i = 0; i < sec_n; i++)
    {
        int64_t ps = (int64_t)(g() % 40000000000000ull) - (i % 5 == 0 ? 20000000000000ll : 0);
        sec_bad += get_seconds(ps) != seconds_x87(ps);
    }
    long rng_bad = 0, rng_n = 0;
    for (int st = 0; st < 200; st++)
    {
        Rng r;
        double s[6];
        for (int j = 0; j < 6; j++)
            r.s[j] = s[j] = (double)(g() % (j < 3 ? 4294967087ull : 4294944443ull));
        for (int i = 0; i < 20000; i++, rng_n++)
            rng_bad += rand_u01(r) != u01_div(s);
    }
    std::uniform_real_distribution<double> U(0, 1);
    long root_bad = 0, cube_bad = 0, trunc_bad = 0, kin_bad = 0, n = 1000000, kin_n = 0;
    for (long i = 0; i < n; i++)
    {
        double x = std::exp(U(g) * 30 - 10);
        root_bad += tb_pow(x, 1 / 3.) != std::pow(x, 1 / 3.);
        double o = U(g) * 5;
        double a = tb_pow(o, 3), b = std::pow(o, 3);
        cube_bad += a != b;
        trunc_bad += (uint32_t)(int64_t)(0.4 * a) != (uint32_t)(int64_t)(0.4 * b);
    }
    for (uint32_t d = 1; d < 65536; d++, kin_n++)
        kin_bad += tb_pow((double)d / 0.4, 1 / 3.) != std::pow((double)d / 0.4, 1 / 3.);
    printf("seconds %ld %ld rng %ld %ld root %ld %ld cube %ld %ld trunc %ld %ld kinputs %ld %ld\n", sec_bad, sec_n, rng_bad, rng_n,
           root_bad, n, cube_bad, n, trunc_bad, n, kin_bad, kin_n);
    return 0;
}
