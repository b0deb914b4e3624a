"""The stage kernels' FMA-corrected divisions against IEEE division, on the CPU.

The FP64 path must reproduce the reference's `dt * (k1 + 2k2 + 2k3 + k4) / 6` and `derivative / h`
bit for bit, and the kernels form those quotients with Markstein's FMA corrections instead of a
division sequence (`div6` and `divBy` in csrc/stage2d.cuh).  This test restates both in C -- the
same constants, operations and guards -- and compares them bit for bit with IEEE division on
random and adversarial inputs in FP64 and FP32.  The host C library's fma() is correctly rounded,
as the device FMA is.
"""
import shutil
import subprocess

import pytest

SOURCE = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static double div6d(double y) {
    const double c = 1.0 / 3.0;
    const double x = y * 0.5, ax = fabs(x);
    if (!(ax <= 0x1p+1000) || (ax < 0x1p-960 && ax != 0)) return y / 6.0;
    const double q0 = x * c;
    const double r = fma(-q0, 3.0, x);
    return fma(r, c, q0);
}
static float div6f(float y) {
    const float c = 1.0f / 3.0f;
    const float x = y * 0.5f, ax = fabsf(x);
    if (!(ax <= 0x1p+120f) || (ax < 0x1p-100f && ax != 0)) return y / 6.0f;
    const float q0 = x * c;
    const float r = fmaf(-q0, 3.0f, x);
    return fmaf(r, c, q0);
}
static double __attribute__((noinline)) plain_div(double x, double d) { return x / d; }
static double divby(double x, double d, double dinv) {
    const double ax = fabs(x);
    if (!(ax <= 0x1p+1000) || (ax < 0x1p-960 && ax != 0)) return plain_div(x, d);
    const double q0 = x * dinv;
    const double q1 = fma(fma(-q0, d, x), dinv, q0);
    return fma(fma(-q1, d, x), dinv, q1);
}
static float divbyf(float x, float d, float dinv) {
    const float ax = fabsf(x);
    if (!(ax <= 0x1p+100f) || (ax < 0x1p-100f && ax != 0)) return x / d;
    const float q0 = x * dinv;
    const float q1 = fmaf(fmaf(-q0, d, x), dinv, q0);
    return fmaf(fmaf(-q1, d, x), dinv, q1);
}
static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint64_t next(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
/* equal bit for bit, or equal as values when both are zero (the sign of a zero may differ) */
static int same_d(double a, double b) {
    if (isnan(a) || isnan(b)) return isnan(a) && isnan(b);
    if (a == 0 && b == 0) return 1;
    return memcmp(&a, &b, sizeof a) == 0;
}
static int same_f(float a, float b) {
    if (isnan(a) || isnan(b)) return isnan(a) && isnan(b);
    if (a == 0 && b == 0) return 1;
    return memcmp(&a, &b, sizeof a) == 0;
}
int main(void) {
    long bad = 0, n = 0;
    for (long i = 0; i < 4000000; ++i) { /* uniform bit patterns: every exponent */
        uint64_t b = next(); double y; memcpy(&y, &b, 8);
        bad += !same_d(div6d(y), y / 6.0), ++n;
        uint32_t c = (uint32_t)(b >> 17); float f; memcpy(&f, &c, 4);
        bad += !same_f(div6f(f), f / 6.0f), ++n;
    }
    for (long i = 0; i < 4000000; ++i) { /* sparse mantissas: exact multiples and near-halfway quotients */
        uint64_t m = (1ull << 52) | (next() & next() & next() & ((1ull << 52) - 1));
        m ^= (next() & 7);
        int e = (int)(next() % 200) - 100;
        double y = ldexp((double)m, e - 52) * ((next() & 1) ? 1 : -1);
        bad += !same_d(div6d(y), y / 6.0), ++n;
        bad += !same_d(div6d(3 * y), 3 * y / 6.0), ++n;
        float f = (float)y;
        bad += !same_f(div6f(f), f / 6.0f), ++n;
        bad += !same_f(div6f(3 * f), 3 * f / 6.0f), ++n;
    }
    for (long i = 0; i < 4000000; ++i) { /* physical magnitudes: velocity / stress increments */
        double y = ldexp((double)(next() >> 11), -53) * ldexp(1.0, (int)(next() % 80) - 60);
        bad += !same_d(div6d(y), y / 6.0), ++n;
        float f = (float)y;
        bad += !same_f(div6f(f), f / 6.0f), ++n;
    }
    const double edges[] = {0x1p-960, 0x1p-960 * 0.75, 0x1p-959, 0x1p+1000, 0x1p+1001, 0.0, -0.0, 1.0 / 0.0, -1.0 / 0.0,
                            6.0, 3.0, 1.5, 0x1.fffffffffffffp-1, 0x1.0000000000001p+0, 4.9406564584124654e-324};
    for (unsigned i = 0; i < sizeof edges / sizeof edges[0]; ++i)
        for (int sg = -1; sg <= 1; sg += 2) {
            const double y = sg * edges[i];
            bad += !same_d(div6d(y), y / 6.0), ++n;
            bad += !same_f(div6f((float)y), (float)y / 6.0f), ++n;
        }
    /* x / d for grid spacings (fixed and random in [2^-20, 2^20]) and random numerators */
    const double spacings[] = {10.0, 2.5, 3.0, 7.0, 0.3, 1.7, 12.5, 0.1, 5.0, 0x1p-20, 0x1p+20};
    for (long i = 0; i < 6000000; ++i) {
        double d;
        if (i % 3 == 0) d = spacings[next() % (sizeof spacings / sizeof spacings[0])];
        else d = ldexp(1.0 + ldexp((double)(next() >> 12), -52), (int)(next() % 41) - 20);
        const double dinv = 1.0 / d;
        uint64_t b = next(); double x;
        if (i & 1) memcpy(&x, &b, 8); /* every exponent */
        else x = ldexp((double)(b >> 11), -53) * ldexp(1.0, (int)(next() % 120) - 60);
        bad += !same_d(divby(x, d, dinv), x / d), ++n;
        const float df = (float)d, dinvf = 1.0f / df;
        uint32_t c = (uint32_t)(b >> 17); float xf; memcpy(&xf, &c, 4);
        if (fabsf(df) >= 0x1p-20f && fabsf(df) <= 0x1p+20f) bad += !same_f(divbyf(xf, df, dinvf), xf / df), ++n;
    }
    printf("%ld %ld\n", bad, n);
    return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_fma_divisions_are_correctly_rounded(tmp_path):
    src = tmp_path / "div6.c"
    exe = tmp_path / "div6"
    src.write_text(SOURCE)
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-o", str(exe), str(src), "-lm"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    bad, n = map(int, out.stdout.split())
    assert n > 40_000_000
    assert bad == 0, out.stdout
