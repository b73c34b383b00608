/* The quotient algorithms of the device code, restated in C for a CPU check
 * against IEEE division (tests/test_div_rn.py compiles and runs this):
 *   div_rn          a / b from y = RN(1/b) with two FMA corrections
 *                   (Markstein's theorem), as eilmer4_b200/csrc/e4c_thermo.cuh;
 *   quotient_below  RN(d / a) < tol decided against RN(tol a) with a 2^-49
 *                   band, as eilmer4_b200/csrc/e4c_physics.cuh.
 * usage: div_rn_check <samples>; prints the mismatch counts, exits 1 on any. */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

static double div_rn(double a, double b, double y) {
    double q = a * y;
    double r = fma(-q, b, a);
    q = fma(r, y, q);
    r = fma(-q, b, a);
    q = fma(r, y, q);
    return a == 0.0 ? a * y : q;
}

static int quotient_below(double d, double a, double tol) {
    const double P = tol * a;
    const double band = fabs(P) * 0x1p-49;
    if (a > 0.0 && tol != 0.0 && fabs(P) >= 0x1p-1000 && fabs(P) <= DBL_MAX && fabs(d) <= DBL_MAX) {
        if (d < P - band) return 1;
        if (d > P + band) return 0;
    }
    return (d / a) < tol;
}

static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint64_t next(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
static double u01(void) { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }

int main(int argc, char** argv) {
    const long n = argc > 1 ? atol(argv[1]) : 1000000;
    long bad_div = 0, bad_cmp = 0;
    for (long i = 0; i < n; ++i) {
        /* divisors as the CEA curves use them: T, T^2, 3, 5, and wide-range values */
        double b;
        switch (i % 5) {
            case 0: b = 20.0 + 1.0e5 * u01(); break;
            case 1: { const double t = 20.0 + 1.0e5 * u01(); b = t * t; break; }
            case 2: b = 3.0; break;
            case 3: b = 5.0; break;
            default: b = ldexp(1.0 + u01(), (int)(next() % 400) - 200); break;
        }
        double a = ldexp(1.0 + u01(), (int)(next() % 200) - 100) * ((next() & 1) ? 1.0 : -1.0);
        if ((next() & 7) == 0) a = ldexp(2.0 - ldexp(u01(), -45), (int)(next() % 60) - 30);
        if ((next() & 63) == 0) a = (next() & 1) ? 0.0 : -0.0;
        const double q = div_rn(a, b, 1.0 / b), t = a / b;
        if (q != t || signbit(q) != signbit(t)) ++bad_div;
        /* compression tests near the threshold tol a */
        const double tol = (i % 3 == 0) ? -0.3 : ((i % 3 == 1) ? -0.05 : 0.2);
        const double as = 50.0 + 2000.0 * u01();
        double d = tol * as * (1.0 + (u01() - 0.5) * ldexp(1.0, -(int)(next() % 60)));
        if (next() & 1) d = nextafter(d, (next() & 1) ? INFINITY : -INFINITY);
        if ((next() & 15) == 0) d = (u01() - 0.5) * 4000.0;
        if (quotient_below(d, as, tol) != ((d / as) < tol)) ++bad_cmp;
    }
    printf("samples %ld div_rn mismatches %ld quotient_below mismatches %ld\n", n, bad_div, bad_cmp);
    return (bad_div || bad_cmp) ? 1 : 0;
}
