// Per-population features of one SNP pair on the haplotype path.
#pragma once
#include "ldk_common.cuh"

template <typename T>
struct HapFeat {
    // two-locus counts n11, n10, n01, n00 (pg_gpu ld_statistics.py:281-290), their sum ns
    // and the sample size n used in denominators (n_valid; equal to ns for haplotypes)
    T c1, c2, c3, c4, ns, n;
    T pA, qA, pB, qB, E, a, b, s, fA, fB;
    T Q1, Q2, Q3, Q4, L1, L2, L3, L4, T1, T2;
    T DDs, DZs, PIs;
    // guarded reciprocals of n, n(n-1), n(n-1)(n-2), n(n-1)(n-2)(n-3): 0 where the product
    // is 0, reproducing the reference's ``den > 0 ? num / den : 0`` (haplotype_kernels.py:78)
    T r1, r2, r3, r4;
};

template <typename T>
LDK_DEV void hap_reciprocals(HapFeat<T>& x) {
    const T n = x.n;
    if (n >= T(4)) {
        const T r4 = T(1) / (n * (n - T(1)) * (n - T(2)) * (n - T(3)));
        x.r4 = r4;
        x.r3 = r4 * (n - T(3));
        x.r2 = x.r3 * (n - T(2));
        x.r1 = x.r2 * (n - T(1));
    } else {
        x.r4 = T(0);
        x.r3 = (n >= T(3)) ? T(1) / (n * (n - T(1)) * (n - T(2))) : T(0);
        x.r2 = (n >= T(2)) ? T(1) / (n * (n - T(1))) : T(0);
        x.r1 = (n >= T(1)) ? T(1) / n : T(0);
    }
}

// Reciprocal table entry for sample size n: {1/n, 1/(n(n-1)), 1/(n(n-1)(n-2)),
// 1/(n(n-1)(n-2)(n-3))}, each 0 where its product is 0 (built once per CTA).
LDK_DEV double4 recip_entry(int n) {
    const double d = (double)n;
    double4 r;
    r.x = n >= 1 ? 1.0 / d : 0.0;
    r.y = n >= 2 ? 1.0 / (d * (d - 1.0)) : 0.0;
    r.z = n >= 3 ? 1.0 / (d * (d - 1.0) * (d - 2.0)) : 0.0;
    r.w = n >= 4 ? 1.0 / (d * (d - 1.0) * (d - 2.0) * (d - 3.0)) : 0.0;
    return r;
}

template <typename T>
LDK_DEV void hap_reciprocals_from(HapFeat<T>& x, const double4& r) {
    x.r1 = T(r.x);
    x.r2 = T(r.y);
    x.r3 = T(r.z);
    x.r4 = T(r.w);
}

template <typename T>
LDK_DEV void hap_set_counts(HapFeat<T>& x, T c1, T c2, T c3, T c4) {
    x.c1 = c1; x.c2 = c2; x.c3 = c3; x.c4 = c4;
    x.ns = (c1 + c2) + (c3 + c4);
    x.n = x.ns;
}

// r^2 of one population from its counts; NaN-free form: returns false where the
// reference returns NaN (pA qA pB qB == 0, haplotype_kernels.py:32-42).
// 1/x in double: hardware reciprocal estimate refined by two Newton-Raphson steps
// r <- r (2 - x r) (quadratic convergence from ~2^-20 to full precision).
LDK_DEV double recip_newton(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}
LDK_DEV float recip_newton(float x) { return 1.0f / x; }

template <typename T>
LDK_DEV bool hap_r2(const HapFeat<T>& x, T& r2) {
    const T den = (x.c1 + x.c2) * (x.c3 + x.c4) * ((x.c1 + x.c3) * (x.c2 + x.c4));
    if (!(den > T(0))) return false;
    const T e = x.c1 * x.c4 - x.c2 * x.c3;
    r2 = (e * e) * recip_newton(den);
    return true;
}
