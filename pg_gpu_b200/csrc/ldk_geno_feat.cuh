// Per-population features of one SNP pair on the unphased genotype path.
#pragma once
#include "ldk_common.cuh"

template <typename T>
struct GenoFeat {
    // nine-cell counts in moments order: g1..g9 = n22, n21, n20, n12, n11, n10, n02, n01, n00
    // (pg_gpu genotype_kernels.py:424-435); ns = their sum, n = n_valid (equal here)
    T g1, g2, g3, g4, g5, g6, g7, g8, g9, ns, n;
    T inn1, invn;              // 1/max(4n(n-1),1) and 1/n (genotype_kernels.py:458-460, 519)
    T r1, r2, r3;              // guarded 1/n, 1/(n(n-1)), 1/(n(n-1)(n-2))
    T u1, u2, u3;              // unguarded 1/ns, 1/(ns(ns-1)), 1/(ns(ns-1)(ns-2))
    T w4;                      // 1/(ns(ns-1)(ns-2)(ns-3)) if ns >= 4 else 0
    T xAB, xAb, xaB, xab, D, pA, qA, pB, qB, BL, BR, C00, C01, C10, C11, Bsgn;
    T p, r, q, s, L0, AQ3, AS3, BP3, BR3, A, Bv, Wjj, U, V, DD1, DZ1, PI1;
};

// counts in the order of pg_gpu's counting kernel: column g_i*3 + g_j (n00 ... n22)
template <typename T>
LDK_DEV void geno_set_counts(GenoFeat<T>& x, const T (&c)[9]) {
    x.g1 = c[8]; x.g2 = c[7]; x.g3 = c[6]; x.g4 = c[5]; x.g5 = c[4];
    x.g6 = c[3]; x.g7 = c[2]; x.g8 = c[1]; x.g9 = c[0];
    x.ns = ((c[0] + c[1]) + (c[2] + c[3])) + ((c[4] + c[5]) + (c[6] + c[7])) + c[8];
    x.n = x.ns;
}

template <typename T>
LDK_DEV void geno_prepare(GenoFeat<T>& x) {
    const T n = x.n, ns = x.ns;
    const T nn1 = T(4) * n * (n - T(1));
    x.inn1 = T(1) / (nn1 > T(1) ? nn1 : T(1));
    x.invn = T(1) / n;
    x.r1 = (n >= T(1)) ? T(1) / n : T(0);
    x.r2 = (n >= T(2)) ? T(1) / (n * (n - T(1))) : T(0);
    x.r3 = (n >= T(3)) ? T(1) / (n * (n - T(1)) * (n - T(2))) : T(0);
    x.u1 = T(1) / ns;
    x.u2 = T(1) / (ns * (ns - T(1)));
    x.u3 = T(1) / (ns * (ns - T(1)) * (ns - T(2)));
    x.w4 = (ns >= T(4)) ? T(1) / (ns * (ns - T(1)) * (ns - T(2)) * (ns - T(3))) : T(0);
}

// geno_prepare's reciprocals as a function of n alone (n = ns on the genotype path): the
// tensor-core parse tabulates them once per parse instead of dividing per pair.
struct GenoRecip {
    double inn1, invn, r1, r2, r3, u1, u2, u3, w4;
};

LDK_DEV GenoRecip geno_recip_entry(int n) {
    GenoFeat<double> x;
    x.n = x.ns = (double)n;
    geno_prepare(x);
    return GenoRecip{x.inn1, x.invn, x.r1, x.r2, x.r3, x.u1, x.u2, x.u3, x.w4};
}

// geno_prepare for n = ns, from the table entry of n (the same values bit for bit).
LDK_DEV void geno_prepare_from(GenoFeat<double>& x, const GenoRecip* e) {
    x.inn1 = e->inn1;
    x.invn = e->invn;
    x.r1 = e->r1;
    x.r2 = e->r2;
    x.r3 = e->r3;
    x.u1 = e->u1;
    x.u2 = e->u2;
    x.u3 = e->u3;
    x.w4 = e->w4;
}

// Pairwise-complete dosage (Rogers-Huff) r^2 from the nine cells; false where either
// locus is constant (pg_gpu ld_statistics.py:410-443 returns NaN there).
template <typename T>
LDK_DEV bool geno_dosage_r2(const T (&c)[9], T& r2) {
    T n = T(0), sx = T(0), sy = T(0), sxx = T(0), syy = T(0), sxy = T(0);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const T a = T(k / 3), b = T(k % 3);
        n += c[k]; sx += a * c[k]; sy += b * c[k];
        sxx += a * a * c[k]; syy += b * b * c[k]; sxy += a * b * c[k];
    }
    const T vx = n * sxx - sx * sx, vy = n * syy - sy * sy, cv = n * sxy - sx * sy;
    const T den = vx * vy;
    if (!(den > T(0))) return false;
    r2 = cv * cv / den;
    return true;
}
