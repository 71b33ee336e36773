// Shared device-side helpers of libldk: status reporting, bounded waits, distance bins
// and the per-thread -> shared -> global accumulation of per-bin statistic sums.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define LDK_DEV __device__ __forceinline__

#define LDK_MAX_BINS 64
#define LDK_MAX_POPS 4

// Device status word bits (written with atomicOr, read back by the host after a call).
enum : unsigned {
    LDK_DEVERR_TIMEOUT = 1u << 0,     // a bounded wait gave up
    LDK_DEVERR_BLOCK_RANGE = 1u << 1, // a SNP's bootstrap block is outside [0, n_blocks)
    LDK_DEVERR_BLOCK_SPAN = 1u << 2,  // a row block spans more bootstrap blocks than staged
    LDK_DEVERR_BAD_INPUT = 1u << 3,   // unexpected genotype/haplotype code
    LDK_DEVERR_ACCUM = 1u << 4,       // a value outside the fixed-point bin accumulator's range
};

struct BinEdges {
    int n_bins;
    double e[LDK_MAX_BINS + 1];
};

// Right-open bins [e_b, e_{b+1}) as cp.digitize(d, edges) - 1 (moments_ld.py:314 of pg_gpu).
// Returns -1 below the first edge and n_bins at or above the last.
LDK_DEV int bin_of(const BinEdges& E, double d) {
    int lo = 0, hi = E.n_bins + 1;  // count of edges <= d, by bisection
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (E.e[mid] <= d) lo = mid + 1; else hi = mid;
    }
    return lo - 1;
}

// Advance a bin index monotonically for non-decreasing distances (amortised O(1)).
LDK_DEV int bin_advance(const double* __restrict__ e, int n_bins, int b, double d) {
    if (b < 0) {
        if (d < e[0]) return -1;
        b = 0;
    }
    while (b < n_bins && d >= e[b + 1]) ++b;
    return b;
}

// int32 -> double by the 2^52 "magic number" method: the bit pattern 0x43300000:(x ^ 2^31) is
// the double 2^52 + 2^31 + x for every int32 x, and subtracting 2^52 + 2^31 is exact.  One
// FP64 add and two integer instructions instead of the int -> FP64 conversion instruction,
// which measured slower in the tensor-core epilogue (full configuration 4: 48.25 vs 49.2 ms).
LDK_DEV double i2d_exact(int x) {
    return __hiloint2double(0x43300000, x ^ (int)0x80000000) - 4503601774854144.0;
}
template <typename T>
LDK_DEV T count_to(int x) {
    if constexpr (sizeof(T) == sizeof(double)) return i2d_exact(x);
    else return T(x);
}

LDK_DEV uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// FP64 add into shared memory.
LDK_DEV void smem_add_f64(double* p, double v) { atomicAdd(p, v); }

// ---------------------------------------------------------------------------
// Order-independent bin sums.  Each FP64 partial sum is converted exactly (truncated below
// 2^-96) into a fixed-point integer X = |v| * 2^96 < 2^160, split into kFxLimbs limbs of 32
// bits, and each nonzero limb (negated for v < 0) is added into a signed 64-bit word with an
// integer atomic.  Integer addition is associative, so the accumulated value does not depend
// on the order in which CTAs flush: two runs of the same parse give the same bits.  A limb
// word takes up to 2^31 additions before it could overflow.  fx_value() normalises the
// words (exact carries) and rounds the integer to FP64 once.
// ---------------------------------------------------------------------------
constexpr int kFxLimbs = 5;
constexpr int kFxLimbBits = 32;

LDK_DEV void fx_add(unsigned long long* acc, double v, unsigned* status) {
    if (v == 0.0) return;
    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
    const int eb = (int)((bits >> 52) & 0x7FF);
    if (eb >= 1023 + 63) {  // not finite, or |v| >= 2^63
        atomicOr(status, LDK_DEVERR_ACCUM);
        return;
    }
    unsigned long long m = bits & ((1ull << 52) - 1);
    int e;  // |v| = m * 2^e
    if (eb == 0) e = -1074;
    else { m |= 1ull << 52; e = eb - 1075; }
    const int s = e + 96;  // X = m * 2^s, s <= 10 + 96, so X < 2^159
    const bool neg = (bits >> 63) != 0;
#pragma unroll
    for (int k = 0; k < kFxLimbs; ++k) {
        const int lo = kFxLimbBits * k;
        unsigned long long limb;
        if (lo >= s) {
            const int d = lo - s;
            limb = d < 64 ? (m >> d) : 0ull;
        } else {
            const int d = s - lo;
            limb = d < kFxLimbBits ? (m << d) : 0ull;  // only the low 32 bits are kept
        }
        limb &= (1ull << kFxLimbBits) - 1;
        if (limb) atomicAdd(acc + k, neg ? (0ull - limb) : limb);
    }
}

// 2^n for normal exponents (n in [-1022, 1023]), exact.
LDK_DEV double pow2i(int n) { return __longlong_as_double((long long)(n + 1023) << 52); }

// The accumulated value: X = sum_k (signed) acc[k] * 2^(32k), rounded to FP64 and scaled by
// 2^-96.  Deterministic (a function of the integer words only).
LDK_DEV double fx_value(const unsigned long long* acc) {
    constexpr unsigned long long mask = (1ull << kFxLimbBits) - 1;
    unsigned long long L[kFxLimbs];
    long long c = 0;
#pragma unroll
    for (int k = 0; k < kFxLimbs; ++k) {  // limbs in [0, 2^32), signed top word c
        const long long t = (long long)acc[k] + c;
        L[k] = (unsigned long long)t & mask;
        c = t >> kFxLimbBits;  // arithmetic shift: floor division
    }
    const bool neg = c < 0;
    if (neg) {  // magnitude: -X renormalised the same way
        long long cc = 0;
#pragma unroll
        for (int k = 0; k < kFxLimbs; ++k) {
            const long long t = -(long long)L[k] + cc;
            L[k] = (unsigned long long)t & mask;
            cc = t >> kFxLimbBits;
        }
        c = -c + cc;
    }
    // non-negative terms, added from the smallest
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < kFxLimbs; ++k) v += (double)L[k] * pow2i(kFxLimbBits * k - 96);
    v += (double)c * pow2i(kFxLimbBits * kFxLimbs - 96);
    return neg ? -v : v;
}
