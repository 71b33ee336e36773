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

LDK_DEV uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// FP64 add into shared memory.
LDK_DEV void smem_add_f64(double* p, double v) { atomicAdd(p, v); }
