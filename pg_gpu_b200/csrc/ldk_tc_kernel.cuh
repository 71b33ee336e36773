// Tensor-core path of the binned parse (sm_100a): the kernel template and its launcher,
// instantiated per path and tile variant in ldk_tc_hap0.cu, ldk_tc_hap1.cu, ldk_tc_geno.cu.
//
// Counting as a Gram product.  For SNPs i, j and one population, with per-haplotype
// indicators h = [allele == 1] and v = [allele != missing], the four products
//   hh = sum_k h_ik h_jk,  hv = sum_k h_ik v_jk,  vh = sum_k v_ik h_jk,  vv = sum_k v_ik v_jk
// give the two-locus counts exactly: n11 = hh, n10 = hv - hh, n01 = vh - hh,
// n00 = vv - hv - vh + hh, n_valid = vv (pg_gpu ld_pipeline.py:155-172).
//
// Layout in HBM (built by k_prep_planes): per SNP two 0/1 byte planes (h, v) over the
// concatenated haplotypes of all populations, each population padded to a multiple of
// 32 bytes, the whole K axis to a multiple of 128 bytes:  planes[snp][plane][k].
// A 3-D TMA box {128 k, 2 planes, R snps} then lands in shared memory as 2R interleaved
// rows (h_i0, v_i0, h_i1, v_i1, ...) in the 128-byte-swizzled K-major layout that
// tcgen05.mma reads directly.  One MMA per 32-byte K step and population:
//   D[128 x 2NJ] (+)= A[128 rows = 64 SNPs x {h,v}] . B[2NJ rows = NJ SNPs x {h,v}]^T
// with u8 inputs and s32 accumulation in tensor memory: TMEM lane 2r holds (hh, hv) and
// lane 2r+1 holds (vh, vv) of SNP i0+r against every j of the tile.
//
// Warp roles (one CTA per SM, persistent over work items: runs of one row block's partner
// tiles, claimed dynamically):
//   warp 0     TMA producer (A: row block, B: 12..128 partner SNPs, per 128-byte K chunk)
//   warp 1     TMEM allocator and single-thread MMA issuer, double-buffered accumulators
//   epilogue   8, 12 or 16 warps (see Cfg), two to four per TMEM lane quarter, each
//              taking its share of every partner tile: tcgen05.ld the counts, swap halves
//              between lane pairs, evaluate the estimators in FP64, sum per
//              distance bin in registers (bins are monotone
//              in j for a fixed i), flush each finished bin run into a per-warp FP64
//              staging copy in shared memory, and add the staged sums to the
//              per-bootstrap-block fixed-point accumulators once per work item (integer
//              atomics, so the result does not depend on the order of the items).
// Every wait is bounded (LDK_DEVERR_TIMEOUT) so a fault cannot hang the GPU.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <math_constants.h>

#include <cstdlib>
#include <mutex>
#include <type_traits>

#include "ldk_estimators.cuh"
#include "ldk_internal.h"

namespace ldk {
namespace {

constexpr int kKChunk = 128;            // K bytes per TMA box / swizzle row
constexpr int kRing = 2;                // claimed work items in flight between the roles
constexpr int kTmemCols = 512;
constexpr uint64_t kTimeoutNs = 5000000000ull;  // 5 s per wait
// Register split of the SPLIT layouts: the launch gives every thread Cfg::REG_LAUNCH
// registers; warpgroup 0 drops to kRegCtrl and the epilogue warpgroups rise to Cfg::REG_EPI,
// which the freed registers cover (Cfg asserts the sum).  The host launches only a kernel
// compiled to Cfg::REG_LAUNCH registers.
constexpr int kRegCtrl = 24;
constexpr size_t kMinSmem = 116 * 1024;
constexpr size_t kMaxSmem = 227 * 1024;

// Tile geometry.  Haplotype path: a row block of 64 SNPs x {h, v} = 128 MMA rows against
// NJ partners x {h, v} (N = 2 NJ), one MMA per K step and population.  Genotype path: a row
// block of 128 SNPs; four stored planes per SNP {g == 1, g == 2, valid, 0}; per K step and
// population three MMAs, plane x (< 3) of the row block against all four planes of NJ
// partners (N = 4 NJ) into region x, so TMEM lane r holds all nine Gram products of SNP r
// (and a zero column per partner, which keeps every partner's columns 4-aligned).
// Partners per tile: tile variant 0 is the default, variant 1 the alternative the
// autotuner also times (half the width on the haplotype path; on the genotype path 8 for
// one population, 16 for two -- one TMEM buffer -- and the default for more).
// Two haplotype populations and one genotype population: 48 (or 24) and 12 (or 24), so that
// each of the three epilogue warps of a lane quarter takes an equal share of the tile.
constexpr int tile_nj(int P, bool GENO, int V) {
    return GENO ? (V == 0 ? (P == 1 ? 12 : 8) : (P == 1 ? 24 : P == 2 ? 16 : 8))
                : ((P == 1 ? 128 : P == 2 ? 48 : 32) >> V);
}

template <int P, bool GENO = false, int V = 0>
struct Cfg {
    static constexpr int ROWS = GENO ? 128 : 64;                      // SNPs per row block
    static constexpr int PLANES = GENO ? 4 : 2;                        // stored planes per SNP
    static constexpr int NJ = tile_nj(P, GENO, V);                     // partners per tile
    static constexpr int N = PLANES * NJ;                              // MMA N
    static constexpr int REGIONS = GENO ? 3 : 1;                       // MMAs per K step and population
    static constexpr int COLS = P * REGIONS * N;                       // TMEM columns per buffer
    static constexpr int NBUF = 2 * COLS <= kTmemCols ? 2 : 1;         // accumulator buffers
    // four genotype populations: two stages, so that the per-bin staging of more bins fits
    // beside them (their epilogue, not the loads, sets the pace)
    static constexpr int STAGES = GENO ? (P == 4 ? 2 : 3) : (P == 1) ? 2 : (P == 2) ? 3 : 4;
    static constexpr int A_BOX = 128 * kKChunk;                        // one 128-row A box
    static constexpr int A_BYTES = REGIONS * A_BOX;
    static constexpr int B_BYTES = N * kKChunk;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int NS = HapNStats<P>::value;
    static constexpr int SLOTS = GENO ? 4 : 2;                         // bootstrap blocks staged per row block
    // Warp layout.  Warp w may read only TMEM lane quarter w % 4, and each of the four
    // schedulers of an SM holds warps w, w + 4, ... with a quarter of the register file.
    // The epilogue warps of a lane quarter each take an equal share of every partner tile.
    //  * SPLIT (genotypes; haplotypes with three or four populations -- estimators that
    //    want ~240 registers): 12 warps.  Warpgroup 0 (TMA, MMA, two idle warps) gives its
    //    registers up with setmaxnreg (kRegCtrl each) and the eight epilogue warps 4..11
    //    take them (240 each), so that every scheduler holds two full-register epilogue
    //    warps beside one control warp (launch: 168 per thread).
    //  * two haplotype populations (~155 registers) and one genotype population, also SPLIT:
    //    16 warps, twelve epilogue warps 4..15 at 160 registers, three per scheduler and lane
    //    quarter (launch: 128).
    //  * one haplotype population (about 100 registers): 18 warps, TMA and MMA in warps 0 and
    //    1, sixteen epilogue warps 2..17, four per lane quarter and scheduler, each taking a
    //    quarter of every partner tile -- its per-pair work is short, so more warps hide the
    //    latency of its dependency chains (113 registers at most).
    static constexpr bool SPLIT = GENO || P >= 2;
    static constexpr int EPI = (!GENO && P == 1) ? 16 : ((!GENO && P == 2) || (GENO && P == 1)) ? 12 : 8;
    static constexpr int W0 = SPLIT ? 4 : 2;  // first epilogue warp
    static constexpr int THREADS = 32 * (W0 + EPI);
    static constexpr int REG_LAUNCH = (EPI == 12) ? 128 : 168;  // SPLIT layouts only
    static constexpr int REG_EPI = (EPI == 12) ? 160 : 240;
    static_assert(!SPLIT || 4 * kRegCtrl + EPI * REG_EPI <= (W0 + EPI) * REG_LAUNCH,
                  "register split must fit the launch allocation");
    static_assert(!SPLIT || THREADS * REG_LAUNCH <= 65536, "register file");
    static_assert(EPI % 4 == 0 && (GENO ? NJ : NJ / 2) % (EPI / 4) == 0, "epilogue warps share tiles equally");
    static_assert(NBUF * COLS <= kTmemCols, "TMEM budget");
    static_assert(N % 16 == 0 && N <= 256, "MMA N");
};

// ---------------------------------------------------------------------------
// PTX wrappers (tcgen05, TMA, mbarrier)
// ---------------------------------------------------------------------------

LDK_DEV uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

LDK_DEV void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count));
}
LDK_DEV void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
LDK_DEV void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
LDK_DEV bool mbar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on a barrier phase.  False on timeout or when another role aborted.
LDK_DEV bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag, unsigned* status) {
    if (mbar_test(b, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_test(b, parity)) return true;
        if (*abort_flag) return false;
        if (global_ns() - t0 > kTimeoutNs) {
            atomicOr(status, LDK_DEVERR_TIMEOUT);
            *abort_flag = 1;
            return false;
        }
    }
}

LDK_DEV void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(su32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(su32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

LDK_DEV void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(dst)), "r"(ncols));
}
LDK_DEV void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;"); }
LDK_DEV void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
LDK_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
LDK_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major operand in the 128-byte swizzle layout: 8-row groups 1024 bytes apart.
LDK_DEV uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset
    d |= (uint64_t)1 << 46;              // descriptor version for sm_100
    d |= (uint64_t)2 << 61;              // SWIZZLE_128B
    return d;
}

// kind::i8 instruction descriptor: u8 x u8 -> s32, K-major A and B, M = 128.
template <int N>
__host__ __device__ constexpr uint32_t idesc_u8() {
    return (2u << 4)                      // D format s32
           | (0u << 7) | (0u << 10)       // A, B unsigned 8-bit
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(128 >> 4) << 24);  // M / 16
}

LDK_DEV void mma_u8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}
LDK_DEV void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

LDK_DEV void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
}
template <int P>
LDK_DEV void tmem_wait4(uint32_t (&r)[P][4]) {
#pragma unroll
    for (int p = 0; p < P; ++p)
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+r"(r[p][0]), "+r"(r[p][1]), "+r"(r[p][2]), "+r"(r[p][3])
                     :
                     : "memory");
}

template <int EPI>
LDK_DEV void epi_bar() { asm volatile("bar.sync 1, %0;" ::"n"(32 * EPI) : "memory"); }
template <int EPI>
LDK_DEV bool epi_bar_or(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "barrier.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "n"(32 * EPI)
        : "memory");
    return r != 0;
}

// Warpgroup-wide register budget changes (all four warps of the warpgroup execute them).
template <int N>
LDK_DEV void setmaxnreg_inc() { asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(N)); }
template <int N>
LDK_DEV void setmaxnreg_dec() { asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(N)); }

LDK_DEV void spin_ns(uint64_t ns) {
    const uint64_t t0 = global_ns();
    while (global_ns() - t0 < ns) {
    }
}

// ---------------------------------------------------------------------------
// the fused count + estimator + bin kernel
// ---------------------------------------------------------------------------

struct TcArgs {
    const double* coord;
    const int32_t* jmax;
    const int32_t* snp_block;
    int n_blocks;
    const int32_t* items;  // (n_items, 4): rows [row0, row1), partner tiles [t0, t1) of that row block
    const int* n_items;    // items in use (written with the list)
    int* item_counter;     // next unclaimed item (zero at launch)
    int nkc;               // K chunks of 128 bytes
    int kofs[LDK_MAX_POPS + 1];
    int max_n;             // largest population (reciprocal table size - 1)
    BinEdges edges;
    unsigned long long* fx;  // fixed-point bin sums [block][bin][NS + 1][kFxLimbs] (r^2 last)
    unsigned long long* pairs;
    unsigned long long* r2_counts;
    unsigned* status;
    const double4* rtab_g;  // haplotype path: reciprocal table in global memory, or null when
                            // each CTA builds it in shared memory
    const GenoRecip* gtab;  // genotype path, P <= 3: geno_prepare's reciprocals per valid count
};

// Shared-memory state of the persistent pipeline (one CTA).
struct Pipe {
    unsigned char* stages;
    uint64_t* full_bar;
    uint64_t* empty_bar;
    uint64_t* tfull;
    uint64_t* tempty;
    uint64_t* ifull;
    uint64_t* iempty;
    volatile int* ring;  // [kRing] claimed items, then [kRing] their tile counts
    volatile int* abort_s;
};

// Item `item`: rows [row0, row1) and the partner tiles [t0, t1) of that row block, t1
// clipped to the row block's tiles (partners up to jmax[row1 - 1]).  Returns the number of
// tiles; the first starts at partner jt0.  The items of one row block partition its tile
// indices (its last item runs to INT32_MAX), so every tile is counted once whatever the
// partner range is when the kernel runs.
template <class C>
LDK_DEV int item_tiles(const TcArgs& a, int item, int& row0, int& row1, int& jt0) {
    const int4 it = reinterpret_cast<const int4*>(a.items)[item];
    row0 = it.x;
    row1 = it.y;
    const int jend = a.jmax[row1 - 1];
    const int n_jt = jend > row0 + 1 ? (jend - row0 + C::NJ - 1) / C::NJ : 0;
    const int te = it.w < n_jt ? it.w : n_jt;
    jt0 = row0 + it.z * C::NJ;
    return te > it.z ? te - it.z : 0;
}

// TMA loads of K chunk c of the tile (row block at row0, partners from j0) into stage s.
template <class C>
LDK_DEV void issue_loads(const Pipe& S, const CUtensorMap* tmA, const CUtensorMap* tmB, int s, int c, int row0,
                         int j0) {
    unsigned char* dst = S.stages + s * C::STAGE_BYTES;
    mbar_expect_tx(&S.full_bar[s], C::STAGE_BYTES);
#pragma unroll
    for (int x = 0; x < C::REGIONS; ++x) tma_load_3d(dst + x * C::A_BOX, tmA, &S.full_bar[s], c * kKChunk, x, row0);
    tma_load_3d(dst + C::A_BYTES, tmB, &S.full_bar[s], c * kKChunk, 0, j0);
}

// MMAs of K chunk c (in stage s) into accumulator buffer buf; frees the stage on completion.
template <class C, int P>
LDK_DEV void issue_mmas(const Pipe& S, uint32_t tmem, const TcArgs& a, int s, int c, uint32_t buf) {
    constexpr uint32_t idesc = idesc_u8<C::N>();
    const uint32_t a_addr = su32(S.stages + s * C::STAGE_BYTES);
    const uint32_t b_addr = a_addr + C::A_BYTES;
#pragma unroll
    for (int ks = 0; ks < kKChunk / 32; ++ks) {
        const int kbyte = c * kKChunk + ks * 32;
        int p = 0;
#pragma unroll
        for (int q = 1; q < P; ++q) p += (kbyte >= a.kofs[q]) ? 1 : 0;
        const uint32_t first = (kbyte == a.kofs[p]) ? 1u : 0u;
#pragma unroll
        for (int x = 0; x < C::REGIONS; ++x) {
            const uint32_t d = tmem + buf * C::COLS + (p * C::REGIONS + x) * C::N;
            mma_u8(d, sw128_desc(a_addr + x * C::A_BOX + ks * 32), sw128_desc(b_addr + ks * 32), idesc, first ^ 1u);
        }
    }
    mma_commit(&S.empty_bar[s]);
}

// Warp 0: claims work items from the global counter, publishes each with its tile count
// through the ring and issues the TMA loads of every partner tile's K chunks.
template <class C>
LDK_DEV void run_producer(const Pipe& S, const CUtensorMap* tmA, const CUtensorMap* tmB, const TcArgs& a,
                          int lane) {
    if (lane == 0) {
        uint32_t it = 0;
        bool ok = true;
        for (uint32_t k = 0; ok; ++k) {
            // claim the next item and publish it to the MMA issuer and the epilogue
            const int sl = k % kRing;
            if (!mbar_wait(&S.iempty[sl], ((k / kRing) & 1u) ^ 1u, S.abort_s, a.status)) { ok = false; break; }
            int item = atomicAdd(a.item_counter, 1);
            if (item >= *a.n_items) item = -1;
            int row0 = 0, row1 = 0, jt0 = 0, n_jt = 0;
            if (item >= 0) n_jt = item_tiles<C>(a, item, row0, row1, jt0);
            S.ring[sl] = item;
            S.ring[kRing + sl] = n_jt;
            mbar_arrive(&S.ifull[sl]);
            if (item < 0) break;
            const int jstop = jt0 + n_jt * C::NJ;
            for (int j0 = jt0; j0 < jstop && ok; j0 += C::NJ) {
                for (int c = 0; c < a.nkc; ++c, ++it) {
                    const int s = it % C::STAGES;
                    const uint32_t ph = (it / C::STAGES) & 1u;
                    if (!mbar_wait(&S.empty_bar[s], ph ^ 1u, S.abort_s, a.status)) { ok = false; break; }
                    issue_loads<C>(S, tmA, tmB, s, c, row0, j0);
                }
            }
        }
        if (!ok) spin_ns(2000000);  // let copies already issued land before teardown
    }
    __syncwarp();
}

// Warp 1: one thread issues the MMAs of every tile into the double-buffered accumulators.
template <class C, int P>
LDK_DEV void run_mma(const Pipe& S, uint32_t tmem, const TcArgs& a, int lane) {
    if (lane == 0) {
        uint32_t it = 0, tcount = 0;
        bool ok = true;
        for (uint32_t k = 0; ok; ++k) {
            const int sl = k % kRing;
            if (!mbar_wait(&S.ifull[sl], (k / kRing) & 1u, S.abort_s, a.status)) { ok = false; break; }
            const int item = S.ring[sl], n_jt = S.ring[kRing + sl];
            mbar_arrive(&S.iempty[sl]);
            if (item < 0) break;
            for (int t = 0; t < n_jt && ok; ++t, ++tcount) {
                const uint32_t buf = tcount % C::NBUF, tph = (tcount / C::NBUF) & 1u;
                if (!mbar_wait(&S.tempty[buf], tph ^ 1u, S.abort_s, a.status)) { ok = false; break; }
                tc_fence_after();
                for (int c = 0; c < a.nkc; ++c, ++it) {
                    const int s = it % C::STAGES;
                    const uint32_t ph = (it / C::STAGES) & 1u;
                    if (!mbar_wait(&S.full_bar[s], ph, S.abort_s, a.status)) { ok = false; break; }
                    tc_fence_after();
                    issue_mmas<C, P>(S, tmem, a, s, c, buf);
                }
                if (!ok) break;
                mma_commit(&S.tfull[buf]);
            }
        }
        if (!ok) spin_ns(2000000);
    }
    __syncwarp();
}

// GT: the haplotype path's reciprocal table is read from the workspace (a.rtab_g) instead of
// being built in shared memory -- a compile-time choice, so that the shared-memory form keeps
// its hot loop unchanged.
template <int P, typename T, bool PRIV, bool GENO, int V, bool GT = false>
__global__ void __launch_bounds__(Cfg<P, GENO, V>::THREADS, 1)
    k_parse_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const TcArgs a) {
    using C = Cfg<P, GENO, V>;
    constexpr int NS = C::NS;
    constexpr int EPI = C::EPI;
    constexpr int SLOTS = C::SLOTS;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int nb = a.edges.n_bins;
    unsigned char* stages = base;
    constexpr int NCOPY = PRIV ? EPI : 1;  // staging copies: one per epilogue warp, or shared
    double* sacc = reinterpret_cast<double*>(base + C::STAGES * C::STAGE_BYTES);  // [NCOPY][SLOTS][nb][NS+1]
    unsigned* scnt = reinterpret_cast<unsigned*>(sacc + NCOPY * SLOTS * nb * (NS + 1));  // [NCOPY][SLOTS][nb][2]
    double4* rtab = reinterpret_cast<double4*>(scnt + ((NCOPY * SLOTS * nb * 2 + 7) & ~7));  // [max_n + 1]

    __shared__ __align__(8) uint64_t full_bar[C::STAGES], empty_bar[C::STAGES], tfull[C::NBUF], tempty[C::NBUF];
    __shared__ __align__(8) uint64_t ifull[kRing], iempty[kRing];
    __shared__ volatile int ring[2 * kRing];
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;
    __shared__ double sedges[LDK_MAX_BINS + 1];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < C::NBUF; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], EPI);
        }
        for (int b = 0; b < kRing; ++b) {
            mbar_init(&ifull[b], 1);
            mbar_init(&iempty[b], 1 + EPI);  // the MMA issuer and every epilogue warp
        }
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int b = threadIdx.x; b <= nb; b += blockDim.x) sedges[b] = a.edges.e[b];
    for (int idx = threadIdx.x; idx < NCOPY * SLOTS * nb * (NS + 1); idx += blockDim.x) sacc[idx] = 0.0;
    for (int idx = threadIdx.x; idx < NCOPY * SLOTS * nb * 2; idx += blockDim.x) scnt[idx] = 0u;
    if constexpr (!GENO && !GT)
        for (int idx = threadIdx.x; idx <= a.max_n; idx += blockDim.x) rtab[idx] = recip_entry(idx);
    if (warp == 1) {
        tmem_alloc(&tmem_base_s, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    const Pipe pipe{stages, full_bar, empty_bar, tfull, tempty, ifull, iempty, ring, &abort_s};
    // Each side changes its register budget once, at its start, and never back: warpgroup
    // 0 releases registers (setmaxnreg.dec never waits) and the epilogue warps take them
    // (setmaxnreg.inc waits only for that release, which comes unconditionally first).
    // No later increase exists that could wait on registers another warp holds -- a
    // restore to the launch count by warpgroup 0, whose idle warps would reach it at once,
    // could take the registers back before the epilogue's increase and starve it.  The
    // code both sides share, the teardown below, fits the smaller budget.  Neither the
    // roles nor the teardown may call a function (printf, a non-inlined helper): a
    // callee's registers are not bounded by the budget, and a call from a warp holding
    // kRegCtrl registers raised an illegal-instruction fault.
    if (warp < C::W0) {
        if constexpr (C::SPLIT) setmaxnreg_dec<kRegCtrl>();
        if (warp == 0) run_producer<C>(pipe, &tmA, &tmB, a, lane);
        else if (warp == 1) run_mma<C, P>(pipe, tmem, a, lane);
    } else {
        if constexpr (C::SPLIT) setmaxnreg_inc<C::REG_EPI>();
        // ------------------------------------------------------------- epilogue
        const int e = warp - C::W0;
        const int L = (warp & 3) * 32 + lane;
        // haplotype rows: lanes 2r, 2r+1 share SNP r and split its partners by parity;
        // genotype rows: lane L is SNP L and takes every partner.  With two warps per lane
        // quarter each takes a contiguous half of every partner tile, so every lane still
        // sees its partners in increasing order.
        const int r = GENO ? L : L >> 1, role = GENO ? 0 : L & 1;
        const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
        const int stage_n = SLOTS * nb * (NS + 1);
        double* my_sacc = sacc + (PRIV ? e * stage_n : 0);
        unsigned* my_scnt = scnt + (PRIV ? e * SLOTS * nb * 2 : 0);
        constexpr int STEPS = GENO ? C::NJ : C::NJ / 2;   // TMEM reads per tile
        constexpr int PARTS = EPI / 4;                    // epilogue warps per lane quarter
        // SSPL (four haplotype populations): the two warps of a lane quarter split the
        // statistics, not the partners -- both take every pair, warp part 0 accumulates
        // statistics [0, K) and counts pairs, part 1 statistics [K, NS) and r^2 -- so that
        // each holds about half of the 105 accumulators.  (The same split of the genotype
        // path measured slower: both warps then compute all four populations' features.)
        constexpr bool SSPL = !GENO && P == 4;
        constexpr int K = HapFusedSplit<P>::value;
        constexpr int NA = SSPL ? ((K > NS - K + 1 ? K : NS - K + 1)) : NS + 1;  // accumulators per lane
        constexpr int MY_STEPS = SSPL ? STEPS : STEPS / PARTS;  // ... each reading a contiguous share
        const int part = e >> 2;
        constexpr int CREGS = (C::NJ + 31) / 32;          // partner coordinates per lane
        uint32_t tcount = 0;
        for (uint32_t k = 0;; ++k) {
            const int sl = k % kRing;
            int item = -1;
            if (lane == 0) {
                if (mbar_wait(&ifull[sl], (k / kRing) & 1u, &abort_s, a.status)) {
                    item = ring[sl];
                    mbar_arrive(&iempty[sl]);
                }
            }
            item = __shfl_sync(0xffffffffu, item, 0);
            if (epi_bar_or<EPI>(abort_s != 0 || item < 0)) break;
            // the item's tiles [tb, te) of row block [row0, row1) (as item_tiles; scalar loads
            // and a loop over tile indices keep this 240-register epilogue free of spills)
            const int row0 = a.items[4 * item], row1 = a.items[4 * item + 1];
            const int jend = a.jmax[row1 - 1];
            const int n_full = jend > row0 + 1 ? (jend - row0 + C::NJ - 1) / C::NJ : 0;
            const int tw = a.items[4 * item + 3];
            const int tb = a.items[4 * item + 2];
            const int te = tw < n_full ? tw : n_full;
            if (te <= tb) continue;
            const int i = row0 + r;
            bool row_ok = i < row1;
            const int my_jmax = row_ok ? a.jmax[i] : 0;
            const double ci = row_ok ? a.coord[i] : 0.0;
            const int blk0 = a.snp_block ? a.snp_block[row0] : 0;
            int slot = 0;
            if (row_ok && a.snp_block) {
                slot = a.snp_block[i] - blk0;
                if (slot < 0 || slot >= SLOTS) {
                    atomicOr(a.status, LDK_DEVERR_BLOCK_SPAN);
                    row_ok = false;
                }
            }
            // Sums of the current bin live in registers.  Partners come in increasing j,
            // so the distance to them never decreases and each (row, bin) run is flushed
            // to shared memory once, when the lane's next partner falls past the bin's
            // upper edge (held in `nxt`).
            T acc[NA];
            // statistic s of this warp's accumulators and where it goes in the staging row
            const int na = SSPL ? (part == 0 ? K : NS - K + 1) : NS + 1;
            const int gofs = SSPL && part == 1 ? K : 0;
#pragma unroll
            for (int s = 0; s < NA; ++s) acc[s] = T(0);
            unsigned np = 0, nr2 = 0;
            int cur = -1;
            double nxt = sedges[0];
            // Adds the flushing lanes' sums into shared memory.  With PRIV every epilogue
            // warp owns its staging copy and the lanes of one warp that flush the same
            // (block, bin) take turns (one lane per key per round), so plain adds suffice;
            // otherwise the copy is shared by the warps and the adds are atomic.  Called by
            // all 32 lanes.
            auto flush = [&](bool want) {
                const int key = slot * nb + cur;
                if constexpr (PRIV) {
                    const unsigned grp = __match_any_sync(0xffffffffu, want ? key : -1);
                    const int rank = __popc(grp & ((1u << lane) - 1u));
                    const int rounds = (int)__reduce_max_sync(0xffffffffu, want ? (unsigned)__popc(grp) : 0u);
                    double* dst = my_sacc + key * (NS + 1);
                    for (int rr = 0; rr < rounds; ++rr) {
                        if (want && rank == rr) {
                            if constexpr (SSPL) {
#pragma unroll
                                for (int s = 0; s < NA; ++s)
                                    if (s < na) dst[gofs + s] += (double)acc[s];
                                if (part == 0) my_scnt[2 * key] += np;
                            } else {
#pragma unroll
                                for (int s = 0; s <= NS; ++s) dst[s] += (double)acc[s];
                                my_scnt[2 * key] += np;
                            }
                            my_scnt[2 * key + 1] += nr2;
                        }
                        __syncwarp();
                    }
                } else if (want) {
                    double* dst = my_sacc + key * (NS + 1);
                    if constexpr (SSPL) {
#pragma unroll
                        for (int s = 0; s < NA; ++s)
                            if (s < na) atomicAdd(dst + gofs + s, (double)acc[s]);
                        if (part == 0) atomicAdd(my_scnt + 2 * key, np);
                    } else {
#pragma unroll
                        for (int s = 0; s <= NS; ++s) atomicAdd(dst + s, (double)acc[s]);
                        atomicAdd(my_scnt + 2 * key, np);
                    }
                    atomicAdd(my_scnt + 2 * key + 1, nr2);
                }
            };
            bool ok = true;
            for (int t = tb; t < te; ++t, ++tcount) {
                const uint32_t buf = tcount % C::NBUF, tph = (tcount / C::NBUF) & 1u;
                const int j0 = row0 + t * C::NJ;
                // partner coordinates of this tile, one per lane and register
                double creg[CREGS];
#pragma unroll
                for (int kk = 0; kk < CREGS; ++kk) {
                    const int j = j0 + 32 * kk + lane;
                    creg[kk] = (32 * kk + lane < C::NJ && j < jend) ? a.coord[j] : 0.0;
                }
                if (!mbar_wait(&tfull[buf], tph, &abort_s, a.status)) { ok = false; break; }
                tc_fence_after();
                // One TMEM read per step, indexed with constants only so the counts stay in
                // registers.  Haplotypes: two partners per step, 4 columns per population.
                // Genotypes: one partner per step, 4 columns per region and population.
#pragma unroll 1
                for (int qq = 0; qq < MY_STEPS; ++qq) {
                    const int q = SSPL ? qq : part * MY_STEPS + qq;
                    uint32_t v[P][C::REGIONS][4];
#pragma unroll
                    for (int p = 0; p < P; ++p)
#pragma unroll
                        for (int x = 0; x < C::REGIONS; ++x)
                            tmem_ld4(tmem + lane_base + buf * C::COLS + (p * C::REGIONS + x) * C::N + q * 4,
                                     v[p][x]);
                    const int jj = GENO ? q : 2 * q + role;
                    double csrc = creg[0];
#pragma unroll
                    for (int kk = 1; kk < CREGS; ++kk)
                        if ((jj >> 5) == kk) csrc = creg[kk];
                    const double cj = __shfl_sync(0xffffffffu, csrc, jj & 31);
#pragma unroll
                    for (int p = 0; p < P; ++p) tmem_wait4<C::REGIONS>(v[p]);
                    if (qq == MY_STEPS - 1) {
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&tempty[buf]);
                    }
                    const int j = j0 + jj;
                    const bool valid = row_ok && j > i && j < my_jmax;
                    const double dist = fabs(cj - ci);
                    const bool change = valid && dist >= nxt;
                    const bool want = change && cur >= 0 && np > 0;
                    if (__ballot_sync(0xffffffffu, want)) flush(want);
                    if (change) {
                        cur = bin_advance(sedges, nb, cur, dist);
                        nxt = cur < nb ? sedges[cur + 1] : CUDART_INF;
#pragma unroll
                        for (int s = 0; s < NA; ++s) acc[s] = T(0);
                        np = nr2 = 0;
                    }
                    if constexpr (!GENO) {
                        HapFeat<T> f[P];
                        int nval[P];
#pragma unroll
                        for (int p = 0; p < P; ++p) {
                            // lane 2r: (hh, hv) of partners 2q, 2q+1; lane 2r+1: (vh, vv)
                            const uint32_t* w = v[p][0];
                            const uint32_t sx = role ? w[0] : w[2];
                            const uint32_t sy = role ? w[1] : w[3];
                            const uint32_t rx = __shfl_xor_sync(0xffffffffu, sx, 1);
                            const uint32_t ry = __shfl_xor_sync(0xffffffffu, sy, 1);
                            int hh, hv, vh, vv;
                            if (role == 0) { hh = (int)w[0]; hv = (int)w[1]; vh = (int)rx; vv = (int)ry; }
                            else { vh = (int)w[2]; vv = (int)w[3]; hh = (int)rx; hv = (int)ry; }
                            hap_set_counts(f[p], count_to<T>(hh), count_to<T>(hv - hh), count_to<T>(vh - hh),
                                           count_to<T>(vv - hv - vh + hh));
                            nval[p] = vv;
                        }
                        if (valid && cur >= 0 && cur < nb) {
#pragma unroll
                            for (int p = 0; p < P; ++p) {
                                hap_features<T, P>(f[p]);
                                if constexpr (GT) hap_reciprocals_from(f[p], a.rtab_g[nval[p]]);
                                else hap_reciprocals_from(f[p], rtab[nval[p]]);
                            }
                            if constexpr (SSPL) {
                                if (part == 0) {
                                    hap_fused<T, P, 1>(f, acc);
                                } else {
                                    hap_fused<T, P, 2>(f, acc);
                                    T r2;
                                    // r^2 is this part's last staged value (global index NS)
                                    if (hap_r2(f[0], r2)) { acc[NS - K] += r2; ++nr2; }
                                }
                            } else {
                                hap_fused<T, P, 0>(f, acc);
                                T r2;
                                if (hap_r2(f[0], r2)) { acc[NS] += r2; ++nr2; }
                            }
                            ++np;
                        }
                    } else {
                        if (valid && cur >= 0 && cur < nb) {
                            // Gram products G[x][y] = plane x of SNP i . plane y of SNP j
                            // (0: g == 1, 1: g == 2, 2: valid); cells in the order of pg_gpu's
                            // counting kernel, column g_i * 3 + g_j (ld_pipeline.py:183-263)
                            GenoFeat<T> f[P];
                            T c0[9];
#pragma unroll
                            for (int p = 0; p < P; ++p) {
                                const uint32_t (&G)[3][4] = v[p];
                                const int n11 = (int)G[0][0], n12 = (int)G[0][1], n21 = (int)G[1][0], n22 = (int)G[1][1];
                                const int n10 = (int)G[0][2] - n11 - n12, n20 = (int)G[1][2] - n21 - n22;
                                const int n01 = (int)G[2][0] - n11 - n21, n02 = (int)G[2][1] - n12 - n22;
                                const int nv = (int)G[2][2];
                                const int n00 = nv - n01 - n02 - n10 - n11 - n12 - n20 - n21 - n22;
                                const T cd[9] = {count_to<T>(n00), count_to<T>(n01), count_to<T>(n02),
                                                 count_to<T>(n10), count_to<T>(n11), count_to<T>(n12),
                                                 count_to<T>(n20), count_to<T>(n21), count_to<T>(n22)};
                                if (p == 0) {
#pragma unroll
                                    for (int m = 0; m < 9; ++m) c0[m] = cd[m];
                                }
                                geno_set_counts(f[p], cd);
                                f[p].n = count_to<T>(nv);
                                if constexpr (P <= 3) {
                                    geno_prepare_from(f[p], a.gtab + nv);  // n = ns = nv here
                                    geno_features<T, P, false>(f[p]);
                                } else {
                                    // four populations divide: the table's registers deepen
                                    // their spill (measured 0.45 vs 0.60 Gpairs/s)
                                    geno_features<T, P>(f[p]);
                                }
                            }
                            geno_stats<T, P>(f, acc);
                            T r2;
                            if (geno_dosage_r2(c0, r2)) { acc[NS] += r2; ++nr2; }
                            ++np;
                        }
                    }
                }
            }
            flush(cur >= 0 && cur < nb && np > 0);
            (void)ok;
            // staging -> global, once per work item
            epi_bar<EPI>();
            const int et = threadIdx.x - 32 * C::W0;
            for (int idx = et; idx < stage_n; idx += 32 * EPI) {
                double val = 0.0;
#pragma unroll
                for (int w = 0; w < (PRIV ? EPI : 1); ++w) {
                    val += sacc[w * stage_n + idx];
                    sacc[w * stage_n + idx] = 0.0;
                }
                const int sl = idx / (nb * (NS + 1));
                const int rem = idx % (nb * (NS + 1));
                const int bb = rem / (NS + 1), s = rem % (NS + 1);
                const int blk = blk0 + sl;
                if (val != 0.0 && blk < a.n_blocks)
                    fx_add(a.fx + (((int64_t)blk * nb + bb) * (NS + 1) + s) * kFxLimbs, val, a.status);
            }
            for (int idx = et; idx < SLOTS * nb; idx += 32 * EPI) {
                unsigned long long c0 = 0, c1 = 0;
#pragma unroll
                for (int w = 0; w < (PRIV ? EPI : 1); ++w) {
                    unsigned* sc = scnt + w * SLOTS * nb * 2;
                    c0 += sc[2 * idx];
                    c1 += sc[2 * idx + 1];
                    sc[2 * idx] = 0u;
                    sc[2 * idx + 1] = 0u;
                }
                const int blk = blk0 + idx / nb, bb = idx % nb;
                if (blk < a.n_blocks) {
                    if (c0) atomicAdd(&a.pairs[(int64_t)blk * nb + bb], c0);
                    if (c1) atomicAdd(&a.r2_counts[(int64_t)blk * nb + bb], c1);
                }
            }
            epi_bar<EPI>();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// planes[snp][plane][k]: boxes of 128 k x plane_box planes x rows_box SNPs
bool make_map(CUtensorMap* m, const uint8_t* planes, int64_t n_var, int ktot, int n_planes, int plane_box,
              int rows_box) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)ktot, (cuuint64_t)n_planes, (cuuint64_t)n_var};
    cuuint64_t strides[2] = {(cuuint64_t)ktot, (cuuint64_t)ktot * n_planes};
    cuuint32_t box[3] = {(cuuint32_t)kKChunk, (cuuint32_t)plane_box, (cuuint32_t)rows_box};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t*>(planes), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Dynamic shared memory: pipeline stages, `ncopy` staging copies and `table` reciprocal
// table entries (32 B each).
template <int P, bool GENO, int V = 0>
size_t smem_bytes_t(int nb, int table, int ncopy) {
    using C = Cfg<P, GENO, V>;
    return 1024 + (size_t)C::STAGES * C::STAGE_BYTES + (size_t)ncopy * C::SLOTS * nb * (C::NS + 1) * sizeof(double) +
           (size_t)((ncopy * C::SLOTS * nb * 2 + 7) & ~7) * sizeof(unsigned) + (size_t)table * sizeof(double4) + 32;
}

// Reciprocal table entries held in shared memory (none on the genotype path, none when the
// table lives in the workspace).
inline int smem_table(const ParseShape& sh) { return (sh.genotypes || sh.rtab_global) ? 0 : sh.max_n + 1; }

// Per-warp staging copies when they fit next to the pipeline stages.
template <int P, bool GENO, int V>
bool private_staging(int nb, int table) {
    return smem_bytes_t<P, GENO, V>(nb, table, Cfg<P, GENO, V>::EPI) <= kMaxSmem;
}

template <bool GENO>
size_t tc_smem_bytes_g(const ParseShape& sh) {
    const int t = smem_table(sh);
    switch (sh.P) {
        case 1: return smem_bytes_t<1, GENO>(sh.n_bins, t, 1);
        case 2: return smem_bytes_t<2, GENO>(sh.n_bins, t, 1);
        case 3: return smem_bytes_t<3, GENO>(sh.n_bins, t, 1);
        default: return smem_bytes_t<4, GENO>(sh.n_bins, t, 1);
    }
}

// Haplotype path: the reciprocal table goes to the workspace when it does not fit in shared
// memory beside the widest tile's pipeline -- with per-warp staging if that fits without
// the table (per-warp staging matters more than a shared-memory table), else beside one
// shared staging copy.
template <int P>
bool rtab_global_t(const ParseShape& sh) {
    using C = Cfg<P, false, 0>;
    const int nb = sh.n_bins, t = sh.max_n + 1;
    if (smem_bytes_t<P, false, 0>(nb, t, C::EPI) <= kMaxSmem) return false;
    if (smem_bytes_t<P, false, 0>(nb, 0, C::EPI) <= kMaxSmem) return true;
    return smem_bytes_t<P, false, 0>(nb, t, 1) > kMaxSmem;
}

template <int P, typename T, bool PRIV, bool GENO, int V, bool GT>
cudaError_t launch_parse_tc_p(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w,
                                     const ParseShape& sh, int max_items, cudaStream_t s) {
    using C = Cfg<P, GENO, V>;
    // A: the row block (haplotypes: both planes of 64 SNPs; genotypes: one plane of 128
    // SNPs per box); B: every plane of NJ partners
    CUtensorMap mA, mB;
    if (!make_map(&mA, w.hv, d->n_var, sh.ktot, C::PLANES, GENO ? 1 : C::PLANES, C::ROWS) ||
        !make_map(&mB, w.hv, d->n_var, sh.ktot, C::PLANES, C::PLANES, C::NJ))
        return cudaErrorInvalidValue;
    TcArgs a;
    a.coord = d->coord ? d->coord : d->pos;
    a.jmax = w.jmax;
    a.snp_block = d->snp_block;
    a.n_blocks = d->n_blocks;
    a.items = w.items;
    a.n_items = w.n_items;
    a.item_counter = w.item_counter;
    a.nkc = sh.ktot / kKChunk;
    for (int p = 0; p <= LDK_MAX_POPS; ++p) a.kofs[p] = sh.kofs[p];
    a.max_n = sh.max_n;
    a.edges.n_bins = d->n_bins;
    for (int b = 0; b <= LDK_MAX_BINS; ++b) a.edges.e[b] = b <= d->n_bins ? d->edges[b] : 0.0;
    a.fx = w.fx;
    a.pairs = reinterpret_cast<unsigned long long*>(o->pairs);
    a.r2_counts = reinterpret_cast<unsigned long long*>(o->r2_counts);
    a.status = w.status;
    a.rtab_g = static_cast<const double4*>(w.rtab);
    a.gtab = static_cast<const GenoRecip*>(w.gtab);
    // at least half of an SM's shared memory, so that one CTA (holding all 512 TMEM
    // columns) runs per SM
    size_t smem = smem_bytes_t<P, GENO, V>(d->n_bins, smem_table(sh), PRIV ? C::EPI : 1);
    if (smem < kMinSmem) smem = kMinSmem;
    if (smem > kMaxSmem) return cudaErrorInvalidConfiguration;
    cudaError_t e =
        cudaFuncSetAttribute(k_parse_tc<P, T, PRIV, GENO, V, GT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if constexpr (C::SPLIT) {
        // the register split adds up only at C::REG_LAUNCH registers per thread; any other
        // allocation would leave setmaxnreg.inc waiting, so such a build is not launched
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, k_parse_tc<P, T, PRIV, GENO, V, GT>);
        if (e != cudaSuccess) return e;
        if (fa.numRegs != C::REG_LAUNCH) return cudaErrorInvalidKernelImage;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (max_items == 0) return cudaSuccess;
    const int grid = max_items < sms ? max_items : sms;
    k_parse_tc<P, T, PRIV, GENO, V, GT><<<grid, C::THREADS, smem, s>>>(mA, mB, a);
    return cudaGetLastError();
}


// One population count of one tile variant: per-warp or shared staging, and the reciprocal
// table in shared memory or (FP64 estimators, widest tile only) in the workspace.  Other
// variants answer cudaErrorInvalidConfiguration for a workspace table, which the tile
// autotuner reads as "does not fit this shape".
template <int PP, bool GENO, int V, typename T>
cudaError_t launch_staged(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, const ParseShape& sh,
                          int max_items, cudaStream_t s) {
    const bool priv = private_staging<PP, GENO, V>(sh.n_bins, smem_table(sh));
    if (!GENO && sh.rtab_global) {
        if constexpr (!GENO && V == 0 && std::is_same<T, double>::value)
            return priv ? launch_parse_tc_p<PP, T, true, GENO, V, true>(d, o, w, sh, max_items, s)
                        : launch_parse_tc_p<PP, T, false, GENO, V, true>(d, o, w, sh, max_items, s);
        else
            return cudaErrorInvalidConfiguration;
    }
    return priv ? launch_parse_tc_p<PP, T, true, GENO, V, false>(d, o, w, sh, max_items, s)
                : launch_parse_tc_p<PP, T, false, GENO, V, false>(d, o, w, sh, max_items, s);
}

// One tile variant of one path, over the population count, accumulator type and staging.
template <bool GENO, int V, typename T>
cudaError_t dispatch_tc(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, const ParseShape& sh,
                        int max_items, cudaStream_t s) {
#define LDK_TC_CASE(PP)                                                                                   \
    case PP:                                                                                              \
        return launch_staged<PP, GENO, V, T>(d, o, w, sh, max_items, s);
    switch (sh.P) {
        LDK_TC_CASE(1)
        LDK_TC_CASE(2)
        LDK_TC_CASE(3)
        LDK_TC_CASE(4)
        default: return cudaErrorInvalidValue;
    }
#undef LDK_TC_CASE
}

}  // namespace
}  // namespace ldk
