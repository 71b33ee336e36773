// All-pairs LD of one SNP set on the tensor-core count pipeline: pairwise r^2, the
// unbiased sigma_D^2 and r^2 from jointly valid counts for every pair i < j, written as a
// full symmetric matrix and/or reduced to the sum and count behind ZnS.
//
// The Gram counts come from the same TMA + tcgen05 pipeline as the binned parse (64-SNP
// row blocks against 128-SNP partner tiles, no distance cutoff, so every partner j > i of
// the set).  Four epilogue warps share each TMEM lane quarter (16 SNPs), one per quarter
// of the partner tile; each evaluates its 16 rows x 32 partners into a padded
// shared-memory tile and then writes the tile's rows (upper triangle, 256-byte runs) and
// columns (lower triangle, 128-byte runs) with coalesced stores.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ldk_tc_kernel.cuh"
#include "ldk_geno_feat.cuh"

namespace ldk {

namespace {

using LdmCfg = Cfg<1, false, 0>;
constexpr int kLdmEpi = 16;                    // epilogue warps: four per TMEM lane quarter
constexpr int kLdmParts = kLdmEpi / 4;         // partner ranges a tile is split into
constexpr int kLdmHalf = LdmCfg::NJ / kLdmParts;  // partners per epilogue warp and tile
constexpr int kLdmStride = kLdmHalf + 1;       // staging row stride (doubles): rows hit distinct banks

struct LdmArgs {
    const double* psite;  // per SNP: derived allele frequency over the site's valid haplotypes
    double* out;          // (n_var rows, stride ld_out) or null
    int64_t ld_out;
    double* sums;         // [sum over pairs i < j, pairs counted] or null
};

__global__ void k_fill_int(int32_t* p, int64_t n, int32_t v) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        p[t] = v;
}

__global__ void k_fill_diag(double* out, int64_t ld, int64_t n, double v) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        out[t * ld + t] = v;
}

// p_i = (sum of derived calls) / (valid calls), 0 for a site without valid calls
// (haplotype_matrix.py:1119-1120), over the selected rows.
__global__ void k_site_freq(const int8_t* __restrict__ X, int64_t ld, int64_t n_var, const int32_t* __restrict__ rows,
                            int n_rows, double* __restrict__ p) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n_var; v += (int64_t)gridDim.x * blockDim.x) {
        int dac = 0, nv = 0;
        for (int k = 0; k < n_rows; ++k) {
            const int8_t x = X[(int64_t)rows[k] * ld + v];
            dac += x > 0 ? x : 0;
            nv += x >= 0;
        }
        p[v] = nv > 0 ? (double)dac / (double)nv : 0.0;
    }
}

template <int EST>
__global__ void __launch_bounds__(128 + 32 * kLdmEpi, 1)
    k_ld_matrix(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const TcArgs a,
                const LdmArgs m) {
    using C = LdmCfg;
    constexpr int NJ = C::NJ, SP = kLdmStride;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* stages = base;
    double* stile = reinterpret_cast<double*>(base + C::STAGES * C::STAGE_BYTES);  // [kLdmEpi][16][SP]

    __shared__ __align__(8) uint64_t full_bar[C::STAGES], empty_bar[C::STAGES], tfull[C::NBUF], tempty[C::NBUF];
    __shared__ __align__(8) uint64_t ifull[kRing], iempty[kRing];
    __shared__ volatile int ring[2 * kRing];
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < C::NBUF; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], kLdmEpi);
        }
        for (int b = 0; b < kRing; ++b) {
            mbar_init(&ifull[b], 1);
            mbar_init(&iempty[b], 1 + kLdmEpi);
        }
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(&tmem_base_s, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    const Pipe pipe{stages, full_bar, empty_bar, tfull, tempty, ifull, iempty, ring, &abort_s};
    if (warp == 0) run_producer<C>(pipe, &tmA, &tmB, a, lane);
    else if (warp == 1) run_mma<C, 1>(pipe, tmem, a, lane);
    if (warp >= 4) {
        // lanes 2r, 2r+1 share SNP r (16 per warp) and split its partners by parity; the
        // warp takes part `half` (of kLdmParts) of every partner tile
        const int e = warp - 4, quarter = warp & 3, half = e >> 2;
        const int rr = lane >> 1, role = lane & 1;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        double* st = stile + e * 16 * SP;
        double zsum = 0.0, zcnt = 0.0;
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
            if (epi_bar_or<kLdmEpi>(abort_s != 0 || item < 0)) break;
            int row0, row1, jt0;
            const int n_jt = item_tiles<C>(a, item, row0, row1, jt0);
            if (n_jt == 0) continue;
            const int jend = a.jmax[row1 - 1];
            const int i = row0 + quarter * 16 + rr;
            const bool row_ok = i < row1;
            const double pi = (EST == 0 && row_ok) ? m.psite[i] : 0.0;
            bool ok = true;
            for (int t = 0; t < n_jt; ++t, ++tcount) {
                const uint32_t buf = tcount % C::NBUF, tph = (tcount / C::NBUF) & 1u;
                const int j0 = jt0 + t * NJ;
                double preg[(kLdmHalf + 31) / 32];
#pragma unroll
                for (int kk = 0; kk < (kLdmHalf + 31) / 32; ++kk) {
                    const int j = j0 + half * kLdmHalf + 32 * kk + lane;
                    preg[kk] = (EST == 0 && j < jend) ? m.psite[j] : 0.0;
                }
                if (!mbar_wait(&tfull[buf], tph, &abort_s, a.status)) { ok = false; break; }
                tc_fence_after();
#pragma unroll 1
                for (int qh = 0; qh < kLdmHalf / 2; ++qh) {
                    const int q = half * (kLdmHalf / 2) + qh;
                    uint32_t v[1][4];
                    tmem_ld4(tmem + lane_base + buf * C::COLS + q * 4, v[0]);
                    const int jl = 2 * qh + role;  // partner within this warp's half tile
                    const int jj = half * kLdmHalf + jl;
                    double psrc = preg[0];
#pragma unroll
                    for (int kk = 1; kk < (kLdmHalf + 31) / 32; ++kk)
                        if ((jl >> 5) == kk) psrc = preg[kk];
                    const double pj = __shfl_sync(0xffffffffu, psrc, jl & 31);
                    tmem_wait4<1>(v);
                    if (qh == kLdmHalf / 2 - 1) {
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&tempty[buf]);
                    }
                    // lane 2r: (hh, hv) of partners 2q, 2q+1; lane 2r+1: (vh, vv)
                    const uint32_t sx = role ? v[0][0] : v[0][2];
                    const uint32_t sy = role ? v[0][1] : v[0][3];
                    const uint32_t rx = __shfl_xor_sync(0xffffffffu, sx, 1);
                    const uint32_t ry = __shfl_xor_sync(0xffffffffu, sy, 1);
                    int hh, hv, vh, vv;
                    if (role == 0) { hh = (int)v[0][0]; hv = (int)v[0][1]; vh = (int)rx; vv = (int)ry; }
                    else { vh = (int)v[0][2]; vv = (int)v[0][3]; hh = (int)rx; hv = (int)ry; }
                    const int j = j0 + jj;
                    const bool valid = row_ok && j > i && j < jend;
                    double val = 0.0;
                    if (valid) {
                        const double c1 = hh, c2 = hv - hh, c3 = vh - hh, c4 = vv - hv - vh + hh, n = vv;
                        if constexpr (EST == 0) {
                            // haplotype_matrix.py:1122-1128, 1171-1175
                            const double pab = n > 0.0 ? c1 * recip_newton(n) : 0.0;
                            const double D = pab - pi * pj;
                            const double den = (pi * (1.0 - pi)) * (pj * (1.0 - pj));
                            val = den > 0.0 ? (D * D) * recip_newton(den) : 0.0;
                            zsum += val;
                            zcnt += 1.0;
                        } else if constexpr (EST == 1) {
                            // ld_statistics.py:326-343 (exact integers in FP64)
                            const double dd = c1 * (c1 - 1) * c4 * (c4 - 1) + c2 * (c2 - 1) * c3 * (c3 - 1) -
                                              2.0 * c1 * c2 * c3 * c4;
                            const double s12 = c1 + c2, s13 = c1 + c3, s24 = c2 + c4, s34 = c3 + c4;
                            const double pi2 = s12 * s13 * s24 * s34 - c1 * c4 * (-1.0 + c1 + 3.0 * c2 + 3.0 * c3 + c4) -
                                               c2 * c3 * (-1.0 + 3.0 * c1 + c2 + c3 + 3.0 * c4);
                            const bool nok = n >= 4.0;
                            val = (nok && pi2 != 0.0) ? dd * recip_newton(pi2) : 0.0;
                            zsum += val;
                            zcnt += nok ? 1.0 : 0.0;
                        } else {
                            // haplotype_kernels.py:32-42: NaN where pA qA pB qB = 0
                            const double D = c1 * c4 - c2 * c3;
                            const double den = (c1 + c2) * (c3 + c4) * ((c1 + c3) * (c2 + c4));
                            if (den > 0.0) {
                                val = (D * D) * recip_newton(den);
                                zsum += val;
                                zcnt += 1.0;
                            } else {
                                val = CUDART_NAN;
                            }
                        }
                    }
                    st[rr * SP + jl] = val;
                }
                __syncwarp();
                if (m.out) {
                    const int gi0 = row0 + quarter * 16, gj0 = j0 + half * kLdmHalf;
                    for (int idx = lane; idx < 16 * kLdmHalf; idx += 32) {  // rows: upper triangle
                        const int r = idx / kLdmHalf, c = idx % kLdmHalf, gi = gi0 + r, gj = gj0 + c;
                        if (gi < row1 && gj > gi && gj < jend) m.out[(int64_t)gi * m.ld_out + gj] = st[r * SP + c];
                    }
                    for (int idx = lane; idx < 16 * kLdmHalf; idx += 32) {  // columns: lower triangle
                        const int r = idx % 16, c = idx / 16, gi = gi0 + r, gj = gj0 + c;
                        if (gi < row1 && gj > gi && gj < jend) m.out[(int64_t)gj * m.ld_out + gi] = st[r * SP + c];
                    }
                }
                __syncwarp();
            }
            (void)ok;
        }
        if (m.sums) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                zsum += __shfl_xor_sync(0xffffffffu, zsum, o);
                zcnt += __shfl_xor_sync(0xffffffffu, zcnt, o);
            }
            if (lane == 0) {
                atomicAdd(&m.sums[0], zsum);
                atomicAdd(&m.sums[1], zcnt);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}


// ---- genotype path: dosage r^2, Rogers-Huff r, sigma_D^2 of genotype pairs ----------------

using LdmGCfg = Cfg<1, true, 0>;               // 128-SNP row blocks, 16-partner tiles
constexpr int kLdmGEpi = 8;                    // two epilogue warps per TMEM lane quarter
constexpr int kLdmGPart = LdmGCfg::NJ / 2;     // partners per epilogue warp and tile
constexpr int kLdmGStride = kLdmGPart + 1;

struct LdmGArgs {
    const double* mu;   // per SNP: mean dosage over the site's valid individuals
    const double* var;  // per SNP: sum of squared deviations from it over those individuals
    double* out;
    int64_t ld_out;
    double* sums;
    double n_ind;       // individuals (Rogers-Huff r: all valid)
};

// mu and the sum of squared deviations per SNP over the selected rows (ld_statistics.py:
// 1000-1011); with `strict` a missing call sets LDK_DEVERR_BAD_INPUT (the Rogers-Huff and
// sigma_D^2 genotype estimators take complete data, ld_statistics.py:389-399).
__global__ void k_site_moments(const int8_t* __restrict__ X, int64_t ld, int64_t n_var, const int32_t* __restrict__ rows,
                               int n_rows, int strict, double* __restrict__ mu, double* __restrict__ var,
                               unsigned* status) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n_var; v += (int64_t)gridDim.x * blockDim.x) {
        int sum = 0, nv = 0;
        for (int k = 0; k < n_rows; ++k) {
            const int8_t x = X[(int64_t)rows[k] * ld + v];
            if (x >= 0) { sum += x; ++nv; }
        }
        if (strict && nv < n_rows) atomicOr(status, LDK_DEVERR_BAD_INPUT);
        const double m = nv > 0 ? (double)sum / (double)nv : 0.0;
        double ss = 0.0;
        for (int k = 0; k < n_rows; ++k) {
            const int8_t x = X[(int64_t)rows[k] * ld + v];
            if (x >= 0) ss += ((double)x - m) * ((double)x - m);
        }
        mu[v] = m;
        var[v] = ss;
    }
}

template <int EST>
__global__ void __launch_bounds__(128 + 32 * kLdmGEpi, 1)
    k_ld_matrix_geno(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const TcArgs a,
                     const LdmGArgs m) {
    using C = LdmGCfg;
    constexpr int NJ = C::NJ, SP = kLdmGStride;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* stages = base;
    double* stile = reinterpret_cast<double*>(base + C::STAGES * C::STAGE_BYTES);  // [kLdmGEpi][32][SP]

    __shared__ __align__(8) uint64_t full_bar[C::STAGES], empty_bar[C::STAGES], tfull[C::NBUF], tempty[C::NBUF];
    __shared__ __align__(8) uint64_t ifull[kRing], iempty[kRing];
    __shared__ volatile int ring[2 * kRing];
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < C::NBUF; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], kLdmGEpi);
        }
        for (int b = 0; b < kRing; ++b) {
            mbar_init(&ifull[b], 1);
            mbar_init(&iempty[b], 1 + kLdmGEpi);
        }
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        tmem_alloc(&tmem_base_s, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    const Pipe pipe{stages, full_bar, empty_bar, tfull, tempty, ifull, iempty, ring, &abort_s};
    if (warp == 0) run_producer<C>(pipe, &tmA, &tmB, a, lane);
    else if (warp == 1) run_mma<C, 1>(pipe, tmem, a, lane);
    if (warp >= 4) {
        // lane = SNP of the row block (32 per warp); the warp takes half `part` of every tile
        const int e = warp - 4, quarter = warp & 3, part = e >> 2;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        double* st = stile + e * 32 * SP;
        double zsum = 0.0, zcnt = 0.0;
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
            if (epi_bar_or<kLdmGEpi>(abort_s != 0 || item < 0)) break;
            int row0, row1, jt0;
            const int n_jt = item_tiles<C>(a, item, row0, row1, jt0);
            if (n_jt == 0) continue;
            const int jend = a.jmax[row1 - 1];
            const int i = row0 + quarter * 32 + lane;
            const bool row_ok = i < row1;
            const double mui = row_ok ? m.mu[i] : 0.0, vari = row_ok ? m.var[i] : 0.0;
            bool ok = true;
            for (int t = 0; t < n_jt; ++t, ++tcount) {
                const uint32_t buf = tcount % C::NBUF, tph = (tcount / C::NBUF) & 1u;
                const int j0 = jt0 + t * NJ;
                if (!mbar_wait(&tfull[buf], tph, &abort_s, a.status)) { ok = false; break; }
                tc_fence_after();
#pragma unroll 1
                for (int cl = 0; cl < kLdmGPart; ++cl) {
                    const int c = part * kLdmGPart + cl;
                    uint32_t G[3][4];
#pragma unroll
                    for (int x = 0; x < 3; ++x) tmem_ld4(tmem + lane_base + buf * C::COLS + x * C::N + 4 * c, G[x]);
                    const int j = j0 + c;
                    const double muj = j < jend ? m.mu[j] : 0.0, varj = j < jend ? m.var[j] : 0.0;
                    tmem_wait4<3>(G);
                    if (cl == kLdmGPart - 1) {
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&tempty[buf]);
                    }
                    const bool valid = row_ok && j > i && j < jend;
                    double val = 0.0;
                    if (valid) {
                        // G[x][y]: plane x of SNP i . plane y of SNP j (0: g == 1, 1: g == 2, 2: valid)
                        const int n11 = (int)G[0][0], n12 = (int)G[0][1], n21 = (int)G[1][0], n22 = (int)G[1][1];
                        const int n10 = (int)G[0][2] - n11 - n12, n20 = (int)G[1][2] - n21 - n22;
                        const int n01 = (int)G[2][0] - n11 - n21, n02 = (int)G[2][1] - n12 - n22;
                        const int nv = (int)G[2][2];
                        if constexpr (EST == 3 || EST == 4) {
                            const double sxy = (double)(n11 + 2 * (n12 + n21) + 4 * n22);
                            if constexpr (EST == 3) {
                                // centred dosages zeroed where missing (ld_statistics.py:1000-1018)
                                const double sx = (double)((n10 + n11 + n12) + 2 * (n20 + n21 + n22));
                                const double sy = (double)((n01 + n11 + n21) + 2 * (n02 + n12 + n22));
                                const double cov = sxy - muj * sx - mui * sy + mui * muj * (double)nv;
                                const double vv = vari * varj;
                                val = vv > 0.0 ? (cov * cov) / vv : 0.0;
                                zsum += val;
                                zcnt += 1.0;
                            } else {
                                // ld_statistics.py:392-437
                                const double cov = sxy - m.n_ind * mui * muj;
                                const double den = sqrt(vari * varj);
                                if (den > 0.0) {
                                    val = cov / den;
                                    zsum += val * val;
                                    zcnt += 1.0;
                                } else {
                                    val = CUDART_NAN;
                                }
                            }
                        } else {
                            // DD over pi2 numerators of one population (genotype_kernels.py:91-170)
                            const int n00 = nv - n01 - n02 - n10 - n11 - n12 - n20 - n21 - n22;
                            const double cd[9] = {(double)n00, (double)n01, (double)n02, (double)n10, (double)n11,
                                                  (double)n12, (double)n20, (double)n21, (double)n22};
                            GenoFeat<double> f;
                            geno_set_counts(f, cd);
                            f.n = (double)nv;
                            geno_features<double, 1>(f);
                            if (nv >= 4 && f.PI1 > 0.0) {
                                val = f.DD1 / f.PI1;
                                zsum += val;
                                zcnt += 1.0;
                            } else {
                                val = CUDART_NAN;
                            }
                        }
                    }
                    st[lane * SP + cl] = val;
                }
                __syncwarp();
                if (m.out) {
                    const int gi0 = row0 + quarter * 32, gj0 = j0 + part * kLdmGPart;
                    for (int idx = lane; idx < 32 * kLdmGPart; idx += 32) {  // rows: upper triangle
                        const int r = idx / kLdmGPart, cc = idx % kLdmGPart, gi = gi0 + r, gj = gj0 + cc;
                        if (gi < row1 && gj > gi && gj < jend) m.out[(int64_t)gi * m.ld_out + gj] = st[r * SP + cc];
                    }
                    for (int idx = lane; idx < 32 * kLdmGPart; idx += 32) {  // columns: lower triangle
                        const int r = idx % 32, cc = idx / 32, gi = gi0 + r, gj = gj0 + cc;
                        if (gi < row1 && gj > gi && gj < jend) m.out[(int64_t)gj * m.ld_out + gi] = st[r * SP + cc];
                    }
                }
                __syncwarp();
            }
            (void)ok;
        }
        if (m.sums) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                zsum += __shfl_xor_sync(0xffffffffu, zsum, o);
                zcnt += __shfl_xor_sync(0xffffffffu, zcnt, o);
            }
            if (lane == 0) {
                atomicAdd(&m.sums[0], zsum);
                atomicAdd(&m.sums[1], zcnt);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

struct LdmLayout {
    size_t status = 0, jmax = 0, items = 0, planes = 0, psite = 0, var = 0, total = 0;
    int n_items = 0, ktot = 0;
};

LdmLayout ldm_layout(int64_t n_var, int32_t n_sel, bool geno) {
    LdmLayout L;
    L.ktot = (int)(((n_sel + 31) / 32 * 32 + 127) / 128 * 128);
    const int rows = geno ? LdmGCfg::ROWS : LdmCfg::ROWS;
    L.n_items = (int)((n_var + rows - 1) / rows);
    auto up = [](size_t x, size_t a) { return (x + a - 1) / a * a; };
    size_t off = 256;
    L.jmax = off;
    off = up(off + (size_t)n_var * 4, 256);
    L.items = off;  // (row0, row1, 0, INT32_MAX): whole row blocks
    off = up(off + (size_t)L.n_items * 16, 1024);
    L.planes = off;
    off = up(off + (size_t)n_var * (geno ? 4 : 2) * L.ktot, 256);
    L.psite = off;
    off = up(off + (size_t)n_var * 8, 256);
    L.var = off;
    off = up(off + (size_t)n_var * 8, 256);
    L.total = off;
    return L;
}

template <int EST>
cudaError_t launch_ldm_geno(const CUtensorMap& mA, const CUtensorMap& mB, const TcArgs& a, const LdmGArgs& m,
                            int n_items, cudaStream_t s) {
    using C = LdmGCfg;
    size_t smem = 1024 + (size_t)C::STAGES * C::STAGE_BYTES + (size_t)kLdmGEpi * 32 * kLdmGStride * sizeof(double);
    if (smem < kMinSmem) smem = kMinSmem;
    if (smem > kMaxSmem) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(k_ld_matrix_geno<EST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = n_items < sms ? n_items : sms;
    k_ld_matrix_geno<EST><<<grid, 128 + 32 * kLdmGEpi, smem, s>>>(mA, mB, a, m);
    return cudaGetLastError();
}

template <int EST>
cudaError_t launch_ldm(const CUtensorMap& mA, const CUtensorMap& mB, const TcArgs& a, const LdmArgs& m, int n_items,
                       cudaStream_t s) {
    using C = LdmCfg;
    size_t smem = 1024 + (size_t)C::STAGES * C::STAGE_BYTES + (size_t)kLdmEpi * 16 * kLdmStride * sizeof(double);
    if (smem < kMinSmem) smem = kMinSmem;
    cudaError_t e = cudaFuncSetAttribute(k_ld_matrix<EST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = n_items < sms ? n_items : sms;
    k_ld_matrix<EST><<<grid, 128 + 32 * kLdmEpi, smem, s>>>(mA, mB, a, m);
    return cudaGetLastError();
}

}  // namespace

size_t ld_matrix_workspace(int64_t n_var, int32_t n_sel) { return ldm_layout(n_var, n_sel, true).total; }

// Enqueues the all-pairs LD of the n_sel selected rows of X (see ldk_ld_matrix).
cudaError_t launch_ld_matrix(const int8_t* X, int64_t ld_x, int64_t n_var, const int32_t* rows, int32_t n_sel,
                             int estimator, double* out, int64_t ld_out, double* sums, unsigned char* ws,
                             unsigned* status, cudaStream_t s) {
    const bool geno = estimator >= 3;
    const LdmLayout L = ldm_layout(n_var, n_sel, geno);
    cudaError_t e;
    int32_t* jmax = reinterpret_cast<int32_t*>(ws + L.jmax);
    int32_t* items = reinterpret_cast<int32_t*>(ws + L.items);
    uint8_t* planes = ws + L.planes;
    double* psite = reinterpret_cast<double*>(ws + L.psite);
    double* svar = reinterpret_cast<double*>(ws + L.var);
    if (sums && (e = cudaMemsetAsync(sums, 0, 2 * sizeof(double), s)) != cudaSuccess) return e;
    if (out && n_var > 0) {
        const bool nan_diag = estimator == LDK_LDM_R2_COUNTS || estimator >= LDK_LDM_ROGERS_HUFF_R;
        k_fill_diag<<<(unsigned)((n_var + 255) / 256), 256, 0, s>>>(out, ld_out, n_var, nan_diag ? std::nan("") : 0.0);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (n_var < 2) return cudaSuccess;
    // every SNP's partner range is the rest of the set
    k_fill_int<<<(unsigned)((n_var + 255) / 256), 256, 0, s>>>(jmax, n_var, (int32_t)n_var);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int rows_per_block = geno ? LdmGCfg::ROWS : LdmCfg::ROWS;
    std::vector<int32_t> it;
    it.reserve((size_t)L.n_items * 4);
    for (int64_t r0 = 0; r0 < n_var; r0 += rows_per_block) {  // most partners first
        it.push_back((int32_t)r0);
        it.push_back((int32_t)std::min<int64_t>(r0 + rows_per_block, n_var));
        it.push_back(0);
        it.push_back(INT32_MAX);
    }
    int* n_items = reinterpret_cast<int*>(ws + 192);
    const int n_items_h = L.n_items;
    if ((e = cudaMemcpyAsync(items, it.data(), it.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(n_items, &n_items_h, sizeof(int), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return e;
    if (estimator == LDK_LDM_R2) {
        k_site_freq<<<(unsigned)((n_var + 255) / 256), 256, 0, s>>>(X, ld_x, n_var, rows, n_sel, psite);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (geno) {
        k_site_moments<<<(unsigned)((n_var + 255) / 256), 256, 0, s>>>(
            X, ld_x, n_var, rows, n_sel, estimator != LDK_LDM_DIPLOID_R2, psite, svar, status);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // the indicator planes of the selected rows, as for a one-population parse
    ldk_parse_t d{};
    d.genotypes = geno ? 1 : 0;
    d.X = X;
    d.ld_x = ld_x;
    d.n_var = n_var;
    d.pop_rows = rows;
    d.n_pops = 1;
    d.pop_offsets[0] = 0;
    for (int p = 1; p <= LDK_MAX_POPS; ++p) d.pop_offsets[p] = n_sel;
    ParseShape sh{};
    sh.P = 1;
    sh.genotypes = geno ? 1 : 0;
    sh.planes = geno ? 4 : 2;
    sh.ktot = L.ktot;
    for (int p = 0; p <= LDK_MAX_POPS; ++p) sh.kofs[p] = p == 0 ? 0 : (n_sel + 31) / 32 * 32;
    sh.max_n = n_sel;
    Scratch w{};
    w.status = status;
    w.hv = planes;
    if ((e = launch_prep_planes(&d, w, sh, s)) != cudaSuccess) return e;
    CUtensorMap mA, mB;
    if (geno ? (!make_map(&mA, planes, n_var, L.ktot, 4, 1, LdmGCfg::ROWS) ||
                !make_map(&mB, planes, n_var, L.ktot, 4, 4, LdmGCfg::NJ))
             : (!make_map(&mA, planes, n_var, L.ktot, 2, 2, LdmCfg::ROWS) ||
                !make_map(&mB, planes, n_var, L.ktot, 2, 2, LdmCfg::NJ)))
        return cudaErrorInvalidValue;
    TcArgs a{};
    a.jmax = jmax;
    a.items = items;
    a.n_items = n_items;
    a.item_counter = reinterpret_cast<int*>(ws + 128);
    a.nkc = L.ktot / kKChunk;
    for (int p = 0; p <= LDK_MAX_POPS; ++p) a.kofs[p] = sh.kofs[p];
    a.status = status;
    if (geno) {
        LdmGArgs g{psite, svar, out, ld_out, sums, (double)n_sel};
        switch (estimator) {
            case LDK_LDM_DIPLOID_R2: return launch_ldm_geno<3>(mA, mB, a, g, L.n_items, s);
            case LDK_LDM_ROGERS_HUFF_R: return launch_ldm_geno<4>(mA, mB, a, g, L.n_items, s);
            default: return launch_ldm_geno<5>(mA, mB, a, g, L.n_items, s);
        }
    }
    LdmArgs m{psite, out, ld_out, sums};
    switch (estimator) {
        case LDK_LDM_R2: return launch_ldm<0>(mA, mB, a, m, L.n_items, s);
        case LDK_LDM_SIGMA_D2: return launch_ldm<1>(mA, mB, a, m, L.n_items, s);
        default: return launch_ldm<2>(mA, mB, a, m, L.n_items, s);
    }
}

}  // namespace ldk
