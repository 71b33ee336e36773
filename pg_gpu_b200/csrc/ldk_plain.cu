// Plain FP64 kernels: the drop-in path.  One thread per SNP pair, byte-wise counting
// over each population's rows of the haplotype-major input (the layout and counting
// scheme of pg_gpu ld_pipeline.py:130-217), FP64 estimators, FP64 per-bin sums.
#include <cub/cub.cuh>

#include "ldk_estimators.cuh"
#include "ldk_internal.h"

namespace ldk {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n, int threads = kThreads) {
    int64_t b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : (b > (1ll << 30) ? (1ll << 30) : b));
}

// ---------------------------------------------------------------------------
// per-pair counts (ld_pipeline.py:155-172 and :183-217)
// ---------------------------------------------------------------------------

LDK_DEV void hap_count(const int8_t* __restrict__ X, int64_t ld, const int32_t* __restrict__ rows,
                       int n_rows, int64_t i, int64_t j, int& c11, int& c10, int& c01, int& c00,
                       int& valid) {
    c11 = c10 = c01 = c00 = valid = 0;
    for (int k = 0; k < n_rows; ++k) {
        const int64_t base = (int64_t)rows[k] * ld;
        const int x = X[base + i], y = X[base + j];
        const int v = (x >= 0) & (y >= 0);
        valid += v;
        c11 += (x == 1) & (y == 1);
        c10 += (x == 1) & (y == 0);
        c01 += (x == 0) & (y == 1);
        c00 += (x == 0) & (y == 0);
    }
}

LDK_DEV void geno_count(const int8_t* __restrict__ X, int64_t ld, const int32_t* __restrict__ rows,
                        int n_rows, int64_t i, int64_t j, int (&c)[9], int& valid) {
#pragma unroll
    for (int m = 0; m < 9; ++m) c[m] = 0;
    valid = 0;
    for (int k = 0; k < n_rows; ++k) {
        const int64_t base = (int64_t)rows[k] * ld;
        const int x = X[base + i], y = X[base + j];
        if (x >= 0 && y >= 0) {
            const int combo = x * 3 + y;
#pragma unroll
            for (int m = 0; m < 9; ++m) c[m] += (combo == m);
            ++valid;
        }
    }
}

__global__ void k_counts_hap(const int8_t* __restrict__ X, int64_t ld, const int32_t* __restrict__ rows,
                             int n_rows, const int32_t* __restrict__ ii, const int32_t* __restrict__ jj,
                             int64_t n, int32_t* __restrict__ counts, int32_t* __restrict__ n_valid) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        int c11, c10, c01, c00, v;
        hap_count(X, ld, rows, n_rows, ii[t], jj[t], c11, c10, c01, c00, v);
        int4 out = make_int4(c11, c10, c01, c00);
        reinterpret_cast<int4*>(counts)[t] = out;
        if (n_valid) n_valid[t] = v;
    }
}

__global__ void k_counts_geno(const int8_t* __restrict__ X, int64_t ld, const int32_t* __restrict__ rows,
                              int n_rows, const int32_t* __restrict__ ii, const int32_t* __restrict__ jj,
                              int64_t n, int32_t* __restrict__ counts, int32_t* __restrict__ n_valid) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        int c[9], v;
        geno_count(X, ld, rows, n_rows, ii[t], jj[t], c, v);
#pragma unroll
        for (int m = 0; m < 9; ++m) counts[t * 9 + m] = c[m];
        if (n_valid) n_valid[t] = v;
    }
}

// ---------------------------------------------------------------------------
// statistics from counts (haplotype_kernels.py:584-640, genotype_kernels.py:881-936)
// ---------------------------------------------------------------------------

template <int P>
__global__ void k_stats_hap(const int32_t* __restrict__ counts, const int32_t* __restrict__ n_valid,
                            int64_t n, double* __restrict__ out) {
    constexpr int NS = HapNStats<P>::value;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        HapFeat<double> f[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int4 c = reinterpret_cast<const int4*>(counts)[p * n + t];
            hap_set_counts(f[p], double(c.x), double(c.y), double(c.z), double(c.w));
            if (n_valid) f[p].n = double(n_valid[p * n + t]);
            hap_features<double, P>(f[p]);
            hap_reciprocals(f[p]);
        }
        double acc[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) acc[s] = 0.0;
        hap_stats<double, P>(f, acc);
#pragma unroll
        for (int s = 0; s < NS; ++s) out[t * NS + s] = acc[s];
    }
}

template <int P>
__global__ void k_stats_geno(const int32_t* __restrict__ counts, const int32_t* __restrict__ n_valid,
                             int64_t n, double* __restrict__ out) {
    constexpr int NS = HapNStats<P>::value;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        GenoFeat<double> f[P];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            double c[9];
#pragma unroll
            for (int m = 0; m < 9; ++m) c[m] = double(counts[(p * n + t) * 9 + m]);
            geno_set_counts(f[p], c);
            if (n_valid) f[p].n = double(n_valid[p * n + t]);
            geno_features<double, P>(f[p]);
        }
        double acc[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) acc[s] = 0.0;
        geno_stats<double, P>(f, acc);
#pragma unroll
        for (int s = 0; s < NS; ++s) out[t * NS + s] = acc[s];
    }
}

struct RawArgs {
    int g[4];
};

__global__ void k_raw_hap(int case_id, RawArgs args, int P_total, const double* __restrict__ counts,
                          const double* __restrict__ n_valid, int64_t n, double* __restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        HapFeat<double> f[LDK_MAX_POPS];
        for (int p = 0; p < P_total; ++p) {
            const double* c = counts + t * 4 * P_total + 4 * p;
            hap_set_counts(f[p], c[0], c[1], c[2], c[3]);
            if (n_valid) f[p].n = n_valid[t * P_total + p];
            hap_features<double, 4>(f[p]);
            hap_reciprocals(f[p]);
        }
        out[t] = hap_raw_by_case<double>(case_id, args.g, f);
    }
}

// r, r^2, D' in the frequency form of haplotype_kernels.py:20-62
__global__ void k_r_family(int which, const double* __restrict__ counts, const double* __restrict__ n_valid,
                           int64_t n, double* __restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
        const double a = counts[4 * t], b = counts[4 * t + 1], c = counts[4 * t + 2], d = counts[4 * t + 3];
        const double nn = n_valid ? n_valid[t] : a + b + c + d;
        const double pA = (a + b) / nn, pB = (a + c) / nn;
        const double D = (a * d - b * c) / (nn * nn);
        double v;
        if (which == 0 || which == 1) {
            const double den = pA * (1.0 - pA) * pB * (1.0 - pB);
            v = (den > 0.0) ? (which == 0 ? D / sqrt(den) : D * D / den) : nan("");
        } else {
            const double qA = 1.0 - pA, qB = 1.0 - pB;
            double dmax;
            if (D >= 0.0) dmax = fmin(pA * qB, qA * pB);
            else dmax = fmin(pA * pB, qA * qB);
            v = (dmax > 0.0) ? D / dmax : nan("");
        }
        out[t] = v;
    }
}

// ---------------------------------------------------------------------------
// pair ranges: jmax[i] = end of SNP i's partners (cutoff on pos, window end); i + 1 for
// SNPs after their window's anchor end (a split parse's right halo)
// ---------------------------------------------------------------------------

__global__ void k_jmax(const double* __restrict__ pos, const double* __restrict__ coord, int64_t n_var, const int64_t* __restrict__ win_off,
                       const int64_t* __restrict__ anc_end, int n_win, double max_dist, const int32_t* __restrict__ snp_block, int n_blocks,
                       int32_t* __restrict__ jmax, unsigned* __restrict__ status) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_var;
         i += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_win;  // window w with win_off[w] <= i < win_off[w+1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (win_off[mid] <= i) lo = mid; else hi = mid;
        }
        const int64_t we = win_off[lo + 1];
        const double lim = pos[i] + max_dist;
        int64_t a = i + 1, b = we;  // first j in [i+1, we) with pos[j] > lim
        while (a < b) {
            const int64_t m = (a + b) >> 1;
            if (pos[m] <= lim) a = m + 1; else b = m;
        }
        jmax[i] = (int32_t)(i < anc_end[lo] ? a : i + 1);  // SNPs past the anchors have no pairs of their own
        if (i + 1 < we && pos[i + 1] < pos[i]) atomicOr(status, LDK_DEVERR_BAD_INPUT);
        if (coord && i + 1 < we && coord[i + 1] < coord[i]) atomicOr(status, LDK_DEVERR_BAD_INPUT);
        if (snp_block) {
            const int blk = snp_block[i];
            if (blk < 0 || blk >= n_blocks) atomicOr(status, LDK_DEVERR_BLOCK_RANGE);
        }
    }
}

// ---------------------------------------------------------------------------
// the plain binned parse: one warp per anchor SNP i, lane per partner j (j = i+1+lane+32k)
// ---------------------------------------------------------------------------

struct PlainArgs {
    const int8_t* X;
    int64_t ld;
    int64_t n_var;
    const int32_t* pop_rows;
    int pop_off[LDK_MAX_POPS + 1];
    const double* coord;
    const int32_t* jmax;
    const int32_t* snp_block;
    int n_blocks;
    BinEdges edges;
    unsigned long long* fx;  // fixed-point bin sums [block][bin][NS + 1][kFxLimbs] (r^2 last)
    unsigned long long* pairs;
    unsigned long long* r2_counts;
    int* row_counter;
    unsigned* status;
};

constexpr int kRowChunk = 8;

template <int NS>
struct WarpSlab {  // warp-private staging of one bootstrap block's bin sums
    double* acc;   // [n_bins][NS + 1]: statistics then r^2 sum
    unsigned long long* cnt;  // [n_bins][2]: pairs, finite r^2
};

template <int NS>
LDK_DEV void slab_flush(const PlainArgs& a, WarpSlab<NS>& w, int blk, int lane) {
    const int nb = a.edges.n_bins;
    for (int idx = lane; idx < nb * (NS + 1); idx += 32) {
        const int b = idx / (NS + 1), s = idx % (NS + 1);
        const double v = w.acc[idx];
        if (v != 0.0) fx_add(a.fx + (((int64_t)blk * nb + b) * (NS + 1) + s) * kFxLimbs, v, a.status);
        w.acc[idx] = 0.0;
    }
    for (int b = lane; b < nb; b += 32) {
        if (w.cnt[2 * b]) atomicAdd(&a.pairs[(int64_t)blk * nb + b], w.cnt[2 * b]);
        if (w.cnt[2 * b + 1]) atomicAdd(&a.r2_counts[(int64_t)blk * nb + b], w.cnt[2 * b + 1]);
        w.cnt[2 * b] = 0;
        w.cnt[2 * b + 1] = 0;
    }
    __syncwarp();
}

template <int P, bool GENO>
__global__ void __launch_bounds__(kThreads) k_parse_plain(PlainArgs a) {
    constexpr int NS = HapNStats<P>::value;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nb = a.edges.n_bins;
    const size_t slab_bytes = (size_t)nb * (NS + 1) * sizeof(double) + (size_t)nb * 2 * sizeof(unsigned long long);
    WarpSlab<NS> w;
    w.acc = reinterpret_cast<double*>(smem_raw + warp * slab_bytes);
    w.cnt = reinterpret_cast<unsigned long long*>(smem_raw + warp * slab_bytes + (size_t)nb * (NS + 1) * sizeof(double));
    __shared__ BinEdges sE;
    if (threadIdx.x == 0) sE = a.edges;
    for (int idx = lane; idx < nb * (NS + 1); idx += 32) w.acc[idx] = 0.0;
    for (int idx = lane; idx < 2 * nb; idx += 32) w.cnt[idx] = 0;
    __syncthreads();

    int cur_blk = -1;
    for (;;) {
        int r0 = 0;
        if (lane == 0) r0 = atomicAdd(a.row_counter, kRowChunk);
        r0 = __shfl_sync(0xffffffffu, r0, 0);
        if (r0 >= a.n_var) break;
        const int64_t r1e = (int64_t)r0 + kRowChunk;
        const int r1 = (int)(r1e < a.n_var ? r1e : a.n_var);
        for (int i = r0; i < r1; ++i) {
            const int jend = a.jmax[i];
            if (jend <= i + 1) continue;
            const int blk = a.snp_block ? a.snp_block[i] : 0;
            if (blk < 0 || blk >= a.n_blocks) continue;  // reported by k_jmax
            if (blk != cur_blk) {
                if (cur_blk >= 0) slab_flush<NS>(a, w, cur_blk, lane);
                cur_blk = blk;
            }
            const double ci = a.coord[i];
            for (int j0 = i + 1; j0 < jend; j0 += 32) {
                const int j = j0 + lane;
                const bool valid = j < jend;
                double v[NS];
#pragma unroll
                for (int s = 0; s < NS; ++s) v[s] = 0.0;
                double r2 = 0.0;
                bool r2ok = false;
                int bin = -1;
                if (valid) {
                    bin = bin_of(sE, fabs(a.coord[j] - ci));
                    if (bin >= nb) bin = -1;
                }
                if (bin >= 0) {
                    if constexpr (!GENO) {
                        HapFeat<double> f[P];
#pragma unroll
                        for (int p = 0; p < P; ++p) {
                            int c11, c10, c01, c00, nv;
                            hap_count(a.X, a.ld, a.pop_rows + a.pop_off[p], a.pop_off[p + 1] - a.pop_off[p],
                                      i, j, c11, c10, c01, c00, nv);
                            hap_set_counts(f[p], double(c11), double(c10), double(c01), double(c00));
                            f[p].n = double(nv);
                            hap_features<double, P>(f[p]);
                            hap_reciprocals(f[p]);
                        }
                        hap_stats<double, P>(f, v);
                        r2ok = hap_r2(f[0], r2);
                    } else {
                        GenoFeat<double> f[P];
                        double c0[9];
#pragma unroll
                        for (int p = 0; p < P; ++p) {
                            int c[9], nv;
                            geno_count(a.X, a.ld, a.pop_rows + a.pop_off[p], a.pop_off[p + 1] - a.pop_off[p],
                                       i, j, c, nv);
                            double cd[9];
#pragma unroll
                            for (int m = 0; m < 9; ++m) cd[m] = double(c[m]);
                            if (p == 0) {
#pragma unroll
                                for (int m = 0; m < 9; ++m) c0[m] = cd[m];
                            }
                            geno_set_counts(f[p], cd);
                            f[p].n = double(nv);
                            geno_features<double, P>(f[p]);
                        }
                        geno_stats<double, P>(f, v);
                        r2ok = geno_dosage_r2(c0, r2);
                    }
                }
                // warp accumulation into the warp-private slab
                const unsigned any = __ballot_sync(0xffffffffu, bin >= 0);
                if (!any) continue;
                const int b0 = __shfl_sync(0xffffffffu, bin, __ffs(any) - 1);
                const bool uniform = __all_sync(0xffffffffu, bin < 0 || bin == b0);
                if (uniform) {
#pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        double x = v[s];
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                        if (lane == 0) w.acc[b0 * (NS + 1) + s] += x;
                    }
                    double x = r2ok ? r2 : 0.0;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                    const unsigned nr2 = __popc(__ballot_sync(0xffffffffu, r2ok && bin >= 0));
                    if (lane == 0) {
                        w.acc[b0 * (NS + 1) + NS] += x;
                        w.cnt[2 * b0] += __popc(any);
                        w.cnt[2 * b0 + 1] += nr2;
                    }
                } else {
                    for (int l = 0; l < 32; ++l) {
                        if (lane == l && bin >= 0) {
#pragma unroll
                            for (int s = 0; s < NS; ++s) w.acc[bin * (NS + 1) + s] += v[s];
                            if (r2ok) {
                                w.acc[bin * (NS + 1) + NS] += r2;
                                w.cnt[2 * bin + 1] += 1;
                            }
                            w.cnt[2 * bin] += 1;
                        }
                        __syncwarp();
                    }
                }
                __syncwarp();
            }
        }
        // flush once per claimed chunk: a slab then holds the sums of one chunk's rows in a
        // fixed order, whichever warp claimed it, so the fixed-point totals are reproducible
        if (cur_blk >= 0) slab_flush<NS>(a, w, cur_blk, lane);
        cur_blk = -1;
    }
}

template <int P, bool GENO>
cudaError_t launch_parse_plain_t(const PlainArgs& a, int nb, cudaStream_t s) {
    constexpr int NS = HapNStats<P>::value;
    const size_t slab = (size_t)nb * (NS + 1) * sizeof(double) + (size_t)nb * 2 * sizeof(unsigned long long);
    int warps = 8;
    while (warps > 1 && slab * warps > 160 * 1024) warps >>= 1;
    const size_t smem = slab * warps;
    if (smem > 200 * 1024) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaFuncSetAttribute(k_parse_plain<P, GENO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_parse_plain<P, GENO>, 32 * warps, smem);
    if (per_sm < 1) per_sm = 1;
    k_parse_plain<P, GENO><<<sms * per_sm, 32 * warps, smem, s>>>(a);
    return cudaGetLastError();
}

// Row blocks of 64 (genotypes: 128) anchor SNPs per window, in window order (one thread: a
// setup step).
__global__ void k_build_items(const int64_t* __restrict__ win_off, const int64_t* __restrict__ anc_end, int n_win,
                              int rows, int32_t* __restrict__ row_blocks) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int k = 0;
    for (int wi = 0; wi < n_win; ++wi)
        for (int64_t r0 = win_off[wi]; r0 < anc_end[wi]; r0 += rows) {
            row_blocks[2 * k] = (int32_t)r0;
            const int64_t r1 = r0 + rows < anc_end[wi] ? r0 + rows : anc_end[wi];
            row_blocks[2 * k + 1] = (int32_t)r1;
            ++k;
        }
}

// sums[blk][bin][s] (s < NS) and r2_sums[blk][bin] from the fixed-point accumulators
__global__ void k_fx_finish(const unsigned long long* __restrict__ fx, int64_t n_rows, int NS,
                            double* __restrict__ sums, double* __restrict__ r2_sums) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_rows * (NS + 1);
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / (NS + 1);
        const int s = (int)(t % (NS + 1));
        const double v = fx_value(fx + t * kFxLimbs);
        if (s < NS) sums[row * NS + s] = v;
        else r2_sums[row] = v;
    }
}

__global__ void k_block_combine(const double* __restrict__ block_sums, int64_t n_blocks, int64_t k,
                                const int32_t* __restrict__ weights, int64_t n_rep, double* __restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_rep * k;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t / k, c = t % k;
        double acc = 0.0;
        for (int64_t b = 0; b < n_blocks; ++b) {
            const int32_t wgt = weights[r * n_blocks + b];
            if (wgt) acc += double(wgt) * block_sums[b * k + c];
        }
        out[t] = acc;
    }
}

}  // namespace

cudaError_t launch_counts(int genotypes, const int8_t* X, int64_t ld, const int32_t* rows, int n_rows,
                          const int32_t* ii, const int32_t* jj, int64_t n, int32_t* counts,
                          int32_t* n_valid, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const int grid = blocks_for(n);
    if (genotypes) k_counts_geno<<<grid, kThreads, 0, s>>>(X, ld, rows, n_rows, ii, jj, n, counts, n_valid);
    else k_counts_hap<<<grid, kThreads, 0, s>>>(X, ld, rows, n_rows, ii, jj, n, counts, n_valid);
    return cudaGetLastError();
}

cudaError_t launch_stats(int genotypes, int P, const int32_t* counts, const int32_t* n_valid, int64_t n,
                         double* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const int grid = blocks_for(n, 128);
#define LDK_STATS_CASE(PP)                                                                     \
    case PP:                                                                                   \
        if (genotypes) k_stats_geno<PP><<<grid, 128, 0, s>>>(counts, n_valid, n, out);         \
        else k_stats_hap<PP><<<grid, 128, 0, s>>>(counts, n_valid, n, out);                    \
        break;
    switch (P) {
        LDK_STATS_CASE(1)
        LDK_STATS_CASE(2)
        LDK_STATS_CASE(3)
        LDK_STATS_CASE(4)
        default: return cudaErrorInvalidValue;
    }
#undef LDK_STATS_CASE
    return cudaGetLastError();
}

cudaError_t launch_raw_hap(int case_id, const int32_t* args, int P_total, const double* counts,
                           const double* n_valid, int64_t n, double* out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    RawArgs ra;
    for (int k = 0; k < 4; ++k) ra.g[k] = args[k];
    k_raw_hap<<<blocks_for(n, 128), 128, 0, s>>>(case_id, ra, P_total, counts, n_valid, n, out);
    return cudaGetLastError();
}

cudaError_t launch_r_family(int which, const double* counts, const double* n_valid, int64_t n, double* out,
                            cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_r_family<<<blocks_for(n), kThreads, 0, s>>>(which, counts, n_valid, n, out);
    return cudaGetLastError();
}

cudaError_t launch_jmax(const ldk_parse_t* d, const Scratch& w, cudaStream_t s) {
    if (d->n_var == 0) return cudaSuccess;
    k_jmax<<<blocks_for(d->n_var), kThreads, 0, s>>>(d->pos, d->coord, d->n_var, w.win_off, w.anc_end, d->n_windows,
                                                      d->max_dist,
                                                      d->snp_block, d->n_blocks, w.jmax, w.status);
    return cudaGetLastError();
}

cudaError_t launch_parse_plain(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w,
                               const ParseShape& sh, cudaStream_t s) {
    PlainArgs a;
    a.X = d->X;
    a.ld = d->ld_x;
    a.n_var = d->n_var;
    a.pop_rows = d->pop_rows;
    for (int p = 0; p <= LDK_MAX_POPS; ++p) a.pop_off[p] = d->pop_offsets[p];
    a.coord = d->coord ? d->coord : d->pos;
    a.jmax = w.jmax;
    a.snp_block = d->snp_block;
    a.n_blocks = d->n_blocks;
    a.edges.n_bins = d->n_bins;
    for (int b = 0; b <= LDK_MAX_BINS; ++b) a.edges.e[b] = b <= d->n_bins ? d->edges[b] : 0.0;
    a.fx = w.fx;
    a.pairs = reinterpret_cast<unsigned long long*>(o->pairs);
    a.r2_counts = reinterpret_cast<unsigned long long*>(o->r2_counts);
    a.row_counter = w.row_counter;
    a.status = w.status;
#define LDK_PLAIN_CASE(PP)                                                               \
    case PP:                                                                             \
        return d->genotypes ? launch_parse_plain_t<PP, true>(a, d->n_bins, s)            \
                            : launch_parse_plain_t<PP, false>(a, d->n_bins, s);
    switch (sh.P) {
        LDK_PLAIN_CASE(1)
        LDK_PLAIN_CASE(2)
        LDK_PLAIN_CASE(3)
        LDK_PLAIN_CASE(4)
        default: return cudaErrorInvalidValue;
    }
#undef LDK_PLAIN_CASE
}

cudaError_t launch_build_items(const Scratch& w, int n_windows, int rows, cudaStream_t s) {
    k_build_items<<<1, 1, 0, s>>>(w.win_off, w.anc_end, n_windows, rows, w.row_blocks);
    return cudaGetLastError();
}

cudaError_t launch_fx_finish(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, int n_stats,
                             cudaStream_t s) {
    const int64_t rows = (int64_t)d->n_blocks * d->n_bins;
    k_fx_finish<<<blocks_for(rows * (n_stats + 1)), kThreads, 0, s>>>(w.fx, rows, n_stats, o->sums, o->r2_sums);
    return cudaGetLastError();
}

cudaError_t launch_block_combine(const double* block_sums, int64_t n_blocks, int64_t k, const int32_t* weights,
                                 int64_t n_rep, double* out, cudaStream_t s) {
    if (n_rep * k == 0) return cudaSuccess;
    k_block_combine<<<blocks_for(n_rep * k), kThreads, 0, s>>>(block_sums, n_blocks, k, weights, n_rep, out);
    return cudaGetLastError();
}

}  // namespace ldk
