// Tensor-core path of the binned parse: indicator-plane preparation, tile-variant
// dispatch and the peak probes (the kernel itself is in ldk_tc_kernel.cuh).
#include "ldk_tc_kernel.cuh"

namespace ldk {

namespace {
// ---------------------------------------------------------------------------
// indicator planes.  Haplotypes: planes[v][0][k] = [x == 1], planes[v][1][k] = [x in {0, 1}].
// Genotypes: planes[v][0..3][k] = [x == 1], [x == 2], [x in {0, 1, 2}], 0.
// ---------------------------------------------------------------------------

struct PrepArgs {
    const int8_t* X;
    int64_t ld;
    int64_t n_var;
    const int32_t* pop_rows;
    int pop_off[LDK_MAX_POPS + 1];
    int kofs[LDK_MAX_POPS + 1];
    int P;
    int ktot;
    int genotypes;
    int planes;
    uint8_t* planes_out;
    unsigned* status;
};  // X: int8 codes, or (PACKED) 2-bit codes + 1, four SNPs per byte (LDK_X_PACKED2)

constexpr int kPrepV = 128, kPrepK = 128;

// One block: 128 K positions (haplotypes / individuals) x 128 SNPs.  The rows of the 128 K
// positions are resolved once; the gather reads 128-byte row segments of X (consecutive
// threads, consecutive SNPs) into a SNP-major shared tile, the scatter turns each 4-byte K
// quad of a SNP into its plane bytes with byte-wise compares and writes every plane as
// 128-byte runs along K.  Plane bytes (GENO: 4 planes, haplotypes: 2):
//   haplotypes  h = [x == 1], v = [x in {0, 1}]
//   genotypes   [x == 1], [x == 2], [x in {0, 1, 2}], 0
// Padding (127) and invalid codes give 0 in every plane; invalid codes also raise
// LDK_DEVERR_BAD_INPUT.
//
// Gather: a lane takes four consecutive SNPs and a warp four consecutive K rows; each row's
// four codes come as one 32-bit word (int8 input) or one byte (packed input: four 2-bit
// fields holding code + 1, SNP v in bits 2 (v % 4) of byte v / 4), the 4 x 4 byte block is
// transposed in registers with byte permutes, and each SNP's four K bytes go to the tile in
// one 32-bit store (the SNP order rotated by lane / 8 so that the 32 lanes' stores fall in 32
// banks).  An int8 row segment that does not start on a 4-byte boundary (odd row stride, or
// an unaligned base) is read as the two aligned words around it and joined with a funnel
// shift; the offset is the same for the 32 lanes of a row, so the branch is warp-uniform.
// The second word is read only where it holds SNPs of the quad, and an aligned word holding
// one byte of the matrix lies in that byte's memory page, so no read can fault; its other
// bytes are shifted or masked out.
template <bool GENO, bool PACKED>
__global__ void __launch_bounds__(256) k_prep_planes(PrepArgs a) {
    constexpr int PL = GENO ? 4 : 2;
    constexpr int RS = kPrepK + 4;  // bytes per SNP row: 33 words, so the scatter's word loads
                                    // (one K quad per lane) hit distinct banks
    __shared__ __align__(16) int8_t tile[kPrepV * RS];
    __shared__ int srow[kPrepK];
    const int64_t v0 = (int64_t)blockIdx.x * kPrepV;
    const int k0 = blockIdx.y * kPrepK;
    constexpr int xmax = GENO ? 2 : 1;
    for (int kk = threadIdx.x; kk < kPrepK; kk += blockDim.x) {
        const int k = k0 + kk;
        int p = 0;
        while (p + 1 < a.P && k >= a.kofs[p + 1]) ++p;
        const int local = k - a.kofs[p];
        const int np = a.pop_off[p + 1] - a.pop_off[p];
        srow[kk] = (local >= 0 && local < np && k < a.kofs[a.P]) ? a.pop_rows[a.pop_off[p] + local] : -1;
    }
    __syncthreads();
    // gather: tile[v][k] = X[row(k), v0 + v]; 127 marks padding
    constexpr int kThreads = 256;
    bool bad = false;
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        static_assert(kPrepV == 4 * 32 && kPrepK % (4 * (kThreads / 32)) == 0, "wide gather geometry");
        const int64_t v = v0 + 4 * lane;
        const int64_t left = a.n_var - v;
        const int nv = left >= 4 ? 4 : (left > 0 ? (int)left : 0);  // SNPs of this quad in the matrix
        // bytes of the quad outside the matrix read as padding (127)
        const uint32_t keep = nv >= 4 ? 0xFFFFFFFFu : ((1u << (8 * nv)) - 1u);
        const int8_t* base = a.X + (PACKED ? (v >> 2) : v);
        const int rot = lane >> 3;
        for (int kk = 4 * warp; kk < kPrepK; kk += 4 * (kThreads / 32)) {
            uint32_t w[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int row = srow[kk + m];
                uint32_t x = 0x7F7F7F7Fu;
                if (row >= 0 && nv > 0) {
                    if constexpr (PACKED) {
                        const uint32_t b = (uint8_t)__ldg(base + (int64_t)row * a.ld);
                        // field j = code + 1 -> byte j = code (two's complement), or 0xFF for missing
                        x = 0u;
#pragma unroll
                        for (int j = 0; j < 4; ++j) x |= (((b >> (2 * j)) & 3u) - 1u & 0xFFu) << (8 * j);
                    } else {
                        const uintptr_t ad = reinterpret_cast<uintptr_t>(base + (int64_t)row * a.ld);
                        const uint32_t* q = reinterpret_cast<const uint32_t*>(ad & ~uintptr_t(3));
                        const int s = (int)(ad & 3u);
                        x = __ldg(q);
                        if (s != 0) {
                            const uint32_t hi = s + nv > 4 ? __ldg(q + 1) : 0u;
                            x = __funnelshift_r(x, hi, 8 * s);
                        }
                    }
                    x = (x & keep) | (0x7F7F7F7Fu & ~keep);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (j < nv) {
                            const int8_t c = (int8_t)(x >> (8 * j));
                            bad |= (c < -1 || c > xmax);
                        }
                    }
                }
                w[m] = x;
            }
            // 4 x 4 byte transpose: t[j] holds SNP j's codes of rows kk .. kk + 3
            const uint32_t x0 = __byte_perm(w[0], w[1], 0x5140), x1 = __byte_perm(w[0], w[1], 0x7362);
            const uint32_t x2 = __byte_perm(w[2], w[3], 0x5140), x3 = __byte_perm(w[2], w[3], 0x7362);
            const uint32_t t[4] = {__byte_perm(x0, x2, 0x5410), __byte_perm(x0, x2, 0x7632),
                                   __byte_perm(x1, x3, 0x5410), __byte_perm(x1, x3, 0x7632)};
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                const int j = (jj + rot) & 3;
                *reinterpret_cast<uint32_t*>(tile + (4 * lane + j) * RS + kk) = t[j];
            }
        }
    }
    if (bad) atomicOr(a.status, LDK_DEVERR_BAD_INPUT);
    __syncthreads();
    // scatter: lane = K quad, warps stride over the SNPs
    const int kq = threadIdx.x % 32;
    constexpr uint32_t kOne = 0x01010101u;
    for (int vv = threadIdx.x / 32; vv < kPrepV; vv += kThreads / 32) {
        const int64_t v = v0 + vv;
        if (v >= a.n_var) break;
        const uint32_t w = *reinterpret_cast<const uint32_t*>(tile + vv * RS + 4 * kq);
        const uint32_t eq0 = __vcmpeq4(w, 0u), eq1 = __vcmpeq4(w, kOne);
        uint8_t* dst = a.planes_out + v * PL * (int64_t)a.ktot + k0 + 4 * kq;
        if constexpr (GENO) {
            const uint32_t eq2 = __vcmpeq4(w, 2u * kOne);
            *reinterpret_cast<uint32_t*>(dst) = eq1 & kOne;
            *reinterpret_cast<uint32_t*>(dst + a.ktot) = eq2 & kOne;
            *reinterpret_cast<uint32_t*>(dst + 2 * (int64_t)a.ktot) = (eq0 | eq1 | eq2) & kOne;
            *reinterpret_cast<uint32_t*>(dst + 3 * (int64_t)a.ktot) = 0u;
        } else {
            *reinterpret_cast<uint32_t*>(dst) = eq1 & kOne;
            *reinterpret_cast<uint32_t*>(dst + a.ktot) = (eq0 | eq1) & kOne;
        }
    }
}

// ---------------------------------------------------------------------------
// peak probes: the two rates the fused parse's roofline is stated against
// ---------------------------------------------------------------------------

// Back-to-back kind::i8 MMAs (M = 128, N = 256, K = 32) from zero-filled shared-memory
// tiles into one TMEM accumulator, issued by one thread per CTA.
constexpr int kProbeN = 256;
__device__ unsigned g_probe_status;  // LDK_DEVERR_* of the probes
__device__ double g_probe_sink;      // keeps the FP64 chains live

__global__ void __launch_bounds__(128, 1) k_probe_i8(int iters) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    constexpr int A_BYTES = 128 * kKChunk, B_BYTES = kProbeN * kKChunk;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ volatile int abort_s;
    for (int idx = threadIdx.x; idx < (A_BYTES + B_BYTES) / 16; idx += blockDim.x)
        reinterpret_cast<uint4*>(base)[idx] = make_uint4(0u, 0u, 0u, 0u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 32) {
        tmem_alloc(&tmem_base_s, kProbeN);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    if (threadIdx.x == 0) {
        constexpr uint32_t idesc = idesc_u8<kProbeN>();
        const uint32_t a_addr = su32(base), b_addr = a_addr + A_BYTES;
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int ks = 0; ks < kKChunk / 32; ++ks)
                mma_u8(tmem, sw128_desc(a_addr + ks * 32), sw128_desc(b_addr + ks * 32), idesc, (it | ks) ? 1u : 0u);
        mma_commit(&bar);
        mbar_wait(&bar, 0u, &abort_s, &g_probe_status);
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc_fence_after();
        tmem_dealloc(tmem, kProbeN);
    }
}

// Eight independent FP64 FMA chains per thread.
__global__ void __launch_bounds__(512) k_probe_fp64(int iters, double b, double c) {
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = fma(x[k], b, c);
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += x[k];
    if (t == 1234.5678) g_probe_sink = t;  // never true for these inputs
}


}  // namespace

int tc_rows_per_block(const ParseShape& sh) { return sh.genotypes ? Cfg<1, true>::ROWS : Cfg<1, false>::ROWS; }
int tc_block_slots(const ParseShape& sh) { return sh.genotypes ? Cfg<1, true>::SLOTS : Cfg<1, false>::SLOTS; }
int tc_tile_width(const ParseShape& sh, int variant) { return tile_nj(sh.P, sh.genotypes != 0, variant); }
int tc_planes(const ParseShape& sh) { return sh.genotypes ? Cfg<1, true>::PLANES : Cfg<1, false>::PLANES; }

size_t tc_smem_bytes(const ParseShape& sh) {
    return sh.genotypes ? tc_smem_bytes_g<true>(sh) : tc_smem_bytes_g<false>(sh);
}

template <bool GENO, int V>
bool private_staging_of(const ParseShape& sh) {
    const int t = smem_table(sh);
    switch (sh.P) {
        case 1: return private_staging<1, GENO, V>(sh.n_bins, t);
        case 2: return private_staging<2, GENO, V>(sh.n_bins, t);
        case 3: return private_staging<3, GENO, V>(sh.n_bins, t);
        default: return private_staging<4, GENO, V>(sh.n_bins, t);
    }
}

bool tc_private_staging(const ParseShape& sh, int variant) {
    if (sh.genotypes) return (variant == 1 && sh.P <= 2) ? private_staging_of<true, 1>(sh) : private_staging_of<true, 0>(sh);
    return variant == 1 ? private_staging_of<false, 1>(sh) : private_staging_of<false, 0>(sh);
}

bool tc_rtab_global(const ParseShape& sh) {
    switch (sh.P) {
        case 1: return rtab_global_t<1>(sh);
        case 2: return rtab_global_t<2>(sh);
        case 3: return rtab_global_t<3>(sh);
        default: return rtab_global_t<4>(sh);
    }
}

namespace {
__global__ void k_fill_rtab(double4* t, int max_n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= max_n) t[i] = recip_entry(i);
}
}  // namespace

namespace {
__global__ void k_fill_gtab(GenoRecip* t, int max_n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= max_n) t[i] = geno_recip_entry(i);
}
}  // namespace

cudaError_t launch_fill_gtab(void* gtab, int max_n, cudaStream_t s) {
    k_fill_gtab<<<(max_n + 256) / 256, 256, 0, s>>>(static_cast<GenoRecip*>(gtab), max_n);
    return cudaGetLastError();
}

cudaError_t launch_fill_rtab(void* rtab, int max_n, cudaStream_t s) {
    k_fill_rtab<<<(max_n + 256) / 256, 256, 0, s>>>(static_cast<double4*>(rtab), max_n);
    return cudaGetLastError();
}

cudaError_t launch_prep_planes(const ldk_parse_t* d, const Scratch& w, const ParseShape& sh, cudaStream_t s) {
    if (d->n_var == 0) return cudaSuccess;
    PrepArgs a;
    a.X = d->X;
    a.ld = d->ld_x;
    a.n_var = d->n_var;
    a.pop_rows = d->pop_rows;
    for (int p = 0; p <= LDK_MAX_POPS; ++p) {
        a.pop_off[p] = d->pop_offsets[p];
        a.kofs[p] = sh.kofs[p];
    }
    a.P = sh.P;
    a.ktot = sh.ktot;
    a.genotypes = sh.genotypes;
    a.planes = sh.planes;
    a.planes_out = w.hv;
    a.status = w.status;
    dim3 grid((unsigned)((d->n_var + kPrepV - 1) / kPrepV), (unsigned)(sh.ktot / kPrepK));
    const bool packed = d->x_format == LDK_X_PACKED2;
    if (sh.genotypes) {
        if (packed) k_prep_planes<true, true><<<grid, 256, 0, s>>>(a);
        else k_prep_planes<true, false><<<grid, 256, 0, s>>>(a);
    } else {
        if (packed) k_prep_planes<false, true><<<grid, 256, 0, s>>>(a);
        else k_prep_planes<false, false><<<grid, 256, 0, s>>>(a);
    }
    return cudaGetLastError();
}

namespace {
// Work items of the persistent parse kernel.  A row block alone is too coarse a unit where
// there are few row blocks per SM (a 5,000-SNP window has 79) or where their count leaves a
// partial last wave; pieces of at most c partner tiles bound the spread of the CTAs' finishing
// times by one piece.  c = max(min_tiles, ceil(total tiles / kItemTarget)), so shapes with
// many small row blocks keep one item per row block, and no piece is so short that the flush
// of its staged sums (which ends every item) outweighs its tiles.  Pieces of one row block are consecutive
// (the claim order of the row blocks stays), its last piece runs to INT32_MAX, and a row block
// without partners gets no item.  One block of 1024 threads: the total, then a block-wide
// scan of the pieces per row block, 1024 row blocks per round.
constexpr int kSplitThreads = 1024;

__device__ __forceinline__ int rb_tiles(const int32_t* __restrict__ rb, const int32_t* __restrict__ jmax, int k,
                                        int nj) {
    const int r0 = rb[2 * k], r1 = rb[2 * k + 1];
    const int jend = jmax[r1 - 1];
    return jend > r0 + 1 ? (jend - r0 + nj - 1) / nj : 0;
}

__global__ void __launch_bounds__(kSplitThreads) k_split_items(const int32_t* __restrict__ rb, int n_rb,
                                                               const int32_t* __restrict__ jmax, int nj,
                                                               int min_tiles, int4* __restrict__ items,
                                                               int* __restrict__ n_items) {
    __shared__ long long s_sum[kSplitThreads / 32];
    __shared__ int s_scan[kSplitThreads / 32];
    __shared__ int s_base;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int NW = kSplitThreads / 32;
    long long t = 0;
    for (int k = tid; k < n_rb; k += kSplitThreads) t += rb_tiles(rb, jmax, k, nj);
#pragma unroll
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) s_sum[wid] = t;
    if (tid == 0) s_base = 0;
    __syncthreads();
    long long total = 0;
#pragma unroll 4
    for (int x = 0; x < NW; ++x) total += s_sum[x];
    const long long cl = (total + kItemTarget - 1) / kItemTarget;
    const int c = cl > min_tiles ? (int)cl : min_tiles;
    for (int b0 = 0; b0 < n_rb; b0 += kSplitThreads) {
        const int k = b0 + tid;
        const int nt = k < n_rb ? rb_tiles(rb, jmax, k, nj) : 0;
        const int parts = (nt + c - 1) / c;
        int x = parts;  // inclusive scan within the warp, then over the warps
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_scan[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int v = s_scan[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += y;
            }
            s_scan[lane] = v;
        }
        __syncthreads();
        const int first = s_base + (wid ? s_scan[wid - 1] : 0) + x - parts;
        if (parts) {
            const int r0 = rb[2 * k], r1 = rb[2 * k + 1];
            for (int q = 0; q < parts; ++q)
                items[first + q] = make_int4(r0, r1, q * c, q == parts - 1 ? INT32_MAX : (q + 1) * c);
        }
        const int round_total = s_scan[NW - 1];
        __syncthreads();
        if (tid == 0) s_base += round_total;
        __syncthreads();
    }
    if (tid == 0) *n_items = s_base;
}
}  // namespace

int tc_min_item_tiles(const ParseShape& sh) {
    const int staged = tc_block_slots(sh) * sh.n_bins * (sh.n_stats + 1);
    const int t = (staged + kFlushValuesPerTile - 1) / kFlushValuesPerTile;
    return t > kMinItemTiles ? t : kMinItemTiles;
}

cudaError_t launch_split_items(const Scratch& w, int n_row_blocks, int nj, int min_tiles, cudaStream_t s) {
    k_split_items<<<1, kSplitThreads, 0, s>>>(w.row_blocks, n_row_blocks, w.jmax, nj, min_tiles,
                                              reinterpret_cast<int4*>(w.items), w.n_items);
    return cudaGetLastError();
}

cudaError_t launch_parse_tc(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w,
                            const ParseShape& sh, int max_items, int variant, cudaStream_t s) {
    if (sh.genotypes) return launch_tc_geno(d, o, w, sh, max_items, variant, s);
    return variant == 1 ? launch_tc_hap_v1(d, o, w, sh, max_items, s) : launch_tc_hap_v0(d, o, w, sh, max_items, s);
}


// Peak probes, each timed with CUDA events on `s` after one untimed warm-up launch.
// *status receives the probes' device status word.
cudaError_t probe_peaks(double* int8_ops_per_s, double* fp64_fma_per_s, unsigned* status, cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = 1024 + 128 * kKChunk + kProbeN * kKChunk;
    cudaError_t e = cudaFuncSetAttribute(k_probe_i8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned zero = 0u;
    if ((e = cudaMemcpyToSymbolAsync(g_probe_status, &zero, sizeof(unsigned), 0, cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
        return e;
    cudaEvent_t e0, e1;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&e1)) != cudaSuccess) { cudaEventDestroy(e0); return e; }
    float ms = 0.f;
    const int i8_iters = 20000, f64_iters = 2000;
    k_probe_i8<<<sms, 128, smem, s>>>(64);
    cudaEventRecord(e0, s);
    k_probe_i8<<<sms, 128, smem, s>>>(i8_iters);
    cudaEventRecord(e1, s);
    if ((e = cudaEventSynchronize(e1)) == cudaSuccess && (e = cudaEventElapsedTime(&ms, e0, e1)) == cudaSuccess)
        *int8_ops_per_s = 2.0 * 128 * kProbeN * kKChunk * (double)i8_iters * sms / (ms * 1e-3);
    if (e == cudaSuccess) {
        k_probe_fp64<<<sms, 512, 0, s>>>(16, 0.999999, 1e-9);
        cudaEventRecord(e0, s);
        k_probe_fp64<<<sms, 512, 0, s>>>(f64_iters, 0.999999, 1e-9);
        cudaEventRecord(e1, s);
        if ((e = cudaEventSynchronize(e1)) == cudaSuccess && (e = cudaEventElapsedTime(&ms, e0, e1)) == cudaSuccess)
            *fp64_fma_per_s = 64.0 * 512 * (double)f64_iters * sms / (ms * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyFromSymbolAsync(status, g_probe_status, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

}  // namespace ldk
