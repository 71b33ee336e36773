/*
 * libldk -- B200 (sm_100a) two-locus LD parse: SNP pairs within a distance cutoff ->
 * per-population two-locus counts -> unbiased DD / Dz / pi2 and r^2 estimators ->
 * distance-bin sums.  C ABI: plain pointers and sizes, no exceptions, no allocation.
 *
 * All array arguments are DEVICE pointers unless marked "host".  Every entry point
 * returns LDK_OK (0) or a negative status; ldk_last_error() gives the message of the
 * calling host thread's last failure.  Work is enqueued on `stream` (a cudaStream_t,
 * NULL = legacy default stream).  Entry points that report device-side status read a
 * 4-byte status word back (a stream synchronisation) before returning.
 *
 * References are to pg_gpu (the drop-in target): file:line within that project.
 */
#ifndef LDK_H
#define LDK_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LDK_API __attribute__((visibility("default")))
#else
#define LDK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define LDK_OK 0
#define LDK_ERR_ARG (-1)         /* invalid argument (null pointer, bad size, unsorted) */
#define LDK_ERR_CUDA (-2)        /* CUDA runtime error */
#define LDK_ERR_ARCH (-3)        /* device is not sm_100 (B200/GB200) */
#define LDK_ERR_WORKSPACE (-4)   /* caller workspace smaller than ldk_*_workspace_size */
#define LDK_ERR_DEVICE (-5)      /* device status word set (timeout, block range, bad code) */
#define LDK_ERR_UNSUPPORTED (-6) /* configuration outside the kernels' limits */

#define LDK_MAX_POPS 4
#define LDK_MAX_BINS 64

/* counting / estimator method of ldk_parse */
#define LDK_METHOD_PLAIN_FP64 0 /* per-pair byte counting + FP64 estimators (the drop-in) */
#define LDK_METHOD_TC 1         /* INT8 tcgen05 Gram counts; exact-integer features, FP64 combination and bins */

LDK_API int ldk_version(void);
LDK_API const char* ldk_last_error(void);

/* Per-pair haplotype counts [n11, n10, n01, n00] and valid-pair counts over the rows
 * `rows[0..n_rows)` of X (n_total_rows x ld_x int8 in {0, 1, -1}).
 * Replaces ld_pipeline.compute_counts_for_pairs (ld_pipeline.py:130-175). */
LDK_API int ldk_counts_hap(const int8_t* X, int64_t ld_x, int64_t n_var, const int32_t* rows,
                   int32_t n_rows, const int32_t* idx_i, const int32_t* idx_j, int64_t n_pairs,
                   int32_t* counts, int32_t* n_valid, void* stream);

/* Per-pair nine-cell genotype counts (column g_i*3 + g_j) and valid counts, X in
 * {0, 1, 2, -1}.  Replaces ld_pipeline.compute_genotype_counts_for_pairs and its
 * _GENO_COUNTS_KERN (ld_pipeline.py:183-263). */
LDK_API int ldk_counts_geno(const int8_t* X, int64_t ld_x, int64_t n_var, const int32_t* rows,
                    int32_t n_rows, const int32_t* idx_i, const int32_t* idx_j, int64_t n_pairs,
                    int32_t* counts, int32_t* n_valid, void* stream);

/* Moments-ordered statistics (n_pairs x n_stats, float64) of P populations from
 * per-population counts: counts (P, n_pairs, 4) [haplotype] or (P, n_pairs, 9)
 * [genotype] int32, n_valid (P, n_pairs) int32 or NULL.
 * Replaces compute_multi_pop_statistics_batch_hap (haplotype_kernels.py:584-640),
 * compute_multi_pop_statistics_batch_geno (genotype_kernels.py:881-936) and
 * compute_two_pop_statistics_batch (ld_pipeline.py:271-322). */
LDK_API int ldk_stats(int genotypes, int P, const int32_t* counts, const int32_t* n_valid,
              int64_t n_pairs, double* out, void* stream);

/* One raw haplotype estimator call on float64 counts (n_pairs, 4*P_total) with
 * n_valid (n_pairs, P_total) or NULL.  case_id and args are the canonical case of
 * the call (see pg_gpu_b200/csrc/gen_estimators.py: RAW_CASES); out is n_pairs.
 * Replaces the per-case kernels behind ld_statistics.dd / dz / pi2
 * (ld_statistics.py:13-129, haplotype_kernels.py:69-304). */
LDK_API int ldk_raw_hap(int case_id, const int32_t* args_host, int P_total, const double* counts,
                const double* n_valid, int64_t n_pairs, double* out, void* stream);

/* r (which=0), r^2 (1) or D' (2) per pair from float64 counts (n_pairs, 4) and n_valid
 * or NULL.  Replaces ld_statistics.r / r_squared / d_prime (ld_statistics.py:153-246,
 * haplotype_kernels.py:20-62). */
LDK_API int ldk_r_family(int which, const double* counts, const double* n_valid, int64_t n_pairs,
                 double* out, void* stream);

/* The binned parse: every pair i < j of one window with pos[j] - pos[i] <= max_dist,
 * binned by |coord[j] - coord[i]| into right-open bins, summed per bootstrap block of
 * its left SNP.  Replaces the loop body of moments_ld._compute_ld_sums
 * (moments_ld.py:309-341) and of HaplotypeMatrix.compute_ld_statistics_gpu_single_pop /
 * _two_pops (haplotype_matrix.py:1657-1689, 1789-1837). */
typedef struct {
    const int8_t* X;            /* (n_rows, ld_x) int8: haplotypes {0,1,-1} or genotypes {0,1,2,-1} */
    int64_t ld_x;               /* row stride of X in elements (>= n_var) */
    int64_t n_rows;
    int64_t n_var;
    int32_t genotypes;          /* 0: haplotype path (4 counts), 1: genotype path (9 counts) */
    int32_t n_pops;             /* P in 1..4 */
    const int32_t* pop_rows;    /* concatenated row indices of the P populations */
    int32_t pop_offsets[LDK_MAX_POPS + 1]; /* host: population p = pop_rows[off[p]..off[p+1]) */
    const double* pos;          /* (n_var) positions, non-decreasing within each window */
    const double* coord;        /* (n_var) binning coordinate (e.g. Morgans) or NULL = pos */
    double max_dist;            /* pair cutoff on pos */
    int32_t n_bins;             /* 1..64 */
    double edges[LDK_MAX_BINS + 1]; /* host: increasing bin edges */
    const int64_t* window_offsets; /* host (n_windows + 1) SNP ranges, or NULL = one window */
    int32_t n_windows;
    const int32_t* snp_block;   /* (n_var) bootstrap block of each SNP, or NULL = all 0 */
    int32_t n_blocks;           /* >= 1 */
    int32_t method;             /* LDK_METHOD_* */
    const int64_t* anchor_end;  /* host (n_windows) or NULL: only SNPs i < anchor_end[w] of window w
                                   are a pair's left SNP; partners still run to the window's end.
                                   A rank of a split parse passes its SNP slab -- its anchors and
                                   the read-only right halo of max_dist after them -- as a window
                                   with anchor_end at the end of its anchors. */
    int32_t x_format;           /* LDK_X_INT8 (0) or LDK_X_PACKED2 (1); see below */
} ldk_parse_t;
/* Layouts of ldk_parse_t.X:
 *  LDK_X_INT8     one int8 code per entry, row stride ld_x >= n_var (pg_gpu's matrix layout,
 *                 haplotype_matrix.py:34-83, genotype_matrix.py:32-71);
 *  LDK_X_PACKED2  two bits per entry holding code + 1 (0: missing, 1..3: codes 0..2), four
 *                 consecutive SNPs of a row per byte, SNP v in bits 2 (v % 4) .. 2 (v % 4) + 1
 *                 of byte v / 4; ld_x is the row stride in bytes (>= ceil(n_var / 4)).  A
 *                 quarter of the bytes to move from the host; read by the tensor-core method
 *                 (the plain method returns LDK_ERR_UNSUPPORTED). */
#define LDK_X_INT8 0
#define LDK_X_PACKED2 1
/* Limits of the tensor-core method (LDK_METHOD_TC), none of which bind
 * LDK_METHOD_PLAIN_FP64:
 *  - each row block -- 64 SNPs (genotypes: 128) counted from each window's first SNP --
 *    may cover at most 2 (genotypes: 4) consecutive bootstrap blocks from its first SNP's
 *    block; otherwise the parse stops with LDK_ERR_DEVICE and status LDK_DEVERR_BLOCK_SPAN;
 *  - the per-bin sums of the row block's bootstrap blocks must fit in shared memory beside
 *    the pipeline, else LDK_ERR_UNSUPPORTED (four genotype populations with more than 36
 *    bins, three with more than 47). */

typedef struct {
    double* sums;        /* (n_blocks, n_bins, n_stats) statistic sums */
    double* r2_sums;     /* (n_blocks, n_bins) sum of finite r^2 of population 0 (dosage r^2 on the genotype path) */
    uint64_t* pairs;     /* (n_blocks, n_bins) pairs binned */
    uint64_t* r2_counts; /* (n_blocks, n_bins) pairs with finite r^2 */
} ldk_parse_out_t;

LDK_API int ldk_n_stats(int P);   /* 3, 15, 45, 105 */
LDK_API size_t ldk_parse_workspace_size(const ldk_parse_t* d);
LDK_API int ldk_parse(const ldk_parse_t* d, const ldk_parse_out_t* out, void* workspace,
              size_t workspace_bytes, void* stream);

/* ldk_parse without a workspace, for callers that cannot allocate device memory: a host
 * runtime reaching this library through a JNI / cgo / N-API layer that owns no device
 * allocator and only hands over its input and output buffers, or a host application whose
 * memory manager forbids allocations outside its own pool.  Scratch comes from a
 * file-scope device array of LDK_NOALLOC_SCRATCH_BYTES held by every GPU that loads the
 * library until exit; a parse needing more returns LDK_ERR_UNSUPPORTED.  The first call
 * on a device (and the first after that device's context was re-created) resolves the
 * array's device address.  All calls share the array, so calls that overlap on the GPU
 * race.  No counterpart in pg_gpu. */
#define LDK_NOALLOC_SCRATCH_BYTES (64ull << 20)
LDK_API int ldk_parse_noalloc(const ldk_parse_t* d, const ldk_parse_out_t* out, void* stream);

/* The parse split for CUDA-graph capture and repeated launches over one plan.  No
 * counterpart in pg_gpu (its parse is a Python loop of CuPy calls).
 *
 * ldk_parse_setup writes the call's plan into the workspace -- window offsets and the
 * tensor-core method's row-block list, from host memory -- and synchronises `stream`.
 * ldk_parse_enqueue then enqueues only device work on `stream` (zeroing the outputs and
 * the status word, pair ranges, indicator planes, the parse kernel): no host <-> device
 * copies, no synchronisation, no allocation, so it can be captured into a CUDA graph and
 * the graph replayed while the input arrays change contents in place.  It requires a
 * preceding ldk_parse_setup with the same descriptor shape (n_var, populations, windows,
 * method) and workspace.  ldk_parse_status synchronises `stream` and returns LDK_OK or
 * LDK_ERR_DEVICE (with ldk_last_error) from the device status word the last enqueued
 * parse on this workspace left.  ldk_parse = setup + enqueue + status. */
LDK_API int ldk_parse_setup(const ldk_parse_t* d, void* workspace, size_t workspace_bytes, void* stream);
LDK_API int ldk_parse_enqueue(const ldk_parse_t* d, const ldk_parse_out_t* out, void* workspace,
                              size_t workspace_bytes, void* stream);
LDK_API int ldk_parse_status(const void* workspace, void* stream);

/* All-pairs LD of one SNP set: for the n_sel selected rows of X and every pair of its
 * n_var SNPs, one of -- for haplotypes (X int8 in {-1, 0, 1}):
 *   LDK_LDM_R2        pg_gpu's pairwise r^2 (HaplotypeMatrix.pairwise_r2('r2'),
 *                     haplotype_matrix.py:1092-1175): D = p_AB - p_i p_j with p_AB over the
 *                     jointly valid haplotypes and p_i over the site's valid ones,
 *                     r^2 = D^2 / (p_i q_i p_j q_j), 0 where that product is 0; diagonal 0;
 *   LDK_LDM_SIGMA_D2  the unbiased sigma_D^2 = D^2 / pi2 of _tile_sigma_d2
 *                     (ld_statistics.py:311-344): 0 where n < 4 or the pi2 numerator is 0;
 *                     diagonal 0;
 *   LDK_LDM_R2_COUNTS r^2 from the jointly valid counts (ld_statistics.r_squared,
 *                     haplotype_kernels.py:32-42): NaN where pA qA pB qB = 0; diagonal NaN.
 * For genotypes (X int8 in {-1, 0, 1, 2}, rows = individuals):
 *   LDK_LDM_DIPLOID_R2    pg_gpu's dosage r^2 (ld_statistics._r2_matrix_diploid,
 *                         ld_statistics.py:973-1021): dosages centred on the site's valid
 *                         mean and zeroed where missing, r^2 = cov^2 / (var_i var_j), 0 where
 *                         that product is 0; diagonal 0;
 *   LDK_LDM_ROGERS_HUFF_R signed Rogers-Huff r (ld_statistics.py:392-524), complete data
 *                         only: NaN where a site is constant; diagonal NaN;
 *   LDK_LDM_SIGMA_D2_GENO the unbiased sigma_D^2 of genotype pairs (genotype_kernels.py:91-170),
 *                         complete data only: NaN where n < 4 or the pi2 numerator <= 0;
 *                         diagonal NaN.  A missing call with the last two sets the device
 *                         status (LDK_ERR_DEVICE).
 * out (device, may be NULL): n_var rows of ld_out doubles, the full symmetric matrix.
 * sums (device double[2], may be NULL): the sum of the values over pairs i < j that enter
 * ZnS's mean and their count -- every pair for LDK_LDM_R2, pairs with n >= 4 for
 * LDK_LDM_SIGMA_D2 (ld_statistics.py:534-596), finite values for LDK_LDM_R2_COUNTS; every
 * pair for LDK_LDM_DIPLOID_R2; for the other two the sum of r^2 (resp. sigma_D^2) over
 * finite values and their count.
 * Counts come from the tensor-core Gram pipeline; values in FP64.  Synchronises `stream`. */
#define LDK_LDM_R2 0
#define LDK_LDM_SIGMA_D2 1
#define LDK_LDM_R2_COUNTS 2
#define LDK_LDM_DIPLOID_R2 3
#define LDK_LDM_ROGERS_HUFF_R 4
#define LDK_LDM_SIGMA_D2_GENO 5
LDK_API size_t ldk_ld_matrix_workspace_size(int64_t n_var, int32_t n_sel);
LDK_API int ldk_ld_matrix(const int8_t* X, int64_t ld_x, int64_t n_var, const int32_t* rows, int32_t n_sel,
                          int estimator, double* out, int64_t ld_out, double* sums, void* workspace,
                          size_t workspace_bytes, void* stream);

/* Autotuning of the tensor-core parse.  Replaces the memory-driven pair-chunk sizing of
 * ld_pipeline.estimate_ld_chunk_size (ld_pipeline.py:16-49): the work here is a fixed tile
 * schedule, and the tuner picks among its variants.  With enable = 1 (or LDK_AUTOTUNE=1 in
 * the environment at the first call), the first ldk_parse of each shape class runs every
 * candidate -- partner-tile width (two widths per population count and path) x row-block
 * claim order (largest windows first, or window order; several windows only) -- twice on
 * its own input, times the second run of each with CUDA events, and keeps the fastest in a
 * process-wide table behind a mutex; that call then clears its outputs and runs the kept
 * candidate.  A shape class is (population count, haplotype or genotype path, padded sample
 * bytes, bin count, decade of max_dist, log2 of the mean window size).  Later ldk_parse,
 * ldk_parse_setup (the order) and ldk_parse_enqueue (the width) calls of the class use the
 * kept choice, tuning enabled or not; classes never tuned use the defaults (the widest
 * haplotype tile, 12 / 8 partners for one / two genotype populations; largest windows first).  ldk_tile_width returns the width (SNPs per partner tile) a call
 * with this descriptor would use now, 0 for the plain method, or a negative status.  No
 * counterpart in pg_gpu. */
LDK_API int ldk_autotune(int enable);
LDK_API int ldk_tile_width(const ldk_parse_t* d);

/* The tuning table as a JSON file ({"format": "ldk-autotune", "version": 1, "entries":
 * [...]}, one entry per shape class with its choice and time).  ldk_autotune_load merges a
 * file into the table (returns the entries read, or LDK_ERR_ARG if the file is not such a
 * table); ldk_autotune_save writes the whole table (returns the entries written).  With
 * LDK_AUTOTUNE_CACHE=<path> in the environment the file is loaded at the first lookup and
 * rewritten after every tuning, so a later process starts from it without re-tuning.
 * ldk_autotune_count returns the table's size and, in *tunings (may be NULL), how many
 * tunings this process ran; ldk_autotune_clear empties the table.  Host-only. */
LDK_API int ldk_autotune_load(const char* path);
LDK_API int ldk_autotune_save(const char* path);
LDK_API int ldk_autotune_count(int* tunings);
LDK_API int ldk_autotune_clear(void);

/* Whether two parses with this descriptor give the same output bits whatever order the GPU
 * runs their work in: 1, or 0 where the bin sums agree only to FP64 rounding; a negative
 * status for an invalid descriptor.  Every kernel adds its partial sums (tensor-core kernel:
 * per work item, a run of one row block's partner tiles cut from the input's pair ranges;
 * plain kernel: per row chunk) as fixed-point integers (an order-independent sum); the
 * partials themselves are a fixed function of the input when each epilogue warp of the
 * tensor-core kernel stages its
 * sums in its own shared-memory copy, and the plain kernel always.  Shapes whose staging
 * does not fit once per warp (four populations; three genotype populations with more than
 * five bins, three haplotype populations with more than about twenty) share one copy
 * updated with shared-memory atomics, whose order varies.  Depends on the tile width in
 * use (after tuning, the tuned one).  Host-only; no counterpart in pg_gpu (its cp.add.at
 * bin sums, moments_ld.py:335-339, are order-dependent). */
LDK_API int ldk_parse_reproducible(const ldk_parse_t* d);

/* Row blocks of the tensor-core methods (genotypes 0: haplotype path, 1: genotype path):
 * *rows SNPs per row block, counted from each window's first SNP, and *max_blocks, the
 * bootstrap blocks one row block may cover from its first SNP's block (more stops the
 * parse with LDK_DEVERR_BLOCK_SPAN).  Host-only; no counterpart in pg_gpu. */
LDK_API int ldk_tc_row_blocks(int genotypes, int32_t* rows, int32_t* max_blocks);

/* Per-thread kernel timing: while enabled, ldk_parse brackets its main counting /
 * estimator kernel with CUDA events on the caller's stream; ldk_profile_last_kernel_ms
 * returns that kernel's duration in the calling thread's last ldk_parse (-1 if none).
 * No counterpart in pg_gpu (measurement support). */
LDK_API int ldk_profile(int enable);
LDK_API double ldk_profile_last_kernel_ms(void);

/* Measured peaks of the calling device, the denominators of the tensor-core parse's
 * roofline: *int8_ops_per_s from back-to-back tcgen05 kind::i8 MMAs (128 x 256 x 32,
 * one CTA per SM, operands in shared memory; ops = 2 x MACs) and *fp64_fma_per_s from
 * eight independent FP64 FMA chains per thread (16 warps per SM).  About 20 ms of GPU
 * time; synchronises `stream`.  No counterpart in pg_gpu (measurement support). */
LDK_API int ldk_probe_peaks(double* int8_ops_per_s, double* fp64_fma_per_s, void* stream);

/* out[r, k] = sum_b weights[r, b] * block_sums[b, k] (float64); weights int32 (R, n_blocks).
 * Block-bootstrap replicates over pre-binned per-block sums, the semantics of
 * resampling.block_bootstrap (resampling.py:201-256); also per-window totals. */
LDK_API int ldk_block_combine(const double* block_sums, int64_t n_blocks, int64_t k,
                      const int32_t* weights, int64_t n_rep, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LDK_H */
