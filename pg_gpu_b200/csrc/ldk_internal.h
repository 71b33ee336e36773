// Internal host/device interface between the C ABI (ldk_api.cu) and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ldk.h"
#include "ldk_common.cuh"

namespace ldk {

// Per-call device scratch carved out of the caller's workspace.
struct Scratch {
    unsigned* status;      // device status word (LDK_DEVERR_* bits)
    int* row_counter;      // dynamic row-chunk counter of the plain parse
    int* item_counter;     // dynamic row-block counter of the tensor-core parse
    int32_t* jmax;         // (n_var) exclusive end of each SNP's partner range
    int64_t* win_off;      // (n_windows + 1) window SNP offsets
    int64_t* anc_end;      // (n_windows) end of each window's anchor SNPs
    uint8_t* hv;           // TC path: (n_var, planes, Ktot) indicator planes
    int32_t* row_blocks;   // TC path: (n_row_blocks, 2) row blocks [row0, row1) in claim order
    int32_t* items;        // TC path: work items (row0, row1, t0, t1): rows [row0, row1),
                           // partner tiles [t0, t1) of that row block
    int* n_items;          // TC path: items in use
    void* rtab;            // TC haplotype path: (max_n + 1) double4 reciprocal table in the
                           // workspace, or null when it lives in shared memory
    void* gtab;            // TC genotype path: (max_n + 1) GenoRecip reciprocal table
    unsigned long long* fx;  // (n_blocks, n_bins, n_stats + 1, kFxLimbs) fixed-point bin sums
};

struct ParseShape {
    int P;
    int genotypes;
    int n_stats;
    int n_bins;
    int kofs[LDK_MAX_POPS + 1];  // TC path: K offset (bytes) of each population segment
    int ktot;                    // TC path: total K bytes (multiple of 128)
    int planes;                  // TC path: indicator planes per SNP (2 haplotype, 4 genotype)
    int max_n;                   // largest population size
    int rtab_global;             // TC haplotype path: the reciprocal table (32 B per n_valid)
                                 // does not fit beside the pipeline in shared memory
};

// launchers (ldk_plain.cu)
cudaError_t launch_counts(int genotypes, const int8_t* X, int64_t ld, const int32_t* rows, int n_rows,
                          const int32_t* ii, const int32_t* jj, int64_t n, int32_t* counts,
                          int32_t* n_valid, cudaStream_t s);
cudaError_t launch_stats(int genotypes, int P, const int32_t* counts, const int32_t* n_valid, int64_t n,
                         double* out, cudaStream_t s);
cudaError_t launch_raw_hap(int case_id, const int32_t* args, int P_total, const double* counts,
                           const double* n_valid, int64_t n, double* out, cudaStream_t s);
cudaError_t launch_r_family(int which, const double* counts, const double* n_valid, int64_t n,
                            double* out, cudaStream_t s);
cudaError_t launch_jmax(const ldk_parse_t* d, const Scratch& w, cudaStream_t s);
cudaError_t launch_parse_plain(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w,
                               const ParseShape& sh, cudaStream_t s);
// sums / r2_sums from the fixed-point accumulators
cudaError_t launch_fx_finish(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, int n_stats,
                             cudaStream_t s);
cudaError_t launch_block_combine(const double* block_sums, int64_t n_blocks, int64_t k,
                                 const int32_t* weights, int64_t n_rep, double* out, cudaStream_t s);

// launchers (ldk_tc.cu)
cudaError_t launch_prep_planes(const ldk_parse_t* d, const Scratch& w, const ParseShape& sh,
                               cudaStream_t s);
// max_items bounds the work items in w (their count is on the device): at most that many CTAs
cudaError_t launch_parse_tc(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w,
                            const ParseShape& sh, int max_items, int variant, cudaStream_t s);
// the tensor-core kernel per path and tile variant (ldk_tc_hap0.cu, ldk_tc_hap1.cu, ldk_tc_geno.cu)
cudaError_t launch_tc_hap_v0(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, const ParseShape& sh,
                             int max_items, cudaStream_t s);
cudaError_t launch_tc_hap_v1(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, const ParseShape& sh,
                             int max_items, cudaStream_t s);
cudaError_t launch_tc_geno(const ldk_parse_t* d, const ldk_parse_out_t* o, const Scratch& w, const ParseShape& sh,
                           int max_items, int variant, cudaStream_t s);
int tc_tile_width(const ParseShape& sh, int variant);  // partners per tile of a tile variant
int tc_rows_per_block(const ParseShape& sh);
int tc_block_slots(const ParseShape& sh);  // bootstrap blocks one row block may cover
int tc_planes(const ParseShape& sh);
cudaError_t probe_peaks(double* int8_ops_per_s, double* fp64_fma_per_s, unsigned* status, cudaStream_t s);
size_t tc_smem_bytes(const ParseShape& sh);
bool tc_rtab_global(const ParseShape& sh);  // where the reciprocal table must live
bool tc_private_staging(const ParseShape& sh, int variant);  // one staging copy per epilogue warp
cudaError_t launch_fill_rtab(void* rtab, int max_n, cudaStream_t s);
cudaError_t launch_fill_gtab(void* gtab, int max_n, cudaStream_t s);

cudaError_t launch_build_items(const Scratch& w, int n_windows, int rows, cudaStream_t s);
// Work items of the tensor-core parse: each row block of w.row_blocks split into pieces of
// at most c partner tiles of width nj, c = max(min_tiles, ceil(total tiles / kItemTarget)),
// from the pair ranges in w.jmax; the count goes to *w.n_items.  At most
// n_row_blocks + kItemTarget items.  min_tiles = tc_min_item_tiles(shape): every item ends
// with a flush of the epilogue's staged sums (block slots x bins x (statistics + 1) values),
// so an item is kept at least one tile per kFlushValuesPerTile staged values long.
constexpr int kItemTarget = 2048;
constexpr int kMinItemTiles = 4;
constexpr int kFlushValuesPerTile = 64;
inline int tc_item_capacity(int n_row_blocks) { return n_row_blocks + kItemTarget; }
int tc_min_item_tiles(const ParseShape& sh);
cudaError_t launch_split_items(const Scratch& w, int n_row_blocks, int nj, int min_tiles, cudaStream_t s);

// all-pairs LD of one SNP set (ldk_ldm.cu)
size_t ld_matrix_workspace(int64_t n_var, int32_t n_sel);
cudaError_t launch_ld_matrix(const int8_t* X, int64_t ld_x, int64_t n_var, const int32_t* rows, int32_t n_sel,
                             int estimator, double* out, int64_t ld_out, double* sums, unsigned char* ws,
                             unsigned* status, cudaStream_t s);

// autotuning table (ldk_tune.cu): shape class -> (tile variant, row-block order)
struct TuneKey {
    int P, genotypes, ktot, n_bins, cutoff_decade, window_log2;
    bool operator<(const TuneKey& o) const {
        const int a[6] = {P, genotypes, ktot, n_bins, cutoff_decade, window_log2};
        const int b[6] = {o.P, o.genotypes, o.ktot, o.n_bins, o.cutoff_decade, o.window_log2};
        for (int i = 0; i < 6; ++i)
            if (a[i] != b[i]) return a[i] < b[i];
        return false;
    }
};
struct TuneChoice {
    int variant = 0;  // partner-tile variant (tc_tile_width)
    int order = 0;    // row blocks: 0 = largest windows first, 1 = window order
    float ms = 0.f;   // the winning candidate's kernel time when tuned
};
TuneKey tune_key_of(const ldk_parse_t* d, const ParseShape& sh);
bool tune_lookup(const TuneKey& k, TuneChoice* c);
void tune_store(const TuneKey& k, const TuneChoice& c);

// ldk_parse with a caller-provided workspace; device_items lists the tensor-core row
// blocks with a device kernel (window order) instead of a host-built upload.
int parse_impl(const ldk_parse_t* d, const ldk_parse_out_t* out, void* workspace, size_t workspace_bytes,
               void* stream, bool device_items);

void set_error(const char* fmt, ...);

}  // namespace ldk
