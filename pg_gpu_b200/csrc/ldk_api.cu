// C ABI of libldk (declared in include/ldk.h).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <array>
#include <atomic>
#include <map>
#include <mutex>
#include <vector>

#include "ldk_internal.h"

namespace ldk {

namespace {
thread_local char g_err[512] = "";

// Optional timing of the main parse kernel (CUDA events on the caller's stream).
thread_local int g_prof = 0;
thread_local float g_kernel_ms = -1.0f;
thread_local cudaEvent_t g_ev[2] = {nullptr, nullptr};
thread_local int g_ev_dev = -1;

bool prof_events() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (g_ev[0] && g_ev_dev == dev) return true;
    if (g_ev[0]) { cudaEventDestroy(g_ev[0]); cudaEventDestroy(g_ev[1]); g_ev[0] = g_ev[1] = nullptr; }
    if (cudaEventCreate(&g_ev[0]) != cudaSuccess || cudaEventCreate(&g_ev[1]) != cudaSuccess) return false;
    g_ev_dev = dev;
    return true;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int stats_of(int P) { return P == 1 ? 3 : P == 2 ? 15 : P == 3 ? 45 : P == 4 ? 105 : 0; }

int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return LDK_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return LDK_ERR_CUDA;
}

// Device check: the library carries sm_100a code only.
int check_arch() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_error("no CUDA device");
        return LDK_ERR_CUDA;
    }
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (major != 10 || minor != 0) {
        set_error("libldk is built for sm_100a (B200); device %d is sm_%d%d", dev, major, minor);
        return LDK_ERR_ARCH;
    }
    return LDK_OK;
}

struct Layout {
    size_t status_off = 0, jmax_off = 0, win_off = 0, rb_off = 0, items_off = 0, hv_off = 0, rtab_off = 0,
           gtab_off = 0, fx_off = 0, fx_bytes = 0, total = 0;
    int n_row_blocks = 0;
};

bool shape_of(const ldk_parse_t* d, ParseShape& sh) {
    sh.P = d->n_pops;
    sh.genotypes = d->genotypes;
    sh.n_stats = stats_of(d->n_pops);
    sh.n_bins = d->n_bins;
    sh.planes = tc_planes(sh);
    int k = 0;
    sh.max_n = 0;
    for (int p = 0; p < LDK_MAX_POPS + 1; ++p) sh.kofs[p] = 0;
    for (int p = 0; p < d->n_pops; ++p) {
        sh.kofs[p] = k;
        const int np = d->pop_offsets[p + 1] - d->pop_offsets[p];
        k += (np + 31) / 32 * 32;
        if (np > sh.max_n) sh.max_n = np;
    }
    for (int p = d->n_pops; p <= LDK_MAX_POPS; ++p) sh.kofs[p] = k;
    sh.ktot = (k + 127) / 128 * 128;
    sh.rtab_global = 0;
    sh.rtab_global = (d->method != LDK_METHOD_PLAIN_FP64 && !sh.genotypes && tc_rtab_global(sh)) ? 1 : 0;
    return true;
}

int window_count(const ldk_parse_t* d) { return d->window_offsets ? d->n_windows : 1; }

int64_t window_bound(const ldk_parse_t* d, int w) {
    if (d->window_offsets) return d->window_offsets[w];
    return w == 0 ? 0 : d->n_var;
}

// End of window w's anchors (left SNPs of its pairs).
int64_t anchor_bound(const ldk_parse_t* d, int w) {
    return d->anchor_end ? d->anchor_end[w] : window_bound(d, w + 1);
}

Layout layout_of(const ldk_parse_t* d, const ParseShape& sh) {
    Layout L;
    size_t off = 0;
    L.status_off = off;
    off += 256;
    L.jmax_off = off;
    off = align_up(off + (size_t)d->n_var * sizeof(int32_t), 256);
    L.win_off = off;  // window offsets, then anchor ends
    off = align_up(off + (size_t)(2 * window_count(d) + 1) * sizeof(int64_t), 256);
    L.fx_off = off;
    L.fx_bytes = (size_t)d->n_blocks * d->n_bins * (sh.n_stats + 1) * kFxLimbs * sizeof(unsigned long long);
    off = align_up(off + L.fx_bytes, 256);
    if (d->method != LDK_METHOD_PLAIN_FP64) {
        int n_rb = 0;
        const int rows = tc_rows_per_block(sh);
        for (int w = 0; w < window_count(d); ++w) {
            const int64_t m = anchor_bound(d, w) - window_bound(d, w);
            n_rb += (int)((m + rows - 1) / rows);
        }
        L.n_row_blocks = n_rb;
        L.rb_off = off;
        off = align_up(off + (size_t)n_rb * 2 * sizeof(int32_t), 256);
        L.items_off = off;
        off = align_up(off + (size_t)tc_item_capacity(n_rb) * 4 * sizeof(int32_t), 1024);
        L.hv_off = off;
        off = align_up(off + (size_t)d->n_var * sh.planes * sh.ktot, 256);
        if (sh.rtab_global) {
            L.rtab_off = off;
            off = align_up(off + (size_t)(sh.max_n + 1) * 4 * sizeof(double), 256);
        }
        if (sh.genotypes && sh.P <= 3) {  // GenoRecip per valid count
            L.gtab_off = off;
            off = align_up(off + (size_t)(sh.max_n + 1) * 9 * sizeof(double), 256);
        }
    }
    L.total = off;
    return L;
}

int validate(const ldk_parse_t* d) {
    if (!d) { set_error("null descriptor"); return LDK_ERR_ARG; }
    if (d->n_pops < 1 || d->n_pops > LDK_MAX_POPS) { set_error("n_pops must be 1..4"); return LDK_ERR_ARG; }
    if (d->n_bins < 1 || d->n_bins > LDK_MAX_BINS) { set_error("n_bins must be 1..64"); return LDK_ERR_ARG; }
    for (int b = 0; b < d->n_bins; ++b)
        if (!(d->edges[b] < d->edges[b + 1])) { set_error("bin edges must increase"); return LDK_ERR_ARG; }
    if (d->n_var < 0 || d->n_var > (int64_t)INT32_MAX - 1024) { set_error("n_var out of range"); return LDK_ERR_ARG; }
    if (d->n_var > 0 && (!d->X || !d->pos || !d->pop_rows)) { set_error("null input pointer"); return LDK_ERR_ARG; }
    if (d->x_format != LDK_X_INT8 && d->x_format != LDK_X_PACKED2) { set_error("unknown x_format"); return LDK_ERR_ARG; }
    if (d->x_format == LDK_X_INT8 && d->ld_x < d->n_var) { set_error("ld_x < n_var"); return LDK_ERR_ARG; }
    if (d->x_format == LDK_X_PACKED2 && d->ld_x < (d->n_var + 3) / 4) { set_error("ld_x < ceil(n_var / 4) packed bytes"); return LDK_ERR_ARG; }
    if (d->pop_offsets[0] != 0) { set_error("pop_offsets[0] must be 0"); return LDK_ERR_ARG; }
    for (int p = 0; p < d->n_pops; ++p)
        if (d->pop_offsets[p + 1] <= d->pop_offsets[p]) { set_error("empty population %d", p); return LDK_ERR_ARG; }
    if (d->n_blocks < 1) { set_error("n_blocks must be >= 1"); return LDK_ERR_ARG; }
    if (d->method != LDK_METHOD_PLAIN_FP64 && d->method != LDK_METHOD_TC) {
        set_error("unknown method");
        return LDK_ERR_ARG;
    }
    if (!(d->max_dist >= 0.0)) { set_error("max_dist must be >= 0"); return LDK_ERR_ARG; }
    if (d->window_offsets) {
        if (d->n_windows < 1) { set_error("n_windows must be >= 1"); return LDK_ERR_ARG; }
        if (d->window_offsets[0] != 0 || d->window_offsets[d->n_windows] != d->n_var) {
            set_error("window_offsets must run from 0 to n_var");
            return LDK_ERR_ARG;
        }
        for (int w = 0; w < d->n_windows; ++w)
            if (d->window_offsets[w + 1] < d->window_offsets[w]) { set_error("window_offsets must not decrease"); return LDK_ERR_ARG; }
    }
    if (d->anchor_end)
        for (int w = 0; w < window_count(d); ++w)
            if (d->anchor_end[w] < window_bound(d, w) || d->anchor_end[w] > window_bound(d, w + 1)) {
                set_error("anchor_end[%d] outside its window", w);
                return LDK_ERR_ARG;
            }
    if (d->x_format == LDK_X_PACKED2 && d->method == LDK_METHOD_PLAIN_FP64) {
        set_error("the plain method reads int8 codes; packed input needs LDK_METHOD_TC");
        return LDK_ERR_UNSUPPORTED;
    }
    return LDK_OK;
}

const char* status_text(unsigned s) {
    if (s & LDK_DEVERR_TIMEOUT) return "device wait timed out";
    if (s & LDK_DEVERR_BLOCK_RANGE) return "snp_block outside [0, n_blocks)";
    if (s & LDK_DEVERR_BLOCK_SPAN)
        return "a tensor-core row block spans more bootstrap blocks than it stages (64 SNPs: two; genotypes, 128 SNPs: four)";
    if (s & LDK_DEVERR_ACCUM) return "a bin sum outside the fixed-point accumulator's range (|x| >= 2^63 or not finite)";
    if (s & LDK_DEVERR_BAD_INPUT) return "unsorted positions or coordinates, or allele codes outside {-1, 0, 1} (haplotypes) or {-1, 0, 1, 2} (genotypes)";
    return "device error";
}

}  // namespace

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

}  // namespace ldk

using namespace ldk;

namespace ldk {
namespace {

// A parse call's geometry and its scratch carved out of the caller's workspace.
struct Prepared {
    ParseShape sh;
    Layout L;
    Scratch w;
    unsigned char* ws = nullptr;
};

int prepare(const ldk_parse_t* d, void* workspace, size_t workspace_bytes, Prepared& P) {
    if (int rc = validate(d)) return rc;
    shape_of(d, P.sh);
    P.L = layout_of(d, P.sh);
    if (!workspace || workspace_bytes < P.L.total) {
        set_error("workspace of %zu bytes is smaller than the %zu required", workspace_bytes, P.L.total);
        return LDK_ERR_WORKSPACE;
    }
    if (reinterpret_cast<uintptr_t>(workspace) % 256) { set_error("workspace must be 256-byte aligned"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    if (d->method != LDK_METHOD_PLAIN_FP64 && tc_smem_bytes(P.sh) > 227 * 1024) {
        set_error("bins x statistics exceed the tensor-core kernel's shared-memory staging");
        return LDK_ERR_UNSUPPORTED;
    }
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    P.ws = ws;
    P.w.status = reinterpret_cast<unsigned*>(ws + P.L.status_off);
    P.w.row_counter = reinterpret_cast<int*>(ws + P.L.status_off + 64);
    P.w.item_counter = reinterpret_cast<int*>(ws + P.L.status_off + 128);
    P.w.n_items = reinterpret_cast<int*>(ws + P.L.status_off + 192);
    P.w.jmax = reinterpret_cast<int32_t*>(ws + P.L.jmax_off);
    P.w.win_off = reinterpret_cast<int64_t*>(ws + P.L.win_off);
    P.w.anc_end = P.w.win_off + window_count(d) + 1;
    P.w.fx = reinterpret_cast<unsigned long long*>(ws + P.L.fx_off);
    P.w.row_blocks = reinterpret_cast<int32_t*>(ws + P.L.rb_off);
    P.w.items = reinterpret_cast<int32_t*>(ws + P.L.items_off);
    P.w.hv = ws + P.L.hv_off;
    P.w.rtab = P.sh.rtab_global ? static_cast<void*>(ws + P.L.rtab_off) : nullptr;
    P.w.gtab = (d->method != LDK_METHOD_PLAIN_FP64 && P.sh.genotypes && P.sh.P <= 3)
                   ? static_cast<void*>(ws + P.L.gtab_off)
                   : nullptr;
    return LDK_OK;
}

int check_outputs(const ldk_parse_out_t* out) {
    if (!out || !out->sums || !out->r2_sums || !out->pairs || !out->r2_counts) {
        set_error("null output pointer");
        return LDK_ERR_ARG;
    }
    return LDK_OK;
}

// The tensor-core row-block list (64 SNPs for haplotypes, 128 for genotypes, up to each
// window's anchor end) in claim order: 0 = the largest windows' row blocks first, 1 = window
// order.  Each launch splits it into work items (launch_split_items), which the kernel's
// CTAs claim in list order.
int upload_items(const ldk_parse_t* d, const Prepared& P, cudaStream_t s, int claim_order) {
    int rc;
    const int rows = tc_rows_per_block(P.sh);
    std::vector<int> order(window_count(d));
    for (int k = 0; k < (int)order.size(); ++k) order[k] = k;
    if (claim_order == 0)
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return (window_bound(d, x + 1) - window_bound(d, x)) > (window_bound(d, y + 1) - window_bound(d, y));
        });
    std::vector<int32_t> rb;
    rb.reserve((size_t)P.L.n_row_blocks * 2);
    for (int wi : order) {
        const int64_t ae = anchor_bound(d, wi);
        for (int64_t r0 = window_bound(d, wi); r0 < ae; r0 += rows) {
            rb.push_back((int32_t)r0);
            rb.push_back((int32_t)std::min<int64_t>(r0 + rows, ae));
        }
    }
    if (!rb.empty() &&
        (rc = check_cuda(cudaMemcpyAsync(P.w.row_blocks, rb.data(), rb.size() * sizeof(int32_t),
                                         cudaMemcpyHostToDevice, s), "upload row blocks")))
        return rc;
    return LDK_OK;
}

// Host-side plan into the workspace: window offsets and, for the tensor-core method, the
// row-block list in the tuned claim order (largest windows first if the shape is untuned)
// -- or, with device_items, the list is built on the device in window order.
int upload_plan(const ldk_parse_t* d, const Prepared& P, cudaStream_t s, bool device_items) {
    int rc;
    const int nw = window_count(d);
    std::vector<int64_t> woff(2 * nw + 1);  // window offsets, then anchor ends (the workspace layout)
    for (int k = 0; k <= nw; ++k) woff[k] = window_bound(d, k);
    for (int k = 0; k < nw; ++k) woff[nw + 1 + k] = anchor_bound(d, k);
    if ((rc = check_cuda(cudaMemcpyAsync(P.w.win_off, woff.data(), woff.size() * sizeof(int64_t),
                                         cudaMemcpyHostToDevice, s), "upload windows")))
        return rc;
    if (d->method == LDK_METHOD_PLAIN_FP64) return LDK_OK;
    if (device_items)
        return check_cuda(launch_build_items(P.w, window_count(d), tc_rows_per_block(P.sh), s), "row blocks");
    TuneChoice c;
    return upload_items(d, P, s, tune_lookup(tune_key_of(d, P.sh), &c) ? c.order : 0);
}

// Zeroes the outputs, the status block and the fixed-point bin accumulators.
int clear(const ldk_parse_t* d, const ldk_parse_out_t* out, const Prepared& P, cudaStream_t s) {
    const int nb = d->n_bins, NS = stats_of(d->n_pops);
    int rc;
    if ((rc = check_cuda(cudaMemsetAsync(out->sums, 0, sizeof(double) * d->n_blocks * nb * NS, s), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(out->r2_sums, 0, sizeof(double) * d->n_blocks * nb, s), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(out->pairs, 0, sizeof(uint64_t) * d->n_blocks * nb, s), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(out->r2_counts, 0, sizeof(uint64_t) * d->n_blocks * nb, s), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(P.ws + P.L.status_off, 0, 256, s), "memset")) ||
        (rc = check_cuda(cudaMemsetAsync(P.ws + P.L.fx_off, 0, P.L.fx_bytes, s), "memset")))
        return rc;
    return LDK_OK;
}

// Device work of one parse (after the plan is in the workspace): pair ranges, indicator
// planes and the parse kernel.  Host work: tensor-map encoding and launch configuration.
// ---- autotuning: the fastest (tile variant, row-block order) per shape class (ldk_tune.cu)
std::atomic<int> g_autotune{-1};  // -1: LDK_AUTOTUNE not read yet

bool autotune_on() {
    if (g_autotune.load() < 0) {
        const char* e = getenv("LDK_AUTOTUNE");
        int v = (e && atoi(e) == 1) ? 1 : 0, expect = -1;
        g_autotune.compare_exchange_strong(expect, v);
    }
    return g_autotune.load() == 1;
}

// The tuned tile variant of this shape; -1 if the shape has not been tuned.
int tuned_variant(const ldk_parse_t* d, const ParseShape& sh) {
    TuneChoice c;
    return tune_lookup(tune_key_of(d, sh), &c) ? c.variant : -1;
}

// Candidates worth timing: the alternative tile only where its width differs, the window
// order only where there are several windows.
int n_variants(const ldk_parse_t* d, const ParseShape& sh) {
    return tc_tile_width(sh, 1) != tc_tile_width(sh, 0) ? 2 : 1;
}
int n_orders(const ldk_parse_t* d) { return window_count(d) > 1 ? 2 : 1; }

// Runs every (tile variant, row-block order) candidate twice on this call's input (outputs
// cleared before each run), times the second run with CUDA events and stores the fastest
// in the table; the row-block list is left in the winner's order.  The outputs keep the
// last candidate's sums.
int autotune_tc(const ldk_parse_t* dd, const ldk_parse_out_t* out, const Prepared& P, cudaStream_t s);
int read_status(const unsigned* status_dev, cudaStream_t s);

// The work items for tile variant `variant` (from this run's pair ranges), then the parse
// kernel, its launch bracketed by the profiling events when `prof`.
cudaError_t launch_tc(const ldk_parse_t* dd, const ldk_parse_out_t* out, const Prepared& P, int variant,
                      cudaStream_t s, bool prof = false) {
    const int n_rb = P.L.n_row_blocks;
    if (n_rb == 0) {
        if (prof) { cudaEventRecord(g_ev[0], s); cudaEventRecord(g_ev[1], s); }
        return cudaSuccess;
    }
    cudaError_t e = launch_split_items(P.w, n_rb, tc_tile_width(P.sh, variant), tc_min_item_tiles(P.sh), s);
    if (e != cudaSuccess) return e;
    if (prof) cudaEventRecord(g_ev[0], s);
    e = launch_parse_tc(dd, out, P.w, P.sh, tc_item_capacity(n_rb), variant, s);
    if (prof) cudaEventRecord(g_ev[1], s);
    return e;
}

int enqueue_device(const ldk_parse_t* d, const ldk_parse_out_t* out, const Prepared& P, cudaStream_t s, bool prof,
                   bool tune = false) {
    int rc;
    ldk_parse_t dd = *d;
    dd.n_windows = window_count(d);
    if ((rc = check_cuda(launch_jmax(&dd, P.w, s), "pair ranges"))) return rc;
    if (d->method == LDK_METHOD_PLAIN_FP64) {
        if (prof) cudaEventRecord(g_ev[0], s);
        if ((rc = check_cuda(launch_parse_plain(&dd, out, P.w, P.sh, s), "plain parse"))) return rc;
        if (prof) cudaEventRecord(g_ev[1], s);
        if ((rc = check_cuda(launch_fx_finish(&dd, out, P.w, P.sh.n_stats, s), "bin sums"))) return rc;
    } else {
        if ((rc = check_cuda(launch_prep_planes(&dd, P.w, P.sh, s), "indicator planes"))) return rc;
        if (P.w.rtab && (rc = check_cuda(launch_fill_rtab(P.w.rtab, P.sh.max_n, s), "reciprocal table"))) return rc;
        if (P.w.gtab && (rc = check_cuda(launch_fill_gtab(P.w.gtab, P.sh.max_n, s), "reciprocal table"))) return rc;
        if (tune && n_variants(d, P.sh) * n_orders(d) > 1 && tuned_variant(d, P.sh) < 0) {
            if ((rc = autotune_tc(&dd, out, P, s))) return rc;
            // the candidate runs left their sums and a spent row-block counter behind
            if ((rc = clear(&dd, out, P, s))) return rc;
        }
        const int v = tuned_variant(d, P.sh);
        if ((rc = check_cuda(launch_tc(&dd, out, P, v < 0 ? 0 : v, s, prof), "tensor-core parse"))) return rc;
        if ((rc = check_cuda(launch_fx_finish(&dd, out, P.w, P.sh.n_stats, s), "bin sums"))) return rc;
    }
    return LDK_OK;
}

int autotune_tc(const ldk_parse_t* dd, const ldk_parse_out_t* out, const Prepared& P, cudaStream_t s) {
    cudaEvent_t e0, e1;
    int rc;
    if ((rc = check_cuda(cudaEventCreate(&e0), "autotune events"))) return rc;
    if ((rc = check_cuda(cudaEventCreate(&e1), "autotune events"))) { cudaEventDestroy(e0); return rc; }
    TuneChoice best;
    bool found = false;
    int uploaded = -1;
    for (int o = 0; o < n_orders(dd) && !rc; ++o) {
        if ((rc = upload_items(dd, P, s, o))) break;
        uploaded = o;
        for (int v = 0; v < n_variants(dd, P.sh) && !rc; ++v) {
            // an untimed run first (first-launch costs, caches), then the timed one
            bool fits = true;
            float ms = 0.f;
            for (int rep = 0; rep < 2 && fits && !rc; ++rep) {
                if ((rc = clear(dd, out, P, s))) break;
                cudaEventRecord(e0, s);
                if (launch_tc(dd, out, P, v, s) != cudaSuccess) {
                    cudaGetLastError();  // this variant does not fit the shape (e.g. shared memory): skip it
                    fits = false;
                    break;
                }
                cudaEventRecord(e1, s);
                if ((rc = read_status(P.w.status, s))) break;
                cudaEventElapsedTime(&ms, e0, e1);
            }
            if (fits && !rc && (!found || ms < best.ms)) {
                best.variant = v;
                best.order = o;
                best.ms = ms;
                found = true;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (!found) best = TuneChoice{};
    if (uploaded != best.order && (rc = upload_items(dd, P, s, best.order))) return rc;
    tune_store(tune_key_of(dd, P.sh), best);
    return LDK_OK;
}

int read_status(const unsigned* status_dev, cudaStream_t s) {
    unsigned status = 0;
    int rc;
    if ((rc = check_cuda(cudaMemcpyAsync(&status, status_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "status")))
        return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(s), "ldk_parse"))) return rc;
    if (status) {
        set_error("%s (status 0x%x)", status_text(status), status);
        return LDK_ERR_DEVICE;
    }
    return LDK_OK;
}

}  // namespace
}  // namespace ldk

int ldk::parse_impl(const ldk_parse_t* d, const ldk_parse_out_t* out, void* workspace, size_t workspace_bytes,
                    void* stream, bool device_items) {
    if (int rc = validate(d)) return rc;
    if (int rc = check_outputs(out)) return rc;
    Prepared P;
    if (int rc = prepare(d, workspace, workspace_bytes, P)) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (int rc = clear(d, out, P, s)) return rc;
    if (d->n_var < 2) return LDK_OK;
    if (int rc = upload_plan(d, P, s, device_items)) return rc;
    const bool prof = !device_items && g_prof && prof_events();
    g_kernel_ms = -1.0f;
    if (int rc = enqueue_device(d, out, P, s, prof, !device_items && autotune_on())) return rc;
    const int rc = read_status(P.w.status, s);
    if (prof) cudaEventElapsedTime(&g_kernel_ms, g_ev[0], g_ev[1]);
    return rc;
}

extern "C" {

int ldk_version(void) { return 10000; }

const char* ldk_last_error(void) { return g_err; }

int ldk_n_stats(int P) { return stats_of(P); }

int ldk_counts_hap(const int8_t* X, int64_t ld_x, int64_t n_var, const int32_t* rows, int32_t n_rows,
                   const int32_t* idx_i, const int32_t* idx_j, int64_t n_pairs, int32_t* counts, int32_t* n_valid,
                   void* stream) {
    if (n_pairs < 0 || n_rows < 0 || ld_x < n_var) { set_error("bad sizes"); return LDK_ERR_ARG; }
    if (n_pairs > 0 && (!X || !rows || !idx_i || !idx_j || !counts)) { set_error("null pointer"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    return check_cuda(launch_counts(0, X, ld_x, rows, n_rows, idx_i, idx_j, n_pairs, counts, n_valid,
                                    (cudaStream_t)stream), "ldk_counts_hap");
}

int ldk_counts_geno(const int8_t* X, int64_t ld_x, int64_t n_var, const int32_t* rows, int32_t n_rows,
                    const int32_t* idx_i, const int32_t* idx_j, int64_t n_pairs, int32_t* counts, int32_t* n_valid,
                    void* stream) {
    if (n_pairs < 0 || n_rows < 0 || ld_x < n_var) { set_error("bad sizes"); return LDK_ERR_ARG; }
    if (n_pairs > 0 && (!X || !rows || !idx_i || !idx_j || !counts)) { set_error("null pointer"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    return check_cuda(launch_counts(1, X, ld_x, rows, n_rows, idx_i, idx_j, n_pairs, counts, n_valid,
                                    (cudaStream_t)stream), "ldk_counts_geno");
}

int ldk_stats(int genotypes, int P, const int32_t* counts, const int32_t* n_valid, int64_t n_pairs, double* out,
              void* stream) {
    if (P < 1 || P > LDK_MAX_POPS || n_pairs < 0) { set_error("bad P or n_pairs"); return LDK_ERR_ARG; }
    if (n_pairs > 0 && (!counts || !out)) { set_error("null pointer"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    return check_cuda(launch_stats(genotypes, P, counts, n_valid, n_pairs, out, (cudaStream_t)stream), "ldk_stats");
}

int ldk_raw_hap(int case_id, const int32_t* args_host, int P_total, const double* counts, const double* n_valid,
                int64_t n_pairs, double* out, void* stream) {
    if (case_id < 0 || case_id > 14 || P_total < 1 || P_total > LDK_MAX_POPS || n_pairs < 0 || !args_host) {
        set_error("bad raw-call arguments");
        return LDK_ERR_ARG;
    }
    static const int arity[15] = {1, 2, 1, 2, 2, 2, 3, 1, 2, 3, 3, 4, 2, 2, 3};
    int32_t g[4] = {0, 0, 0, 0};
    for (int k = 0; k < arity[case_id]; ++k) {
        if (args_host[k] < 0 || args_host[k] >= P_total) { set_error("population index out of range"); return LDK_ERR_ARG; }
        g[k] = args_host[k];
    }
    if (n_pairs > 0 && (!counts || !out)) { set_error("null pointer"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    return check_cuda(launch_raw_hap(case_id, g, P_total, counts, n_valid, n_pairs, out, (cudaStream_t)stream),
                      "ldk_raw_hap");
}

int ldk_r_family(int which, const double* counts, const double* n_valid, int64_t n_pairs, double* out, void* stream) {
    if (which < 0 || which > 2 || n_pairs < 0) { set_error("bad arguments"); return LDK_ERR_ARG; }
    if (n_pairs > 0 && (!counts || !out)) { set_error("null pointer"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    return check_cuda(launch_r_family(which, counts, n_valid, n_pairs, out, (cudaStream_t)stream), "ldk_r_family");
}

size_t ldk_parse_workspace_size(const ldk_parse_t* d) {
    if (validate(d) != LDK_OK) return 0;
    ParseShape sh;
    shape_of(d, sh);
    return layout_of(d, sh).total;
}

int ldk_parse(const ldk_parse_t* d, const ldk_parse_out_t* out, void* workspace, size_t workspace_bytes,
              void* stream) {
    return parse_impl(d, out, workspace, workspace_bytes, stream, false);
}

int ldk_parse_setup(const ldk_parse_t* d, void* workspace, size_t workspace_bytes, void* stream) {
    Prepared P;
    if (int rc = prepare(d, workspace, workspace_bytes, P)) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (int rc = upload_plan(d, P, s, false)) return rc;
    return check_cuda(cudaStreamSynchronize(s), "ldk_parse_setup");
}

int ldk_parse_enqueue(const ldk_parse_t* d, const ldk_parse_out_t* out, void* workspace, size_t workspace_bytes,
                      void* stream) {
    if (int rc = check_outputs(out)) return rc;
    Prepared P;
    if (int rc = prepare(d, workspace, workspace_bytes, P)) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (int rc = clear(d, out, P, s)) return rc;
    if (d->n_var < 2) return LDK_OK;
    return enqueue_device(d, out, P, s, false);
}

size_t ldk_ld_matrix_workspace_size(int64_t n_var, int32_t n_sel) {
    if (n_var < 0 || n_sel < 1) return 0;
    return ld_matrix_workspace(n_var, n_sel);
}

int ldk_ld_matrix(const int8_t* X, int64_t ld_x, int64_t n_var, const int32_t* rows, int32_t n_sel, int estimator,
                  double* out, int64_t ld_out, double* sums, void* workspace, size_t workspace_bytes, void* stream) {
    if (n_var < 0 || n_var > (int64_t)INT32_MAX - 1024 || n_sel < 1 || ld_x < n_var) {
        set_error("bad sizes");
        return LDK_ERR_ARG;
    }
    if (estimator < LDK_LDM_R2 || estimator > LDK_LDM_SIGMA_D2_GENO) { set_error("unknown estimator"); return LDK_ERR_ARG; }
    if (n_var > 0 && (!X || !rows)) { set_error("null input pointer"); return LDK_ERR_ARG; }
    if (out && ld_out < n_var) { set_error("ld_out < n_var"); return LDK_ERR_ARG; }
    const size_t need = ld_matrix_workspace(n_var, n_sel);
    if (!workspace || workspace_bytes < need) {
        set_error("workspace of %zu bytes is smaller than the %zu required", workspace_bytes, need);
        return LDK_ERR_WORKSPACE;
    }
    if (reinterpret_cast<uintptr_t>(workspace) % 256) { set_error("workspace must be 256-byte aligned"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    unsigned* status = reinterpret_cast<unsigned*>(ws);
    if (int rc = check_cuda(cudaMemsetAsync(ws, 0, 256, s), "memset")) return rc;
    if (int rc = check_cuda(launch_ld_matrix(X, ld_x, n_var, rows, n_sel, estimator, out, ld_out, sums, ws, status, s),
                            "all-pairs LD"))
        return rc;
    return read_status(status, s);
}

int ldk_autotune(int enable) {
    g_autotune.store(enable ? 1 : 0);
    return LDK_OK;
}

int ldk_tile_width(const ldk_parse_t* d) {
    if (int rc = validate(d)) return rc;
    if (d->method == LDK_METHOD_PLAIN_FP64) return 0;
    ParseShape sh;
    shape_of(d, sh);
    const int v = tuned_variant(d, sh);
    return tc_tile_width(sh, v < 0 ? 0 : v);
}

int ldk_parse_reproducible(const ldk_parse_t* d) {
    if (int rc = validate(d)) return rc;
    if (d->method == LDK_METHOD_PLAIN_FP64) return 1;
    ParseShape sh;
    shape_of(d, sh);
    const int v = tuned_variant(d, sh);
    return tc_private_staging(sh, v < 0 ? 0 : v) ? 1 : 0;
}

int ldk_tc_row_blocks(int genotypes, int32_t* rows, int32_t* max_blocks) {
    if (!rows || !max_blocks) { set_error("null output pointer"); return LDK_ERR_ARG; }
    ParseShape sh{};
    sh.genotypes = genotypes ? 1 : 0;
    *rows = tc_rows_per_block(sh);
    *max_blocks = tc_block_slots(sh);
    return LDK_OK;
}

int ldk_parse_status(const void* workspace, void* stream) {
    if (!workspace) { set_error("null workspace"); return LDK_ERR_ARG; }
    return read_status(static_cast<const unsigned*>(workspace), (cudaStream_t)stream);
}

int ldk_profile(int enable) {
    g_prof = enable ? 1 : 0;
    return LDK_OK;
}

double ldk_profile_last_kernel_ms(void) { return (double)g_kernel_ms; }

int ldk_probe_peaks(double* int8_ops_per_s, double* fp64_fma_per_s, void* stream) {
    if (!int8_ops_per_s || !fp64_fma_per_s) { set_error("null pointer"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    *int8_ops_per_s = 0.0;
    *fp64_fma_per_s = 0.0;
    unsigned st = 0;
    if (int rc = check_cuda(probe_peaks(int8_ops_per_s, fp64_fma_per_s, &st, (cudaStream_t)stream), "peak probes"))
        return rc;
    if (st) {
        set_error("peak probe: %s (status 0x%x)", status_text(st), st);
        return LDK_ERR_DEVICE;
    }
    return LDK_OK;
}

int ldk_block_combine(const double* block_sums, int64_t n_blocks, int64_t k, const int32_t* weights, int64_t n_rep,
                      double* out, void* stream) {
    if (n_blocks < 0 || k < 0 || n_rep < 0) { set_error("bad sizes"); return LDK_ERR_ARG; }
    if (n_rep * k > 0 && (!block_sums || !weights || !out)) { set_error("null pointer"); return LDK_ERR_ARG; }
    if (int rc = check_arch()) return rc;
    return check_cuda(launch_block_combine(block_sums, n_blocks, k, weights, n_rep, out, (cudaStream_t)stream),
                      "ldk_block_combine");
}

}  // extern "C"
