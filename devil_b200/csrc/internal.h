// Host-side declarations shared by the kernel translation units and the
// C-ABI implementation (not installed; the public interface is
// include/devil_b200.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "passes.cuh"

namespace devil {

enum PassKind { PASS_IRLS = 0, PASS_MOM = 1, PASS_MLE = 2, PASS_SANDWICH = 3 };
enum Engine { ENGINE_REG = 0, ENGINE_GEN = 1, ENGINE_GRP = 2, ENGINE_TC = 3, ENGINE_TCW = 4 };

inline int pass_nw(PassKind k) { return k == PASS_MLE ? 3 : (k == PASS_MOM ? 0 : 1); }
inline int pass_nv(PassKind k) { return (k == PASS_IRLS || k == PASS_SANDWICH) ? 1 : 0; }
inline int pass_ns(PassKind k) { return k == PASS_MOM ? 2 : (k == PASS_MLE ? 4 : 0); }
inline int pass_nf(PassKind k) { return k == PASS_MLE ? 2 : 0; }
inline int pass_na(PassKind k, int P) {
    return pass_nw(k) * P * (P + 1) / 2 + pass_nv(k) * P + pass_nf(k);
}

struct PassParamsAny {
    const float* beta;        // G x P float (FP32 passes)
    const double* beta_d;     // G x P double (FP64 passes)
    const float* k;           // IRLS
    const double* log_theta;  // MLE
    const double* theta;      // SANDWICH
};

struct PassLaunch {
    PassKind kind;
    Engine engine;
    int P;
    int xs_pad;     // row stride of geo.X
    int GT;
    int val_u16;    // 1: uint16 values, 0: float values
    int use_tma;    // FP32 passes, p <= 8: TMA-staged register engine
    int nseg;       // grid.x
    int ntiles;     // grid.y
    PassGeom geo;
    PassParamsAny prm;
    cudaStream_t stream;
    int* occ_out = nullptr;  // non-null: report the kernel's resident blocks per SM, launch nothing
    int plain = 0;           // the plain comparison form (FP32 staging in the shared-memory engine)
};

// engine choice helpers
int reg_max_p();
int tma_chunk_cells(int xs);  // fine-segment size the TMA engine expects
int reg_default_gt(PassKind k, int P);
bool reg_gt_supported(PassKind k, int P, int GT);
int gen_default_gt(PassKind k, int P);
size_t gen_smem_bytes(PassKind k, int P, int GT, int plain);
bool gen_f32_staging(PassKind k, int plain);

cudaError_t launch_reg_pass(const PassLaunch& L);

// Raise the kernel's dynamic shared-memory cap to at least `bytes` on the
// current device; never lowers it.  The cap is process-wide per kernel, so
// concurrent callers (devil_fit_batch workers with different problem
// shapes) must not set it to their own size just before another caller's
// larger launch.
cudaError_t raise_dyn_smem_raw(const void* func, size_t bytes);
template <class K>
cudaError_t raise_dyn_smem(K* kern, size_t bytes) {
    return raise_dyn_smem_raw(reinterpret_cast<const void*>(kern), bytes);
}

// resident blocks per SM of the kernel a pass launch would use (cached)
int pass_blocks_per_sm(PassKind kind, Engine engine, int P, int GT, int val_u16, int plain = 0);

// ---- tensor-core IRLS engine (kernels_tc.cu) ----
int tc_max_p();
int tc_tile_genes(PassKind k);  // genes per block tile: 128 (IRLS), 32 (MLE)
int tc_chunk_cells();
bool tc_enabled(PassKind k);  // DEVIL_TC=1 (IRLS), DEVIL_TC_MLE=1 (MLE) select the engine
int64_t tc_zimg_quads(int64_t n);    // cell quads covered by the product image
int64_t tc_zimg_float4s(int64_t n);  // its size in float4
cudaError_t launch_tc_zimg(const float* Xrm, int xs, int64_t n, int P, float4* zimg, cudaStream_t st);
cudaError_t launch_tc_pass(const PassLaunch& L, const float4* zimg);
cudaError_t launch_gen_pass(const PassLaunch& L);

// ---- tensor-core IRLS engine for p = 5..32 (kernels_tcw.cu) ----
// Inputs built once per fit by launch_tcw_prepare: the counts as a dense
// image (gene rows of ld = npad cells, uint16 or float, zero where the CSR
// has no entry), the design's feature rows xt [xs][npad] (zero past n) and
// the offsets offp [npad] (-1e30 past n: mu = 0 in the padding).
struct TcwGeom {
    const float* xt = nullptr;
    const float* offp = nullptr;
    const void* ydense = nullptr;
    int64_t ld = 0;
    int64_t npad = 0;
    int P = 0, NE = 0, NA = 0;
    int nblk = 0;  // product columns per block (tcw_nblk(P))
};
int tcw_blocks(int P);          // product blocks (grid.z)
int tcw_tile_genes(PassKind k); // genes per tile: 128 (IRLS), 32 (MLE)
int tcw_nblk(int P);
int64_t tcw_npad(int64_t n);
bool tcw_supported(int P, int xs);
cudaError_t launch_tcw_prepare(const int64_t* rowptr, const int32_t* col, const void* val, int val_u16,
                               int64_t G, int64_t n, const float* Xrm, int xs, const float* off,
                               const TcwGeom& tw, cudaStream_t st);
cudaError_t launch_tcw_pass(const PassLaunch& L, const TcwGeom& tw);
// genes with more than `limit` IRLS steps or a coefficient beyond
// +-beta_limit (or NaN): listed in act (count in *cnt, which starts at 0),
// flag[g] = 1, beta / beta_f reset to beta0, iteration count and status
// cleared; flag[g] = 0 for the others
cudaError_t launch_irls_rescue_select(const int32_t* iters_in, int64_t G, int limit, double beta_limit,
                                      const double* beta0, int P, double* beta, float* beta_f, int32_t* iters,
                                      int32_t* status, int32_t* act, int32_t* cnt, int32_t* flag, cudaStream_t st);
// out[g] = flag[g] ? v[g] : 0
cudaError_t launch_mask_i32(const int32_t* v, const int32_t* flag, int64_t G, int32_t* out, cudaStream_t st);

// ---- design-group engine (kernels_grp.cu) ----
constexpr int kBinNodes = 10;         // Gauss nodes per offset bin
constexpr double kBinWidth = 2.0;     // bin width in log size factor
constexpr int kMaxBins = 32;          // bins per group (offsets spread over < 64)
constexpr int kRuleCap = kMaxBins * kBinNodes;  // node capacity of one rule
constexpr int kMaxGroups = 256;       // distinct design rows
constexpr int kMaxFine = 4096;        // (design row, cluster) pairs
constexpr int kMinCellsPerGroup = 32; // grouping pays when groups are larger
// slice-major passes: genes below this many entries per slice on average
// take eight lanes instead of a warp (IRLS; the MLE pass, whose light genes
// load one 16-byte piece per lane at a time, switches lower).  Measured on
// the headline: IRLS 96 / 192 / 384 / 768 / 1536 -> 103.9 / 99.5 / 98.0 /
// 99.7 / 106.9 ms per step; MLE 96 / 192 / 384 -> 29.2 / 29.5 / 30.2 ms.
constexpr int kLightEntries = 384;
constexpr int kLightEntriesMle = 96;
constexpr int kSliceCells = 16384;    // cells per slice (its FP64 exp(offset), 128 KB, fits shared memory)
constexpr int kGrpTab = 2 * kPsiTab + 2;  // per-gene psi tables + psi(a), psi1(a)
constexpr int kMaxSlices = 12288;     // the CSR copy's per-warp key table stays <= 48 KB; keys fit 16 bits

// One entry of the slice-ordered CSR copy of the design-group engine: the
// cell's index within its slice and the count.
template <class VT> struct GrpEnt;
template <> struct GrpEnt<uint16_t> {
    using T = uint32_t;  // low 16 bits: index within the slice; high 16 bits: the count
    static __device__ __forceinline__ T pack(int32_t loc, uint16_t v) {
        return (uint32_t)loc | ((uint32_t)v << 16);
    }
    static __device__ __forceinline__ int loc(T e) { return (int)(e & 0xffffu); }
    static __device__ __forceinline__ float y(T e) { return (float)(e >> 16); }
};
template <> struct GrpEnt<float> {
    using T = uint2;     // x: index within the slice; y: the count's float bits
    static __device__ __forceinline__ T pack(int32_t loc, float v) {
        return make_uint2((unsigned)loc, __float_as_uint(v));
    }
    static __device__ __forceinline__ int loc(T e) { return (int)e.x; }
    static __device__ __forceinline__ float y(T e) { return __uint_as_float(e.y); }
};

struct GrpGeom {
    int P, U, C;           // design columns, groups, clusters folded into the keys (1: none)
    int S;                 // slices
    int fine;              // 1: groups are (row, cluster) pairs, one output segment per cluster
    const double* xg;      // [U][P] distinct design rows
    const double* E;       // [n] exp(offset), cells in slice order
    const void* gent;      // CSR copy: GrpEnt entries ordered by slice within each gene
    const int64_t* gptr;   // [G][S + 1] absolute start of every slice's entries
    const int32_t* sl_start;  // [S + 1] first cell (slice order) of every slice
    const int32_t* sl_key;    // [S] its key u * C + c
    const int32_t* kslice;    // [U*C + 1] first slice of every key (slices ordered by key)
    double* gsum;          // slice-major IRLS: [slots][S][NQ] per-(gene, slice) sums
    double* rowexp;        // slice-major passes: [G][U] exp(x_u . beta) by gene
    double* psitab;        // slice-major MLE: [slots][kGrpTab] psi tables, psi(a), psi1(a)
    const double* rs;      // [rules][kRuleCap] node offsets; rules 0..U-1 coarse, U.. fine
    const double* rw;      // [rules][kRuleCap] node weights
    const int32_t* rm;     // [rules] node counts
    const double* res;     // [rules][kRuleCap] exp(node offset)
    // the design rows as sparse rows (nonzero entries of xg, ascending
    // column), and for every output of the p x p assembly the list of the
    // groups that contribute to it (ascending group) with their weight:
    //   outer output q = (i <= j, packed upper triangle): x_ui x_uj
    //   vector output i: x_ui
    const int32_t* rptr;   // [U + 1]
    const int32_t* rcol;
    const double* rval;
    const int32_t* qptr;   // [P(P+1)/2 + 1]
    const int32_t* qu;
    const double* qv;
    const int32_t* vptr;   // [P + 1]
    const int32_t* vu;
    const double* vv;
    // exclusive columns: no design row has two of them nonzero (one-hot
    // cell types), so the p x p Hessian restricted to them is diagonal and
    // a Newton step needs only the Schur complement on the nA other
    // columns.  nA = 0: no such structure (dense solve).
    int nA;
    const int32_t* colA;   // [nA] the dense columns
    const int32_t* colD;   // [P - nA] the exclusive columns
    const int32_t* colpos; // [P] position in colA (>= 0) or -1 - position in colD
    // the Hessian entries that step needs (rows of the dense columns and the
    // diagonal): packed output index and up to three destinations in the
    // compact store [nA][P] rows then [P] diagonal (-1: none)
    int n_need;
    const int32_t* need_q;
    const int32_t* need_d;  // [n_need][3]
    const int32_t* act;
    const int32_t* n_act;
    // slice-major passes: the first *n_heavy active genes (the list is in
    // decreasing order of entries) take a warp each, the others eight lanes
    // each; null: a warp each
    const int32_t* n_heavy;
    int32_t* reset_next;
    double* partW;         // FP64 partial sums, layout of the other engines
    double* partS;
    int slot_stride;
};
// ---- overdispersion "new" (kernels_newod.cu) ----
struct NodArgs {
    int64_t G, n;
    int P, xs;
    const double* Xd;       // [n][xs] row-major FP64 design
    const double* off;      // [n]
    const double* xcolsum;  // [P] column sums of the design
    const int64_t* rowptr;
    const int32_t* col;
    const void* val;
    int val_u16;
    const double* beta;     // [G][P]
    const double* stats;    // [G][6] gene statistics (mean, var, ...)
    int max_iter;
    double eps;             // eps_theta (the fit tolerance)
    int gh_m, max_newton;   // Gauss-Hermite order and mode-search steps (newton_max)
    const double* gx;       // [gh_m] Gauss-Hermite nodes
    const double* gw;       // [gh_m] weights
    double* theta;          // [G] kappa
    int32_t* iters;         // [G] kappa_iters
    int32_t* err;           // [G] 0, or the reference's stop() condition (1..4)
};
cudaError_t launch_new_od(const NodArgs& a, const double* Xcm, double* xcolsum, cudaStream_t st);

cudaError_t launch_grp_pass(PassKind kind, const GrpGeom& geo, const PassParamsAny& prm, int val_u16,
                            int max_slots, cudaStream_t st);
// the IRLS, MLE, MOM and bread passes of the design-group engine,
// slice-major: a block stages one slice's exp(offset) in shared memory and
// runs its share of the genes over it, then a block per gene assembles the
// p x p sums (geo.gsum: slots x S x grp_slices_nq(kind) doubles;
// geo.rowexp: G x U exp(x_u . beta) by gene, recomputed first unless
// rowexp_fresh; geo.psitab, MLE: slots x kGrpTab)
int grp_slices_tile(int64_t hint, int S, int sm_count, int waves = 3);
// key[g] = entries of gene g, idx[g] = g (sorted descending into the work
// order of the slice-major passes)
cudaError_t launch_gene_entries(const int64_t* rowptr, int64_t G, int32_t* key, int32_t* idx,
                                cudaStream_t st);
int grp_slices_nq(PassKind k);
cudaError_t launch_grp_slices(PassKind kind, const GrpGeom& geo, const PassParamsAny& prm,
                              int val_u16, int max_slots, int tile, bool assemble, cudaStream_t st,
                              bool rowexp_fresh = false);
// cells in key order, per original cell: cslice = its slice, cloc = slice
// << 16 | index within the slice; E in slice order
cudaError_t launch_slice_cells(const int32_t* pnew, const int32_t* sl_start, int S, int64_t n,
                               const double* off, int32_t* cslice, int32_t* cloc, double* E,
                               cudaStream_t st);
// beta_0 of a grouped design: geo.act / geo.n_act list every gene, geo.gsum
// holds G x S doubles; zero_beta is G x P zeros
cudaError_t launch_grp_init_beta(const GrpGeom& geo, int val_u16, const double* zero_beta,
                                 const double* ginv, int64_t G, int tile, double* beta,
                                 float* beta_f, cudaStream_t st);
cudaError_t launch_row_hash(const double* X, int64_t n, int P, uint64_t* h, int32_t* idx,
                            cudaStream_t st);
cudaError_t launch_group_heads(const double* X, int64_t n, int P, const uint64_t* hs,
                               const int32_t* is, int32_t* flag, int32_t* bad, cudaStream_t st);
cudaError_t launch_group_assign(const int32_t* is, const int32_t* incl, const int32_t* flag,
                                int64_t n, int32_t* ucell, int32_t* head, cudaStream_t st);
cudaError_t launch_group_rows(const double* X, int64_t n, int P, const int32_t* head, int U,
                              double* xg, cudaStream_t st);
cudaError_t launch_fine_keys(const int32_t* ucell, const int32_t* ends, int C, int64_t n,
                             int32_t* fkey, int32_t* cell, cudaStream_t st);
cudaError_t launch_group_starts(const int32_t* ks, int64_t n, int K, int64_t* gstart,
                                cudaStream_t st);
cudaError_t launch_exp(const double* x, int64_t n, double* y, cudaStream_t st);
cudaError_t launch_group_rules(const int32_t* permC, const int64_t* gsC, const int32_t* permF,
                               const int64_t* gsF, int U, int nrules, const double* off, int64_t n,
                               double* scr, double* rs, double* rw, int32_t* rm, double* rerr,
                               int32_t* bad, cudaStream_t st);
cudaError_t launch_gather_keys(const int32_t* keys, const int32_t* cells, int64_t n, int32_t* out,
                               cudaStream_t st);
int group_csr_segment(int64_t nnz, int64_t G, int K);  // entries per segment
// segbase (G+1) = exclusive scan of ceil(row length / S); segcnt: G+1
// scratch; a null scan_tmp queries the scan's temporary bytes
cudaError_t launch_group_segments(const int64_t* rowptr, int64_t G, int S, int64_t* segcnt,
                                  int64_t* segbase, void* scan_tmp, size_t* scan_bytes,
                                  cudaStream_t st);
// hist: nsegs x K (nsegs = segbase[G]); ckey: the slice of every cell;
// cloc: slice << 16 | index within the slice (one gather per entry for the
// scatter); gent: GrpEnt entries
cudaError_t launch_group_csr(const int64_t* rowptr, const int32_t* col, const void* val, int val_u16,
                             int64_t G, const int64_t* segbase, int S, const int32_t* ckey,
                             const int32_t* cloc, int K, int32_t* hist, int64_t nsegs,
                             int64_t* gptr, void* gent, cudaStream_t st);

// ---- preparation kernels (kernels_prep.cu) ----
cudaError_t launch_dense_count(const void* Y, int is_f64, int cell_major, int64_t G, int64_t n,
                               int64_t* rowcnt, cudaStream_t st);
cudaError_t launch_dense_fill(const void* Y, int is_f64, int cell_major, int64_t G, int64_t n,
                              const int64_t* rowptr, int32_t* col, float* val, cudaStream_t st);
cudaError_t launch_csr_f64_to_f32(const double* in, float* out, int64_t nnz, cudaStream_t st);
cudaError_t launch_csc_keys(const int64_t* colptr, const int32_t* rowidx, int64_t n, int64_t G,
                            int64_t nnz, int64_t* keys, int32_t* bad, cudaStream_t st);
cudaError_t launch_keys_to_csr(const int64_t* keys, int64_t nnz, int64_t n, int64_t G,
                               int32_t* col, int64_t* rowcnt, cudaStream_t st);
cudaError_t launch_x_rowmajor(const double* Xcm, int64_t n, int P, int xs, float* Xrm,
                              cudaStream_t st);
cudaError_t launch_x_rowmajor_d(const double* Xcm, int64_t n, int P, int xs, double* Xrm,
                                cudaStream_t st);
cudaError_t launch_double_to_float(const double* in, float* out, int64_t m, cudaStream_t st);
// (order: the genes in the order the warps take them, largest first; null:
// gene order)
cudaError_t launch_gene_stats(const int64_t* rowptr, const void* val, int val_u16, int64_t G,
                              int64_t n, double* stats /* G x 6 */, cudaStream_t st,
                              const int32_t* order = nullptr);
// (colsum_u32, n: zeroed scratch of n cells; normed_sum of 16-bit counts
// then sums with 32-bit integer atomics)
cudaError_t launch_colstats(const int64_t* rowptr, const int32_t* col, const void* val,
                            int val_u16, int64_t G, int64_t nnz, double* colsum,
                            double* collog, int32_t* colcnt, int32_t* colmin_bits,
                            cudaStream_t st,
                            uint32_t* colsum_u32 = nullptr, int64_t n = 0);
cudaError_t launch_sf_finalize(int method, int64_t G, int64_t n, const double* colsum,
                               const double* collog, const int32_t* colcnt,
                               const int32_t* colmin_bits, double offset, double* sf,
                               double* off, float* off_f, int32_t* err, cudaStream_t st);
cudaError_t launch_sf_given(const double* sf_in, int64_t n, double offset, int use_sf, double* sf,
                            double* off, float* off_f, cudaStream_t st);
cudaError_t launch_theta0(const double* stats, const double* off, int64_t G, int64_t n,
                          int has_init, double init_value, double* theta0, float* k,
                          cudaStream_t st);
int xtx_blocks(int64_t n);  // partial-sum blocks launch_xtx_inverse needs
cudaError_t launch_xtx_inverse(const double* Xcm, int64_t n, int P, double* part, double* ginv,
                               int32_t* err, cudaStream_t st);
cudaError_t launch_init_beta(const int64_t* rowptr, const int32_t* col, const void* val,
                             int val_u16, const double* Xrm, int xs, const double* off,
                             double* inv_sf, const double* ginv, const double* stats, int64_t G,
                             int64_t n, int P, int rough, double* beta, float* beta_f,
                             cudaStream_t st);
cudaError_t launch_segptr(const int64_t* rowptr, const int32_t* col, int64_t G,
                          const int32_t* bound, int nbound, int64_t* segptr, cudaStream_t st);
cudaError_t launch_validate_csr(const int64_t* rowptr, const int32_t* col, int64_t G, int64_t n,
                                int64_t nnz, int32_t* bad, cudaStream_t st, const int32_t* order = nullptr);
cudaError_t launch_iota(int32_t* a, int64_t m, cudaStream_t st);
cudaError_t launch_pass_volume(const int64_t* rowptr, const int32_t* passes, int64_t G,
                               int64_t* acc, cudaStream_t st);
cudaError_t launch_fill_i32(int32_t* a, int32_t v, int64_t m, cudaStream_t st);
cudaError_t launch_mle_passes(const int32_t* it, const int32_t* phase, const double* stats,
                              int64_t G, int32_t* out, cudaStream_t st);
cudaError_t launch_set_i32(int32_t* a, int32_t v, cudaStream_t st);
// act_next = the genes g of act[0, n) (n = *n_act, or n_fixed when n_act is
// null) with keep[g] != 0, in order; *n_next = their count
// (wkey non-null: *n_heavy_next = the kept genes with wkey[g] >= thr;
// mirror non-null: the count also written there, a pinned mapped host slot)
cudaError_t launch_compact_kept(const int32_t* act, const int32_t* n_act, int64_t n_fixed, const int8_t* keep,
                                int32_t* act_next, int32_t* n_next, cudaStream_t st,
                                const int32_t* wkey = nullptr, int32_t thr = 0, int32_t* n_heavy_next = nullptr,
                                volatile int32_t* mirror = nullptr);
// *out = the number of leading entries of key (in descending order) >= thr
cudaError_t launch_count_at_least(const int32_t* key, int64_t n, int32_t thr, int32_t* out, cudaStream_t st);
cudaError_t launch_copy_i32_to_host_mapped(const int32_t* src, volatile int32_t* dst,
                                           cudaStream_t st);

// ---- finalize kernels (kernels_fin.cu) ----
// wide: partial sums are FP64 (generic engine) instead of FP32
cudaError_t launch_irls_finalize(const void* partW, bool wide, int nseg, int slot_stride, int P,
                                 const int32_t* act, const int32_t* n_act, int max_slots,
                                 int32_t* act_next, int32_t* n_next, double* beta, float* beta_f,
                                 int32_t* iters, int32_t* status, int max_iter, double eps,
                                 const float* k, cudaStream_t st);
// the IRLS step of the design-group engine's slice-major pass, the p x p
// assembly from geo.gsum folded in (geo.act / geo.n_act: this iteration's
// active genes)
// (keep non-null: keep[g] = 1 for the genes that go on, 0 for the others,
// and act_next / n_next untouched: launch_compact_kept lists them in order)
cudaError_t launch_grp_irls_finalize(const GrpGeom& geo, int max_slots, int32_t* act_next,
                                     int32_t* n_next, double* beta, float* beta_f, int32_t* iters,
                                     int32_t* status, int max_iter, double eps, const float* k,
                                     cudaStream_t st, int8_t* keep = nullptr);
cudaError_t launch_mom_finalize(const double* partS, int nseg, int slot_stride,
                                const int32_t* act, const int32_t* n_act, int max_slots,
                                int64_t n, int P, double* theta, cudaStream_t st);
struct MleState {
    double* x;       // current log theta to evaluate (pass reads it)
    double* lo;
    double* hi;
    int32_t* it;
    int32_t* phase;  // 0: far-left check pending, 1: Newton, 2: done
    double* theta;   // result
    double* dx;      // last step and the one before (bisection safeguard)
    double* dxold;
    const double* start_hint;  // optional per-gene start (MOM theta), may be null
    int8_t* keep = nullptr;    // non-null: keep[g] marks the genes that go on (launch_compact_kept
                               // lists them in order); null: appended to the next list
};
cudaError_t launch_mle_init(const double* stats, int64_t G, int64_t n, MleState s,
                            int32_t* act, int32_t* n_act, cudaStream_t st);
cudaError_t launch_mle_finalize(const void* partW, bool wide, const double* partS, int nseg,
                                int slot_stride, int P, const double* stats, int64_t n,
                                const int32_t* act, const int32_t* n_act, int max_slots,
                                int32_t* act_next, int32_t* n_next, MleState s, int max_iter,
                                int cox_reid, volatile int32_t* mirror, cudaStream_t st, int nA = 0,
                                const int32_t* colA = nullptr, const int32_t* colD = nullptr);
cudaError_t launch_sandwich_finalize(const double* partW, int nseg, int slot_stride, int P,
                                     const int32_t* seg_cluster, int n_clusters, int64_t n,
                                     const int32_t* act, const int32_t* n_act, int max_slots,
                                     double* bread, double* sandwich, double* meat,
                                     cudaStream_t st);

// ---- test kernels (kernels_test.cu) ----
cudaError_t launch_test_pvalues(int64_t G, int P, const double* beta, const double* bread,
                                const double* sandwich, double df, const double* contrast_dev,
                                double max_lfc, double* pval, double* lfc, cudaStream_t st);
// p.adjust with temp storage from the caller (bytes from p_adjust_temp_bytes)
size_t p_adjust_temp_bytes(int64_t m);
cudaError_t launch_p_adjust(int64_t m, const double* p, int method, double* out, void* temp,
                            size_t temp_bytes, cudaStream_t st);
cudaError_t launch_nb_adjoint(int64_t n, const double* y, const double* eta, double log_theta,
                              double* ll, double* d_eta, double* d_lt, cudaStream_t st);

}  // namespace devil
