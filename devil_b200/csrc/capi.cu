// C-ABI of the devil B200 path: context, uploads, the fit pipeline in the
// order of cpu_fit (R/main.R:375-523), the DE test and the single-step
// entry points.  See include/devil_b200.h for the contract.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <thread>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/devil_b200.h"
#include "internal.h"

using namespace devil;

namespace devil {
cudaError_t raise_dyn_smem_raw(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> cap;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = cap[{func, dev}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// resident blocks per SM of the kernel a pass would launch, from the CUDA
// occupancy calculator; cached per configuration (all contexts, all threads)
int pass_blocks_per_sm(PassKind kind, Engine engine, int P, int GT, int val_u16, int plain) {
    static std::mutex mu;
    static std::map<int64_t, int> cache;
    const int64_t key =
        (((((int64_t)kind * 8 + engine) * 64 + P) * 512 + GT) * 2 + (val_u16 ? 1 : 0)) * 2 + (plain ? 1 : 0);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    PassLaunch L{};
    L.kind = kind;
    L.engine = engine;
    L.P = P;
    L.xs_pad = P <= 8 ? (P <= 1 ? 1 : (P <= 2 ? 2 : (P <= 4 ? 4 : 8))) : (P + 3) & ~3;
    L.GT = GT;
    L.val_u16 = val_u16;
    L.nseg = 1;
    L.ntiles = 1;
    L.plain = plain;
    int occ = 0;
    L.occ_out = &occ;
    cudaError_t e = cudaErrorInvalidValue;
    if (engine == ENGINE_REG) e = launch_reg_pass(L);
    else if (engine == ENGINE_GEN) e = launch_gen_pass(L);
    else if (engine == ENGINE_TC) e = launch_tc_pass(L, nullptr);
    else if (engine == ENGINE_TCW) e = launch_tcw_pass(L, TcwGeom{});
    if (e != cudaSuccess || occ < 1) {
        cudaGetLastError();  // a failed query leaves no sticky error; use one block per SM
        occ = 1;
    }
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = occ;
    return occ;
}
}  // namespace devil

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct devil_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int64_t launches = 0;
    std::map<std::string, DevBuf> bufs;
    int32_t* mapped_host = nullptr;   // pinned, mapped: active-gene count mirrors, one slot per
    int32_t* mapped_dev = nullptr;    // loop iteration mod 4
    int64_t mapped_host_at(int t) const { return *(volatile int32_t*)(mapped_host + (t & 3)); }
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int sm_count = 148;
    int use_tma = 0;
    int use_groups = 1;
    // slice-major passes of the design-group engine, a bit mask: 1 IRLS, 2 MLE,
    // 4 MOM, 8 bread (unclustered) (DEVIL_GRP_SLICES; 0: every pass block per gene)
    int grp_slices = 15;
    int debug = 0;  // DEVIL_DEBUG=1: engine choices on stderr
    // profiling: CUDA events around every pass launch, per pass kind
    int profiling = 0;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    struct Rec { int kind; size_t e0, e1; };
    std::vector<Rec> recs;
    int64_t prof_launches[4] = {0, 0, 0, 0};
    double prof_ms[4] = {0, 0, 0, 0};
    double prof_bytes[4] = {0, 0, 0, 0};
    double prof_tc_flops[4] = {0, 0, 0, 0};  // tensor-core FLOPs issued (MMA shapes, padding included)
    int64_t irls_rescued = 0;                 // genes the last fit refitted on the CUDA-core engine
    int last_engine[4] = {-1, -1, -1, -1};
    // DEVIL_DEBUG: CUDA events at the phase boundaries of a fit
    std::vector<std::pair<const char*, cudaEvent_t>> marks;
};

namespace {

struct Fail {
    int code;
};

void set_err(devil_ctx* ctx, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
}

#define CK(expr)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (expr);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            set_err(ctx, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_),        \
                    __FILE__, __LINE__);                                                \
            throw Fail{e_ == cudaErrorMemoryAllocation ? DEVIL_ERR_NOMEM : DEVIL_ERR_CUDA}; \
        }                                                                               \
    } while (0)

#define LAUNCH(expr)            \
    do {                        \
        CK(expr);               \
        ctx->launches++;        \
    } while (0)

void fail(devil_ctx* ctx, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
    throw Fail{code};
}

// grow-only named device workspace
template <class T>
T* ws(devil_ctx* ctx, const std::string& name, size_t count) {
    size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    DevBuf& b = ctx->bufs[name];
    if (b.bytes < bytes) {
        if (b.p) CK(cudaFree(b.p));
        b.p = nullptr;
        b.bytes = 0;
        CK(cudaMalloc(&b.p, bytes));
        b.bytes = bytes;
    }
    return static_cast<T*>(b.p);
}

size_t prof_event(devil_ctx* ctx) {
    if (ctx->ev_used == ctx->ev_pool.size()) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        ctx->ev_pool.push_back(e);
    }
    size_t i = ctx->ev_used++;
    CK(cudaEventRecord(ctx->ev_pool[i], ctx->stream));
    return i;
}

// fold recorded event pairs into the per-kind totals (synchronizes)
void prof_collect(devil_ctx* ctx) {
    if (!ctx->profiling || ctx->recs.empty()) {
        ctx->ev_used = 0;
        return;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    for (auto& r : ctx->recs) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->ev_pool[r.e0], ctx->ev_pool[r.e1]));
        ctx->prof_ms[r.kind] += ms;
        ctx->prof_launches[r.kind] += 1;
    }
    ctx->recs.clear();
    ctx->ev_used = 0;
}

// phase marks of a fit (DEVIL_DEBUG=1); dbg_report prints the gaps
void dbg_mark(devil_ctx* ctx, const char* label) {
    if (!ctx->debug) return;
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    CK(cudaEventRecord(e, ctx->stream));
    ctx->marks.emplace_back(label, e);
}
void dbg_report(devil_ctx* ctx) {
    if (!ctx->debug || ctx->marks.empty()) return;
    CK(cudaStreamSynchronize(ctx->stream));
    std::string out = "devil_b200 phases (ms):";
    for (size_t i = 1; i < ctx->marks.size(); ++i) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->marks[i - 1].second, ctx->marks[i].second));
        char buf[96];
        snprintf(buf, sizeof buf, " %s %.2f", ctx->marks[i].first, ms);
        out += buf;
    }
    for (auto& m : ctx->marks) cudaEventDestroy(m.second);
    ctx->marks.clear();
    fprintf(stderr, "%s\n", out.c_str());
}

template <class T>
void h2d(devil_ctx* ctx, T* dst, const T* src, size_t count) {
    if (count) CK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
}
template <class T>
void d2h(devil_ctx* ctx, T* dst, const T* src, size_t count) {
    if (count && dst) CK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
}

// ------------------------------------------------------------------
// device-resident problem
// ------------------------------------------------------------------
struct DevProblem {
    int64_t G = 0, n = 0;
    int P = 0;
    int xs = 0;
    int val_u16 = 0;
    const int64_t* rowptr = nullptr;
    const int32_t* col = nullptr;
    const void* val = nullptr;
    int64_t nnz = 0;
    const double* Xcm = nullptr;
    float* Xrm = nullptr;
    // products image of the tensor-core IRLS engine (p <= 4), built by its
    // first launch
    mutable float4* zimg = nullptr;
    // inputs of the tensor-core IRLS engine for p = 5..32 (dense count
    // image, feature rows, padded offsets), built by its first launch
    mutable TcwGeom tcw;
    mutable bool tcw_ready = false;
    mutable int tcw_fits = -1;  // the dense count image fits half of the free device memory (-1: not asked)
    int precision = DEVIL_PREC_FP32;  // DEVIL_PREC_*: tensor-core passes at p <= 4
    double* Xdrm = nullptr;  // row-major FP64 copy for the FP64 passes
    double* sf = nullptr;
    double* off = nullptr;
    float* off_f = nullptr;
    double* stats = nullptr;
    // genes by decreasing entry count (sorted once per fit, right after the
    // counts arrive): the order in which warp-per-gene kernels take the
    // genes (the largest first, so they do not set the kernel's length) and
    // the work order of the slice-major passes
    int32_t* gorder = nullptr;
    int32_t* gwkey = nullptr;  // [G] entries of every gene
    int32_t* gskey = nullptr;  // [G] the same in gorder (descending)
    int nfine = 1;
    int32_t* fine_bound = nullptr;
    int64_t* fine_ptr = nullptr;
    // design groups (kernels_grp.cu); active only for the chosen form
    struct Groups {
        bool active = false;
        int U = 0, C = 1;
        double* xg = nullptr;
        double* E = nullptr;
        int S = 0;                    // slices
        void* gent = nullptr;         // slice-ordered CSR copy (GrpEnt entries)
        int64_t* gptr = nullptr;      // [G][S + 1]
        int32_t *sl_start = nullptr, *sl_key = nullptr, *kslice = nullptr;
        double* rs = nullptr;
        double* rw = nullptr;
        int32_t* rm = nullptr;
        double* res = nullptr;
        // sparse design rows and the assembly's (group, weight) lists
        int32_t *rptr = nullptr, *rcol = nullptr, *qptr = nullptr, *qu = nullptr, *vptr = nullptr,
                *vu = nullptr;
        int nA = 0;  // exclusive-column structure (GrpGeom)
        int32_t *colA = nullptr, *colD = nullptr, *colpos = nullptr;
        int n_need = 0;
        int32_t *need_q = nullptr, *need_d = nullptr;
        double *rval = nullptr, *qv = nullptr, *vv = nullptr;
        int32_t* order = nullptr;  // genes by decreasing entry count (the passes' work order)
        int32_t* wkey = nullptr;   // [G] entries of every gene
        int32_t* skey = nullptr;   // [G] the same in the work order (descending)
    } grp;
};

int xs_for(int P) {
    if (P <= 8) return P <= 1 ? 1 : (P <= 2 ? 2 : (P <= 4 ? 4 : 8));
    return (P + 3) & ~3;
}

void check_counts(devil_ctx* ctx, const devil_counts* c) {
    if (!c) fail(ctx, DEVIL_ERR_ARG, "counts is NULL");
    if (c->n_genes < 0 || c->n_cells < 2) fail(ctx, DEVIL_ERR_ARG, "need n_genes >= 0 and n_cells >= 2");
    if (c->n_cells > INT32_MAX) fail(ctx, DEVIL_ERR_ARG, "n_cells must fit int32");
    if (c->n_genes > INT32_MAX) fail(ctx, DEVIL_ERR_ARG, "n_genes must fit int32");
    if (c->format < 0 || c->format > 4) fail(ctx, DEVIL_ERR_ARG, "unknown counts format %d", c->format);
    if (c->n_genes > 0 && c->n_cells > 0 && !c->values && c->nnz != 0)
        fail(ctx, DEVIL_ERR_ARG, "counts values is NULL");
}

// every kernel indexes the design with CSR cell indices: check them first
void gene_order(devil_ctx* ctx, DevProblem& dp) {
    cudaStream_t st = ctx->stream;
    const int64_t G = dp.G;
    dp.gorder = dp.gwkey = dp.gskey = nullptr;
    if (G <= 0) return;
    int32_t* idx = ws<int32_t>(ctx, "ord_idx", G);
    dp.gwkey = ws<int32_t>(ctx, "ord_key", G);
    dp.gskey = ws<int32_t>(ctx, "ord_key_sorted", G);
    dp.gorder = ws<int32_t>(ctx, "ord_genes", G);
    // (row lengths clamped to [0, INT32_MAX]: a malformed row pointer gives a
    // meaningless order, and the check below rejects the call)
    LAUNCH(launch_gene_entries(dp.rowptr, G, dp.gwkey, idx, st));
    size_t ob = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, ob, dp.gwkey, dp.gskey, idx, dp.gorder, (int)G);
    CK(cub::DeviceRadixSort::SortPairsDescending(ws<char>(ctx, "ord_tmp", ob), ob, dp.gwkey, dp.gskey, idx,
                                                 dp.gorder, (int)G, 0, 32, st));
    ctx->launches++;
}

void validate_csr(devil_ctx* ctx, DevProblem& dp) {
    gene_order(ctx, dp);
    int32_t* bad = ws<int32_t>(ctx, "csr_bad", 1);
    CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), ctx->stream));
    LAUNCH(launch_validate_csr(dp.rowptr, dp.col, dp.G, dp.n, dp.nnz, bad, ctx->stream, dp.gorder));
    int32_t h = 0;
    CK(cudaMemcpyAsync(&h, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h)
        fail(ctx, DEVIL_ERR_ARG,
             "invalid CSR: row pointers must be non-decreasing and end at nnz, cell indices in "
             "[0, n) and strictly increasing within each gene");
}

// upload host counts to a device CSR (gene-major)
void upload_counts(devil_ctx* ctx, const devil_counts* c, DevProblem& dp) {
    const int64_t G = c->n_genes, n = c->n_cells;
    dp.G = G;
    dp.n = n;
    cudaStream_t st = ctx->stream;
    switch (c->format) {
        case DEVIL_COUNTS_CSR_U16:
        case DEVIL_COUNTS_CSR_F32: {
            if (!c->ptr || (!c->idx && c->nnz)) fail(ctx, DEVIL_ERR_ARG, "CSR needs ptr and idx");
            int64_t nnz = c->ptr[G];
            if (nnz != c->nnz) fail(ctx, DEVIL_ERR_ARG, "CSR nnz mismatch (%lld vs rowptr %lld)",
                                    (long long)c->nnz, (long long)nnz);
            int64_t* rp = ws<int64_t>(ctx, "rowptr", G + 1);
            int32_t* col = ws<int32_t>(ctx, "col", nnz);
            h2d(ctx, rp, c->ptr, G + 1);
            h2d(ctx, col, c->idx, nnz);
            if (c->format == DEVIL_COUNTS_CSR_U16) {
                uint16_t* v = ws<uint16_t>(ctx, "val16", nnz);
                h2d(ctx, v, static_cast<const uint16_t*>(c->values), nnz);
                dp.val = v;
                dp.val_u16 = 1;
            } else {
                float* v = ws<float>(ctx, "val32", nnz);
                h2d(ctx, v, static_cast<const float*>(c->values), nnz);
                dp.val = v;
                dp.val_u16 = 0;
            }
            dp.rowptr = rp;
            dp.col = col;
            dp.nnz = nnz;
            validate_csr(ctx, dp);
            return;
        }
        case DEVIL_COUNTS_DENSE_F64:
        case DEVIL_COUNTS_DENSE_F32: {
            const int is64 = c->format == DEVIL_COUNTS_DENSE_F64;
            const size_t esz = is64 ? 8 : 4;
            void* Yd = ws<char>(ctx, "dense", (size_t)G * n * esz);
            if (G * n) CK(cudaMemcpyAsync(Yd, c->values, (size_t)G * n * esz, cudaMemcpyHostToDevice, st));
            int64_t* cnt = ws<int64_t>(ctx, "rowcnt", G + 1);
            CK(cudaMemsetAsync(cnt, 0, (G + 1) * sizeof(int64_t), st));
            LAUNCH(launch_dense_count(Yd, is64, c->dense_layout == DEVIL_DENSE_CELL_MAJOR, G, n, cnt, st));
            int64_t* rp = ws<int64_t>(ctx, "rowptr", G + 1);
            size_t tb = 0;
            cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, rp, (int)(G + 1), st);
            void* tmp = ws<char>(ctx, "scan_tmp", tb);
            CK(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, rp, (int)(G + 1), st));
            ctx->launches++;
            int64_t nnz = 0;
            CK(cudaMemcpyAsync(&nnz, rp + G, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            int32_t* col = ws<int32_t>(ctx, "col", nnz);
            float* v = ws<float>(ctx, "val32", nnz);
            LAUNCH(launch_dense_fill(Yd, is64, c->dense_layout == DEVIL_DENSE_CELL_MAJOR, G, n, rp, col, v, st));
            dp.rowptr = rp;
            dp.col = col;
            dp.val = v;
            dp.val_u16 = 0;
            dp.nnz = nnz;
            return;
        }
        case DEVIL_COUNTS_CSC_F64: {
            if (!c->ptr || (!c->idx && c->nnz)) fail(ctx, DEVIL_ERR_ARG, "CSC needs ptr and idx");
            int64_t nnz = c->ptr[n];
            if (nnz != c->nnz) fail(ctx, DEVIL_ERR_ARG, "CSC nnz mismatch");
            int64_t* cp = ws<int64_t>(ctx, "colptr", n + 1);
            int32_t* ri = ws<int32_t>(ctx, "rowidx", nnz);
            double* vin = ws<double>(ctx, "csc_val", nnz);
            h2d(ctx, cp, c->ptr, n + 1);
            h2d(ctx, ri, c->idx, nnz);
            h2d(ctx, vin, static_cast<const double*>(c->values), nnz);
            int64_t* keys = ws<int64_t>(ctx, "keys", nnz);
            int64_t* keys2 = ws<int64_t>(ctx, "keys2", nnz);
            double* v2 = ws<double>(ctx, "csc_val2", nnz);
            int32_t* bad = ws<int32_t>(ctx, "csr_bad", 1);
            CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
            LAUNCH(launch_csc_keys(cp, ri, n, G, nnz, keys, bad, st));
            int32_t hbad = 0;
            CK(cudaMemcpyAsync(&hbad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (hbad) fail(ctx, DEVIL_ERR_ARG, "invalid CSC: pointers or gene indices out of range");
            size_t tb = 0;
            cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, vin, v2, (int)nnz);
            void* tmp = ws<char>(ctx, "sort_tmp", tb);
            CK(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, vin, v2, (int)nnz, 0, 64, st));
            ctx->launches++;
            int32_t* col = ws<int32_t>(ctx, "col", nnz);
            int64_t* cnt = ws<int64_t>(ctx, "rowcnt", G + 1);
            CK(cudaMemsetAsync(cnt, 0, (G + 1) * sizeof(int64_t), st));
            LAUNCH(launch_keys_to_csr(keys2, nnz, n, G, col, cnt, st));
            int64_t* rp = ws<int64_t>(ctx, "rowptr", G + 1);
            size_t tb2 = 0;
            cub::DeviceScan::ExclusiveSum(nullptr, tb2, cnt, rp, (int)(G + 1), st);
            void* tmp2 = ws<char>(ctx, "scan_tmp", tb2);
            CK(cub::DeviceScan::ExclusiveSum(tmp2, tb2, cnt, rp, (int)(G + 1), st));
            ctx->launches++;
            float* v = ws<float>(ctx, "val32", nnz);
            LAUNCH(launch_csr_f64_to_f32(v2, v, nnz, st));
            dp.rowptr = rp;
            dp.col = col;
            dp.val = v;
            dp.val_u16 = 0;
            dp.nnz = nnz;
            return;
        }
    }
    fail(ctx, DEVIL_ERR_ARG, "unsupported counts format");
}

void use_device_counts(devil_ctx* ctx, const devil_counts* c, DevProblem& dp) {
    if (c->format != DEVIL_COUNTS_CSR_U16 && c->format != DEVIL_COUNTS_CSR_F32)
        fail(ctx, DEVIL_ERR_ARG, "device counts must be CSR (uint16 or float)");
    dp.G = c->n_genes;
    dp.n = c->n_cells;
    dp.rowptr = c->ptr;
    dp.col = c->idx;
    dp.val = c->values;
    dp.val_u16 = c->format == DEVIL_COUNTS_CSR_U16;
    dp.nnz = c->nnz;
    validate_csr(ctx, dp);
}

// design, segmentation, statistics
void prepare_design(devil_ctx* ctx, DevProblem& dp, const double* X, int P, bool X_on_device) {
    if (P < 1 || P > 32) fail(ctx, DEVIL_ERR_UNSUPPORTED, "p = %d outside 1..32", P);
    if (dp.n <= P) fail(ctx, DEVIL_ERR_ARG, "need more cells than design columns");
    dp.P = P;
    dp.xs = xs_for(P);
    cudaStream_t st = ctx->stream;
    if (X_on_device) {
        dp.Xcm = X;
    } else {
        double* xd = ws<double>(ctx, "Xcm", (size_t)dp.n * P);
        h2d(ctx, xd, X, (size_t)dp.n * P);
        dp.Xcm = xd;
    }
    // 16 padding rows: TMA copies of the last chunk round up to 4 cells
    dp.Xrm = ws<float>(ctx, "Xrm", (size_t)(dp.n + 16) * dp.xs);
    CK(cudaMemsetAsync(dp.Xrm + (size_t)dp.n * dp.xs, 0, (size_t)16 * dp.xs * sizeof(float), st));
    LAUNCH(launch_x_rowmajor(dp.Xcm, dp.n, P, dp.xs, dp.Xrm, st));
    dp.Xdrm = ws<double>(ctx, "Xdrm", (size_t)dp.n * dp.xs);
    LAUNCH(launch_x_rowmajor_d(dp.Xcm, dp.n, P, dp.xs, dp.Xdrm, st));
    // fine segmentation: chunks of CH cells (a multiple of 16), the unit
    // the TMA engine stages; work items are runs of consecutive chunks
    const int CH = tma_chunk_cells(dp.xs);
    const int nf = (int)((dp.n + CH - 1) / CH);
    dp.nfine = nf;
    std::vector<int32_t> hb(nf + 1);
    for (int s = 0; s <= nf; ++s) hb[s] = (int32_t)std::min<int64_t>(dp.n, (int64_t)s * CH);
    dp.fine_bound = ws<int32_t>(ctx, "fine_bound", nf + 1);
    h2d(ctx, dp.fine_bound, hb.data(), nf + 1);
    dp.fine_ptr = ws<int64_t>(ctx, "fine_ptr", (size_t)dp.G * (nf + 1));
    LAUNCH(launch_segptr(dp.rowptr, dp.col, dp.G, dp.fine_bound, nf + 1, dp.fine_ptr, st));
    dp.stats = ws<double>(ctx, "stats", (size_t)dp.G * 6);
    LAUNCH(launch_gene_stats(dp.rowptr, dp.val, dp.val_u16, dp.G, dp.n, dp.stats, st, dp.gorder));
    CK(cudaStreamSynchronize(st));  // host copies above must stay valid until here
}

// whether the wide tensor-core engine's dense count image fits half of the
// free device memory (asked once per fit, and only where that engine could
// run: the query costs milliseconds on a busy device)
bool tcw_fits(const DevProblem& dp) {
    if (dp.tcw_fits < 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
        const double need = (double)dp.G * tcw_npad(dp.n) * (dp.val_u16 ? 2.0 : 4.0) +
                            (double)(dp.xs + 1) * tcw_npad(dp.n) * 4.0;
        dp.tcw_fits = need <= 0.5 * (double)fr ? 1 : 0;
    }
    return dp.tcw_fits == 1;
}

// size factors and offsets (R/main.R:224-230, R/size_factors.R)
void compute_offsets(devil_ctx* ctx, DevProblem& dp, int method, const double* sf_given_host,
                     const double* sf_given_dev, double offset) {
    cudaStream_t st = ctx->stream;
    const int64_t n = dp.n;
    dp.sf = ws<double>(ctx, "sf", n);
    dp.off = ws<double>(ctx, "off", n);
    dp.off_f = ws<float>(ctx, "off_f", n + 16);
    CK(cudaMemsetAsync(dp.off_f + n, 0, 16 * sizeof(float), st));
    if (method == DEVIL_SF_NONE) {
        LAUNCH(launch_sf_given(nullptr, n, offset, 0, dp.sf, dp.off, dp.off_f, st));
        return;
    }
    if (method == DEVIL_SF_GIVEN) {
        const double* src = sf_given_dev;
        if (!src) {
            if (!sf_given_host) fail(ctx, DEVIL_ERR_ARG, "size factors not given");
            double* t = ws<double>(ctx, "sf_in", n);
            h2d(ctx, t, sf_given_host, n);
            src = t;
        }
        LAUNCH(launch_sf_given(src, n, offset, 1, dp.sf, dp.off, dp.off_f, st));
        return;
    }
    if (method != DEVIL_SF_NORMED_SUM && method != DEVIL_SF_PSINORM)
        fail(ctx, DEVIL_ERR_ARG, "unknown size factor method %d", method);
    double* colsum = ws<double>(ctx, "colsum", n);
    CK(cudaMemsetAsync(colsum, 0, n * sizeof(double), st));
    double* collog = nullptr;
    int32_t *colcnt = nullptr, *colmin = nullptr;
    if (method == DEVIL_SF_PSINORM) {
        collog = ws<double>(ctx, "collog", n);
        colcnt = ws<int32_t>(ctx, "colcnt", n);
        colmin = ws<int32_t>(ctx, "colmin", n);
        CK(cudaMemsetAsync(collog, 0, n * sizeof(double), st));
        CK(cudaMemsetAsync(colcnt, 0, n * sizeof(int32_t), st));
        CK(cudaMemsetAsync(colmin, 0x7f, n * sizeof(int32_t), st));  // ~ +3.4e38
    }
    uint32_t* colsum_u32 = nullptr;
    if (method == DEVIL_SF_NORMED_SUM && dp.val_u16 && dp.G <= 65537) {
        colsum_u32 = ws<uint32_t>(ctx, "colsum_u32", n);
        CK(cudaMemsetAsync(colsum_u32, 0, n * sizeof(uint32_t), st));
    }
    LAUNCH(launch_colstats(dp.rowptr, dp.col, dp.val, dp.val_u16, dp.G, dp.nnz, colsum, collog,
                           colcnt, colmin, st, colsum_u32, n));
    int32_t* err = ws<int32_t>(ctx, "sf_err", 1);
    LAUNCH(launch_sf_finalize(method == DEVIL_SF_NORMED_SUM ? 1 : 2, dp.G, n, colsum, collog, colcnt,
                              colmin, offset, dp.sf, dp.off, dp.off_f, err, st));
    int32_t herr = 0;
    CK(cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr)
        fail(ctx, DEVIL_ERR_ZERO_COLUMN,
             "At least one column (sample) contains all zeros, unable to compute size factor. "
             "Please filter out empty samples from input matrix.");
}

// ------------------------------------------------------------------
// design groups: distinct design rows (x cluster) of the cells, their
// Gauss rules and the CSR copy ordered by group (kernels_grp.cu).  Used
// when the rows take at most kMaxGroups values and the rules are smaller
// than the cells; otherwise, or when a rule fails its check, the passes
// stay on the per-cell engines.
// ------------------------------------------------------------------
void build_groups(devil_ctx* ctx, DevProblem& dp, const int32_t* ends_host, int n_clusters, int form) {
    dp.grp = DevProblem::Groups{};
    if (form != DEVIL_FORM_CHOSEN || !ctx->use_groups || dp.G == 0) return;
    if (n_clusters > 1 && !ends_host) fail(ctx, DEVIL_ERR_ARG, "cluster_ends is NULL");
    cudaStream_t st = ctx->stream;
    const int64_t n = dp.n;
    const int P = dp.P;
    uint64_t* hk = ws<uint64_t>(ctx, "grp_hash", n);
    uint64_t* hk2 = ws<uint64_t>(ctx, "grp_hash2", n);
    int32_t* ix = ws<int32_t>(ctx, "grp_idx", n);
    int32_t* ix2 = ws<int32_t>(ctx, "grp_idx2", n);
    LAUNCH(launch_row_hash(dp.Xcm, n, P, hk, ix, st));
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, hk, hk2, ix, ix2, (int)n);
    CK(cub::DeviceRadixSort::SortPairs(ws<char>(ctx, "grp_sort_tmp", tb), tb, hk, hk2, ix, ix2,
                                       (int)n, 0, 64, st));
    ctx->launches++;
    int32_t* flag = ws<int32_t>(ctx, "grp_flag", n);
    int32_t* incl = ws<int32_t>(ctx, "grp_incl", n);
    int32_t* bad = ws<int32_t>(ctx, "grp_bad", 2);
    CK(cudaMemsetAsync(bad, 0, 2 * sizeof(int32_t), st));
    LAUNCH(launch_group_heads(dp.Xcm, n, P, hk2, ix2, flag, bad, st));
    tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, flag, incl, (int)n);
    CK(cub::DeviceScan::InclusiveSum(ws<char>(ctx, "grp_scan_tmp", tb), tb, flag, incl, (int)n, st));
    ctx->launches++;
    int32_t h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, incl + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h + 1, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int U = h[0];
    if (h[1] || U < 1 || U > kMaxGroups || (int64_t)U * kMinCellsPerGroup >= n) {
        if (ctx->debug)
            fprintf(stderr, "devil_b200: design not grouped (%d distinct rows%s)\n", U,
                    h[1] ? ", hash collision" : "");
        return;
    }
    dbg_mark(ctx, "g.rows");
    const int C = (n_clusters > 1 && (int64_t)U * n_clusters <= kMaxFine) ? n_clusters : 1;
    const int K = U * C;
    int32_t* ucell = ws<int32_t>(ctx, "grp_ucell", n);
    int32_t* head = ws<int32_t>(ctx, "grp_head", U);
    LAUNCH(launch_group_assign(ix2, incl, flag, n, ucell, head, st));
    double* xg = ws<double>(ctx, "grp_xg", (size_t)U * P);
    LAUNCH(launch_group_rows(dp.Xcm, n, P, head, U, xg, st));
    // fine keys u * C + cluster
    int32_t* ends_d = ws<int32_t>(ctx, "grp_ends", std::max(1, C));
    if (C > 1) {
        for (int b = 0; b < C; ++b) {
            const int64_t prev = b ? ends_host[b - 1] : 0;
            if (ends_host[b] < prev || ends_host[b] > n)
                fail(ctx, DEVIL_ERR_ARG, "cluster ends must be non-decreasing and <= n");
        }
        if (ends_host[C - 1] != n) fail(ctx, DEVIL_ERR_ARG, "last cluster end must equal the number of cells");
        h2d(ctx, ends_d, ends_host, C);
    }
    int32_t* fkey = ws<int32_t>(ctx, "grp_fkey", n);
    int32_t* cells = ix;  // reuse
    LAUNCH(launch_fine_keys(ucell, ends_d, C, n, fkey, cells, st));
    auto bits_for = [](int K) {
        int b = 1;
        while ((1 << b) < K) ++b;
        return b;
    };
    // the cells renumbered in key order (stable: original order within a
    // key), so that every key is a contiguous range of the new numbering
    int32_t* pnew = ws<int32_t>(ctx, "grp_pnew", n);
    int32_t* ksorted = ws<int32_t>(ctx, "grp_ksorted", n);
    int64_t* kst = ws<int64_t>(ctx, "grp_kst", K + 1);
    tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, fkey, ksorted, cells, pnew, (int)n, 0, bits_for(K));
    CK(cub::DeviceRadixSort::SortPairs(ws<char>(ctx, "grp_sort_tmp0", tb), tb, fkey, ksorted, cells,
                                       pnew, (int)n, 0, bits_for(K), st));
    ctx->launches++;
    LAUNCH(launch_group_starts(ksorted, n, K, kst, st));
    // cells by offset, then (stable) by group and by fine group: each
    // group's cells sorted by offset, as the rules need
    double* offs = ws<double>(ctx, "grp_offs", n);
    int32_t* byoff = ws<int32_t>(ctx, "grp_byoff", n);
    tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, dp.off, offs, cells, byoff, (int)n);
    CK(cub::DeviceRadixSort::SortPairs(ws<char>(ctx, "grp_sort_tmp", tb), tb, dp.off, offs, cells,
                                       byoff, (int)n, 0, 64, st));
    ctx->launches++;
    int32_t* kin = ws<int32_t>(ctx, "grp_kin", n);
    int32_t* kout = ws<int32_t>(ctx, "grp_kout", n);
    int32_t* permC = ws<int32_t>(ctx, "grp_permC", n);
    int64_t* gsC = ws<int64_t>(ctx, "grp_gsC", U + 1);
    LAUNCH(launch_gather_keys(ucell, byoff, n, kin, st));
    tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, byoff, permC, (int)n, 0, bits_for(U));
    CK(cub::DeviceRadixSort::SortPairs(ws<char>(ctx, "grp_sort_tmp2", tb), tb, kin, kout, byoff, permC,
                                       (int)n, 0, bits_for(U), st));
    ctx->launches++;
    LAUNCH(launch_group_starts(kout, n, U, gsC, st));
    int32_t* permF = permC;
    int64_t* gsF = gsC;
    if (C > 1) {
        permF = ws<int32_t>(ctx, "grp_permF", n);
        gsF = ws<int64_t>(ctx, "grp_gsF", K + 1);
        LAUNCH(launch_gather_keys(fkey, byoff, n, kin, st));
        tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, byoff, permF, (int)n, 0, bits_for(K));
        CK(cub::DeviceRadixSort::SortPairs(ws<char>(ctx, "grp_sort_tmp3", tb), tb, kin, kout, byoff,
                                           permF, (int)n, 0, bits_for(K), st));
        ctx->launches++;
        LAUNCH(launch_group_starts(kout, n, K, gsF, st));
    }
    dbg_mark(ctx, "g.sort");
    // slices: each key's range cut into pieces of at most kSliceCells cells
    std::vector<int64_t> hks(K + 1);
    CK(cudaMemcpyAsync(hks.data(), kst, (K + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<int32_t> sl_start{0}, sl_key, kslice(K + 1);
    for (int k = 0; k < K; ++k) {
        kslice[k] = (int32_t)sl_key.size();
        const int64_t a = hks[k], cnt = hks[k + 1] - hks[k];
        const int64_t pieces = (cnt + kSliceCells - 1) / kSliceCells;
        for (int64_t q = 1; q <= pieces; ++q) {
            sl_start.push_back((int32_t)(a + cnt * q / pieces));
            sl_key.push_back(k);
        }
    }
    kslice[K] = (int32_t)sl_key.size();
    const int NSL = (int)sl_key.size();
    if (NSL < 1 || NSL > kMaxSlices) {
        if (ctx->debug) fprintf(stderr, "devil_b200: design not grouped (%d slices)\n", NSL);
        return;
    }
    int32_t* d_sl_start = ws<int32_t>(ctx, "grp_sl_start", NSL + 1);
    int32_t* d_sl_key = ws<int32_t>(ctx, "grp_sl_key", NSL);
    int32_t* d_kslice = ws<int32_t>(ctx, "grp_kslice", K + 1);
    h2d(ctx, d_sl_start, sl_start.data(), NSL + 1);
    h2d(ctx, d_sl_key, sl_key.data(), NSL);
    h2d(ctx, d_kslice, kslice.data(), K + 1);
    int32_t* cslice = ws<int32_t>(ctx, "grp_cslice", n);
    int32_t* cloc = ws<int32_t>(ctx, "grp_cloc", n);
    double* E = ws<double>(ctx, "grp_E", n);  // exp(offset) in slice order
    LAUNCH(launch_slice_cells(pnew, d_sl_start, NSL, n, dp.off, cslice, cloc, E, st));
    const int nrules = U + (C > 1 ? K : 0);
    double* rs = ws<double>(ctx, "grp_rs", (size_t)nrules * kRuleCap);
    double* rw = ws<double>(ctx, "grp_rw", (size_t)nrules * kRuleCap);
    int32_t* rm = ws<int32_t>(ctx, "grp_rm", nrules);
    double* scr = ws<double>(ctx, "grp_scr", (size_t)6 * n);
    double* rerr = ws<double>(ctx, "grp_rerr", nrules);
    LAUNCH(launch_group_rules(permC, gsC, permF, gsF, U, nrules, dp.off, n, scr, rs, rw, rm, rerr,
                              bad + 1, st));
    dbg_mark(ctx, "g.rules");
    // CSR copy ordered by slice within each gene: 4-byte entries (index in
    // the slice, 16-bit count) or 8-byte ones for float counts
    // (padded to a whole 16-byte group: the pass reads the groups covering a range)
    void* gent = ws<char>(ctx, "grp_ent", (size_t)(dp.nnz + 4) * (dp.val_u16 ? 4 : 8));
    int64_t* gptr = ws<int64_t>(ctx, "grp_ptr", (size_t)dp.G * (NSL + 1));
    const int S = group_csr_segment(dp.nnz, dp.G, NSL);
    int64_t* segcnt = ws<int64_t>(ctx, "grp_segcnt", dp.G + 1);
    int64_t* segbase = ws<int64_t>(ctx, "grp_segbase", dp.G + 1);
    size_t sb = 0;
    CK(launch_group_segments(dp.rowptr, dp.G, S, segcnt, segbase, nullptr, &sb, st));
    LAUNCH(launch_group_segments(dp.rowptr, dp.G, S, segcnt, segbase, ws<char>(ctx, "grp_seg_tmp", sb),
                                 &sb, st));
    int64_t nsegs = 0;
    CK(cudaMemcpyAsync(&nsegs, segbase + dp.G, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int32_t* hist = ws<int32_t>(ctx, "grp_hist", (size_t)std::max<int64_t>(nsegs, 1) * NSL);
    LAUNCH(launch_group_csr(dp.rowptr, dp.col, dp.val, dp.val_u16, dp.G, segbase, S, cslice, cloc,
                            NSL, hist, nsegs, gptr, gent, st));
    dbg_mark(ctx, "g.csr");
    CK(cudaMemcpyAsync(h + 1, bad + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (ctx->debug) {
        std::vector<double> he(nrules);
        std::vector<int32_t> hm(nrules);
        CK(cudaMemcpy(he.data(), rerr, nrules * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hm.data(), rm, nrules * sizeof(int32_t), cudaMemcpyDeviceToHost));
        double we = 0.0;
        int mm = 0;
        for (int i = 0; i < nrules; ++i) {
            we = std::max(we, he[i]);
            mm = std::max(mm, (int)hm[i]);
        }
        fprintf(stderr, "devil_b200: %d design groups x %d clusters, %d rules (max %d nodes, "
                        "worst check error %.3g)%s\n", U, C, nrules, mm, we,
                h[1] ? ": check failed, per-cell engines" : "");
    }
    if (h[1]) return;  // a rule missed its accuracy check: per-cell engines
    // exp of every rule node's offset (mu = exp(x_u . beta) * exp(s) in the passes)
    double* res = ws<double>(ctx, "grp_res", (size_t)nrules * kRuleCap);
    LAUNCH(launch_exp(rs, (int64_t)nrules * kRuleCap, res, st));
    // Sparse design rows and, per output of the p x p assembly, the groups
    // whose entries are nonzero (ascending group, so the sums keep a fixed
    // order).  A one-hot row (intercept, condition, one cell type) has three
    // nonzeros: six (group, pair) terms instead of p(p+1)/2.
    std::vector<double> hx((size_t)U * P);
    CK(cudaMemcpyAsync(hx.data(), xg, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int NE = P * (P + 1) / 2;
    std::vector<int32_t> rptr(U + 1, 0), rcol, qptr(NE + 1, 0), qu, vptr(P + 1, 0), vu;
    std::vector<double> rval, qv, vv;
    for (int u = 0; u < U; ++u) {
        for (int j = 0; j < P; ++j)
            if (hx[(size_t)u * P + j] != 0.0) {
                rcol.push_back(j);
                rval.push_back(hx[(size_t)u * P + j]);
            }
        rptr[u + 1] = (int32_t)rcol.size();
    }
    for (int j = 0; j < P; ++j)
        for (int i = 0; i <= j; ++i) {
            for (int u = 0; u < U; ++u) {
                const double xi = hx[(size_t)u * P + i], xj = hx[(size_t)u * P + j];
                if (xi != 0.0 && xj != 0.0) {
                    qu.push_back(u);
                    qv.push_back(xi * xj);
                }
            }
            qptr[j * (j + 1) / 2 + i + 1] = (int32_t)qu.size();
        }
    for (int i = 0; i < P; ++i) {
        for (int u = 0; u < U; ++u)
            if (hx[(size_t)u * P + i] != 0.0) {
                vu.push_back(u);
                vv.push_back(hx[(size_t)u * P + i]);
            }
        vptr[i + 1] = (int32_t)vu.size();
    }
    // exclusive columns (no design row with two of them nonzero), chosen
    // greedily in order of fewest collisions: the one-hot cell-type
    // indicators of a design; the rest stay dense.  Used when at least four
    // columns are exclusive and at most eight are dense.
    std::vector<int32_t> colA, colD, colpos(P, 0);
    {
        std::vector<int> coll(P, 0);
        auto collide = [&](int i, int j) {
            for (int u = 0; u < U; ++u)
                if (hx[(size_t)u * P + i] != 0.0 && hx[(size_t)u * P + j] != 0.0) return true;
            return false;
        };
        for (int i = 0; i < P; ++i)
            for (int j = 0; j < P; ++j)
                if (i != j && collide(i, j)) ++coll[i];
        std::vector<int> order(P);
        for (int i = 0; i < P; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return coll[a] < coll[b]; });
        std::vector<char> inD(P, 0);
        for (int c : order) {
            bool ok = true;
            for (int d = 0; d < P && ok; ++d)
                if (inD[d] && collide(c, d)) ok = false;
            if (ok) inD[c] = 1;
        }
        for (int c = 0; c < P; ++c) {
            if (inD[c]) {
                colpos[c] = -1 - (int32_t)colD.size();
                colD.push_back(c);
            } else {
                colpos[c] = (int32_t)colA.size();
                colA.push_back(c);
            }
        }
        if (colD.size() < 4 || colA.size() > 8 || colA.empty()) colA.clear();
    }
    // the Hessian entries the Schur step reads: for every packed output
    // (i <= j) with i or j dense, or i == j, its places in the compact store
    // (rows of the dense columns [nA][P], then the diagonal [P])
    std::vector<int32_t> need_q, need_d;
    if (!colA.empty()) {
        const int k = (int)colA.size();
        for (int j = 0; j < P; ++j)
            for (int i = 0; i <= j; ++i) {
                const int pi = colpos[i], pj = colpos[j];
                int d[3] = {-1, -1, -1}, nd = 0;
                if (pi >= 0) d[nd++] = pi * P + j;
                if (pj >= 0 && i != j) d[nd++] = pj * P + i;
                if (i == j) d[nd++] = k * P + i;
                if (nd == 0) continue;
                need_q.push_back(j * (j + 1) / 2 + i);
                for (int t = 0; t < 3; ++t) need_d.push_back(d[t]);
            }
    }
    auto up_i = [&](const char* nm, const std::vector<int32_t>& v) {
        int32_t* d = ws<int32_t>(ctx, nm, std::max<size_t>(v.size(), 1));
        h2d(ctx, d, v.data(), v.size());
        return d;
    };
    auto up_d = [&](const char* nm, const std::vector<double>& v) {
        double* d = ws<double>(ctx, nm, std::max<size_t>(v.size(), 1));
        h2d(ctx, d, v.data(), v.size());
        return d;
    };
    auto& g = dp.grp;
    g.rptr = up_i("grp_rptr", rptr);
    g.rcol = up_i("grp_rcol", rcol);
    g.rval = up_d("grp_rval", rval);
    g.qptr = up_i("grp_qptr", qptr);
    g.qu = up_i("grp_qu", qu);
    g.qv = up_d("grp_qv", qv);
    g.vptr = up_i("grp_vptr", vptr);
    g.vu = up_i("grp_vu", vu);
    g.vv = up_d("grp_vv", vv);
    g.nA = (int)colA.size();
    if (g.nA > 0) {
        g.colA = up_i("grp_colA", colA);
        g.colD = up_i("grp_colD", colD);
        g.colpos = up_i("grp_colpos", colpos);
        g.n_need = (int)need_q.size();
        g.need_q = up_i("grp_need_q", need_q);
        g.need_d = up_i("grp_need_d", need_d);
    }
    g.res = res;
    // the work order of the slice-major passes: genes by decreasing entries
    // (sorted with the CSR check; counts converted from dense or CSC input
    // are sorted here)
    if (!dp.gorder) gene_order(ctx, dp);
    g.order = dp.gorder;
    g.wkey = dp.gwkey;
    g.skey = dp.gskey;
    CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
    g.active = true;
    g.U = U;
    g.C = C;
    g.S = NSL;
    g.xg = xg;
    g.E = E;
    g.gent = gent;
    g.gptr = gptr;
    g.sl_start = d_sl_start;
    g.sl_key = d_sl_key;
    g.kslice = d_kslice;
    g.rs = rs;
    g.rw = rw;
    g.rm = rm;
}

GrpGeom grp_geom(const DevProblem& dp) {
    const auto& gr = dp.grp;
    GrpGeom gg{};
    gg.P = dp.P;
    gg.U = gr.U;
    gg.C = gr.C;
    gg.xg = gr.xg;
    gg.S = gr.S;
    gg.E = gr.E;
    gg.gent = gr.gent;
    gg.gptr = gr.gptr;
    gg.sl_start = gr.sl_start;
    gg.sl_key = gr.sl_key;
    gg.kslice = gr.kslice;
    gg.rs = gr.rs;
    gg.rw = gr.rw;
    gg.rm = gr.rm;
    gg.res = gr.res;
    gg.rptr = gr.rptr;
    gg.rcol = gr.rcol;
    gg.rval = gr.rval;
    gg.qptr = gr.qptr;
    gg.qu = gr.qu;
    gg.qv = gr.qv;
    gg.vptr = gr.vptr;
    gg.nA = gr.nA;
    gg.colA = gr.colA;
    gg.colD = gr.colD;
    gg.colpos = gr.colpos;
    gg.n_need = gr.n_need;
    gg.need_q = gr.need_q;
    gg.need_d = gr.need_d;
    gg.vu = gr.vu;
    gg.vv = gr.vv;
    return gg;
}

// ------------------------------------------------------------------
// the gene x cell pass driver
// ------------------------------------------------------------------
struct PassPlan {
    Engine engine;
    int GT;
    PassKind kind = PASS_IRLS;
    int plain = 0;  // the plain comparison form
    int waves = 0;  // design groups: waves of a slice-major step; wide tensor cores: minimum waves
                    // (0: the engine's default)
};

// the tensor-core IRLS engine for p = 5..32 (kernels_tcw.cu): DEVIL_TCW=1
// selects it wherever it applies, DEVIL_TCW=0 never; otherwise it runs for
// the DEVIL_PREC_TC_TF32 precision and, by default, from p = 9 on, where
// the alternative is the FP64 shared-memory engine (about 20x slower per
// IRLS pass at p = 16 and 32 on the 20,000 x 100,000 continuous workload)
bool tcw_wanted(const DevProblem& dp) {
    if (!tcw_supported(dp.P, dp.xs) || !tcw_fits(dp)) return false;
    const char* e = getenv("DEVIL_TCW");
    if (e && *e) return atoi(e) == 1;
    return dp.precision == DEVIL_PREC_TC_TF32 || dp.P > reg_max_p();
}
// its dispersion (MLE) pass: DEVIL_TCW_MLE=1 / 0; otherwise as the IRLS
// pass (the FP64 shared-memory pass it replaces from p = 9 on is about 13x
// slower on the 20,000 x 100,000 continuous workload at p = 16 and 32)
bool tcw_mle_wanted(const DevProblem& dp) {
    if (!tcw_supported(dp.P, dp.xs) || !tcw_fits(dp)) return false;
    const char* e = getenv("DEVIL_TCW_MLE");
    if (e && *e) return atoi(e) == 1;
    return dp.precision == DEVIL_PREC_TC_TF32 || dp.P > reg_max_p();
}

PassPlan plan_engine(PassKind k, const DevProblem& dp, int form, bool allow_tcw = true) {
    const int P = dp.P;
    // the plain comparison form: every pass on the per-cell shared-memory
    // engine, FP32 per-cell arithmetic for the FP32 passes (IRLS, MLE)
    if (form == DEVIL_FORM_PLAIN) return {ENGINE_GEN, gen_default_gt(k, P), k, 1};
    if (dp.grp.active) return {ENGINE_GRP, 1};
    if (k == PASS_IRLS && allow_tcw && tcw_wanted(dp)) return {ENGINE_TCW, tcw_tile_genes(k)};
    if (k == PASS_MLE && allow_tcw && tcw_mle_wanted(dp)) return {ENGINE_TCW, tcw_tile_genes(k)};
    const bool tc = tc_enabled(k) ||
                    (dp.precision == DEVIL_PREC_TC_TF32 && (k == PASS_IRLS || k == PASS_MLE));
    if (P <= tc_max_p() && tc) return {ENGINE_TC, tc_tile_genes(k)};
    if (P <= reg_max_p()) {
        int gt = reg_default_gt(k, P);
        if (k == PASS_MLE) {
            const char* e = getenv("DEVIL_MLE_GT");
            if (e) {
                int v = atoi(e);
                if (reg_gt_supported(k, P, v)) gt = v;
            }
        }
        if (k == PASS_IRLS) {
            const char* e = getenv("DEVIL_IRLS_GT");
            if (e) {
                int v = atoi(e);
                if (reg_gt_supported(k, P, v)) gt = v;
            }
        }
        return {ENGINE_REG, gt};
    }
    return {ENGINE_GEN, gen_default_gt(k, P)};
}

PassPlan plan_for(PassKind k, const DevProblem& dp, int form, bool allow_tcw = true) {
    PassPlan p = plan_engine(k, dp, form, allow_tcw);
    p.kind = k;
    return p;
}

// number of cell-segment work items for `tiles` gene tiles.  The grid has
// tiles x nseg blocks; `cap` of them are resident at once (SMs x the
// kernel's occupancy).  At least one full wave (four for the heavy
// tensor-core blocks), then the smallest nseg whose last wave is nearly
// full: with 1.1 waves the second wave would keep 90 % of the SMs idle
// (active-gene counts in the IRLS tail produce exactly such grids).
int choose_nseg(devil_ctx* ctx, const DevProblem& dp, const PassPlan& plan, int tiles, int form) {
    (void)form;
    if (plan.engine == ENGINE_GRP) return 1;
    const int occ = pass_blocks_per_sm(plan.kind, plan.engine, dp.P, plan.GT, dp.val_u16, plan.plain);
    const int64_t cap = (int64_t)ctx->sm_count * std::max(1, occ);
    const int64_t min_waves =
        plan.engine == ENGINE_TC ? 4 : (plan.engine == ENGINE_TCW ? (plan.waves > 0 ? plan.waves : 2) : 1);
    // the wide tensor-core engine has tcw_blocks(p) product blocks per tile
    if (plan.engine == ENGINE_TCW) tiles *= tcw_blocks(dp.P);
    int want = (int)((min_waves * cap + tiles - 1) / tiles);
    want = std::max(1, std::min(want, dp.nfine));
    const int hi = std::min(dp.nfine, 4 * want);
    int best = want;
    double best_eff = 0.0;
    for (int ns = want; ns <= hi; ++ns) {
        const double waves = (double)tiles * ns / (double)cap;
        const double eff = waves / std::ceil(waves);
        if (eff > best_eff + 1e-9) {
            best = ns;
            best_eff = eff;
        }
        if (eff >= 0.92) break;
    }
    return best;
}

// largest nseg * tiles * GT over every active-gene count the loops can see
size_t max_slot_segs(devil_ctx* ctx, const DevProblem& dp, const PassPlan& plan, int form) {
    const int GT = plan.GT;
    const int max_tiles = (int)((dp.G + GT - 1) / GT);
    size_t best = 0;
    for (int tiles = 1; tiles <= max_tiles; ++tiles) {
        size_t v = (size_t)choose_nseg(ctx, dp, plan, tiles, form) * tiles * GT;
        if (v > best) best = v;
    }
    return best;
}

struct PassBuffers {
    void* partW;     // partial sums: Pass::AW from the register engine, double from the generic one
    double* partS;
    double* partWd() const { return static_cast<double*>(partW); }
};

PassBuffers pass_buffers(devil_ctx* ctx, PassKind k, int P, size_t slots_x_segs) {
    PassBuffers b;
    b.partW = ws<double>(ctx, "partW", slots_x_segs * std::max(1, pass_na(k, P)));
    b.partS = ws<double>(ctx, "partS", slots_x_segs * std::max(1, pass_ns(k)));
    return b;
}

void launch_pass(devil_ctx* ctx, const DevProblem& dp, PassKind kind, const PassPlan& plan,
                 int nseg, int tiles, const int32_t* bound, const int64_t* segptr,
                 int nbound, const int32_t* act, const int32_t* n_act, int32_t* reset_next,
                 const PassBuffers& pb, const PassParamsAny& prm, int fine = 0,
                 const int32_t* n_heavy = nullptr, bool rowexp_fresh = false) {
    PassLaunch L;
    L.kind = kind;
    L.engine = plan.engine;
    L.P = dp.P;
    L.xs_pad = dp.xs;
    L.GT = plan.GT;
    L.val_u16 = dp.val_u16;
    L.nseg = nseg;
    L.ntiles = tiles;
    L.geo.X = dp.Xrm;
    L.geo.xs = dp.xs;
    L.geo.off = dp.off_f;
    L.geo.Xd = dp.Xdrm;
    L.geo.offd = dp.off;
    L.geo.col = dp.col;
    L.geo.val = dp.val;
    L.geo.segptr = segptr;
    L.geo.bound = bound;
    L.geo.nbound = nbound;
    L.geo.nseg = nseg;
    L.geo.err = ws<int32_t>(ctx, "kernel_err", 1);
    L.use_tma = plan.engine == ENGINE_REG && ctx->use_tma &&
                (kind == PASS_IRLS || kind == PASS_MLE) && bound == dp.fine_bound;
    L.geo.act = act;
    L.geo.n_act = n_act;
    L.geo.reset_next = reset_next;
    L.geo.partW = pb.partW;
    L.geo.partS = pb.partS;
    L.geo.slot_stride = tiles * plan.GT;
    L.prm = prm;
    L.stream = ctx->stream;
    L.plain = plan.plain;
    size_t e0 = ctx->profiling ? prof_event(ctx) : 0;
    ctx->last_engine[kind] = (int)plan.engine;
    if (plan.engine == ENGINE_GRP) {
        GrpGeom gg = grp_geom(dp);
        gg.fine = fine;
        gg.act = act;
        gg.n_act = n_act;
        gg.n_heavy = n_heavy;
        gg.reset_next = reset_next;
        gg.partW = static_cast<double*>(pb.partW);
        gg.partS = pb.partS;
        gg.slot_stride = tiles;
        const int slice_bit =
            kind == PASS_IRLS ? 1 : (kind == PASS_MLE ? 2 : (kind == PASS_MOM ? 4 : (kind == PASS_SANDWICH ? 8 : 0)));
        if ((ctx->grp_slices & slice_bit) && !fine) {
            // slice-major pass: per-(gene, slice) sums, then the assembly
            gg.gsum = ws<double>(ctx, "grp_gsum", (size_t)tiles * gg.S * grp_slices_nq(kind));
            gg.rowexp = ws<double>(ctx, "grp_rowexp", (size_t)dp.G * gg.U);
            if (kind == PASS_MLE) gg.psitab = ws<double>(ctx, "grp_psitab", (size_t)tiles * kGrpTab);
            // (the IRLS step folds the assembly into its finalize)
            LAUNCH(launch_grp_slices(kind, gg, prm, dp.val_u16, tiles,
                                     grp_slices_tile(tiles, gg.S, ctx->sm_count, plan.waves > 0 ? plan.waves : 3),
                                     kind != PASS_IRLS,
                                     ctx->stream, rowexp_fresh));
        } else {
            LAUNCH(launch_grp_pass(kind, gg, prm, dp.val_u16, tiles, ctx->stream));
        }
    } else if (plan.engine == ENGINE_REG) {
        LAUNCH(launch_reg_pass(L));
    } else if (plan.engine == ENGINE_TC) {
        if (!dp.zimg) {
            dp.zimg = ws<float4>(ctx, "tc_zimg", (size_t)tc_zimg_float4s(dp.n));
            LAUNCH(launch_tc_zimg(dp.Xrm, dp.xs, dp.n, dp.P, dp.zimg, ctx->stream));
        }
        LAUNCH(launch_tc_pass(L, dp.zimg));
    } else if (plan.engine == ENGINE_TCW) {
        if (!dp.tcw_ready) {
            TcwGeom& t = dp.tcw;
            t.npad = tcw_npad(dp.n);
            t.ld = t.npad;
            t.P = dp.P;
            t.NE = dp.P * (dp.P + 1) / 2;
            t.NA = t.NE + dp.P;
            t.nblk = tcw_nblk(dp.P);
            t.ydense = dp.val_u16 ? (const void*)ws<uint16_t>(ctx, "tcw_y", (size_t)dp.G * t.ld)
                                  : (const void*)ws<float>(ctx, "tcw_y", (size_t)dp.G * t.ld);
            t.xt = ws<float>(ctx, "tcw_xt", (size_t)dp.xs * t.npad);
            t.offp = ws<float>(ctx, "tcw_off", (size_t)t.npad);
            LAUNCH(launch_tcw_prepare(dp.rowptr, dp.col, dp.val, dp.val_u16, dp.G, dp.n, dp.Xrm, dp.xs,
                                      dp.off_f, t, ctx->stream));
            dp.tcw_ready = true;
        }
        LAUNCH(launch_tcw_pass(L, dp.tcw));
    } else {
        LAUNCH(launch_gen_pass(L));
    }
    if (ctx->profiling) {
        size_t e1 = prof_event(ctx);
        ctx->recs.push_back({(int)kind, e0, e1});
        if (ctx->ev_used > 4096) prof_collect(ctx);
    }
}

// algorithmic bytes of the passes one gene took part in: its CSR entries
// (uint16 value + int32 cell index, or float + int32), its beta / gene
// parameters, its partial sums; plus the design and offsets once per launch
void prof_add_bytes(devil_ctx* ctx, const DevProblem& dp, PassKind kind, const int32_t* passes,
                    int64_t launches, const PassPlan& plan) {
    if (!ctx->profiling) return;
    int64_t* acc = ws<int64_t>(ctx, "prof_acc", 2);
    CK(cudaMemsetAsync(acc, 0, 2 * sizeof(int64_t), ctx->stream));
    LAUNCH(launch_pass_volume(dp.rowptr, passes, dp.G, acc, ctx->stream));
    int64_t h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // CSR entries: value + 4-byte cell index; the design-group copy packs a
    // 16-bit index within the slice with the value (4 B for 16-bit counts)
    const double ebytes = plan.engine == ENGINE_GRP ? (dp.val_u16 ? 4.0 : 8.0) : (dp.val_u16 ? 6.0 : 8.0);
    const int na = pass_na(kind, dp.P), ns = pass_ns(kind);
    const double per_gene = 4.0 * dp.P + 8.0 + 4.0 * na + 8.0 * ns + 16.0;
    // per launch: the design and offsets, or the group rows, rules and exp(offset)
    const double per_launch = plan.engine == ENGINE_GRP
                                  ? (double)dp.grp.U * dp.P * 8.0 + (double)dp.n * 8.0 +
                                        (double)(dp.grp.U * (dp.grp.C > 1 ? dp.grp.C + 1 : 1)) *
                                            kRuleCap * 16.0
                                  : (double)dp.n * 4.0 * (dp.xs + 1);
    if (plan.engine == ENGINE_TCW) {
        // the dense count image: every cell of the gene once per pass; the
        // MMA work: 3 TF32 products of 128 x nblk x npad per tile and block
        const double npad = (double)tcw_npad(dp.n);
        const double rows = npad * (dp.val_u16 ? 2.0 : 4.0);
        ctx->prof_bytes[kind] += rows * (double)h[1] + per_gene * (double)h[1] +
                                 (double)launches * npad * 4.0 * (dp.xs + 1);
        // (an MMA covers 128 rows: 128 genes in the IRLS pass, 32 genes x 4
        // weights in the MLE pass)
        ctx->prof_tc_flops[kind] += 6.0 * npad * tcw_blocks(dp.P) * tcw_nblk(dp.P) * (double)h[1] *
                                    (128.0 / tcw_tile_genes(kind));
        return;
    }
    ctx->prof_bytes[kind] += ebytes * (double)h[0] + per_gene * (double)h[1] +
                             (double)launches * per_launch;
}

// all-genes list (for one-shot passes)
// (ordered: in decreasing order of entries when the counts were sorted, the
// work order of the slice-major passes, for passes whose finalize maps list
// slots to genes; otherwise slot g is gene g)
const int32_t* all_genes(devil_ctx* ctx, const DevProblem& dp, int32_t** count_out, bool ordered = false) {
    int32_t* a = ws<int32_t>(ctx, "all_genes", dp.G);
    int32_t* c = ws<int32_t>(ctx, "all_count", 4);
    if (ordered && dp.gorder)
        CK(cudaMemcpyAsync(a, dp.gorder, dp.G * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
    else
        LAUNCH(launch_iota(a, dp.G, ctx->stream));
    LAUNCH(launch_set_i32(c, (int32_t)dp.G, ctx->stream));
    *count_out = c;
    return a;
}

// ------------------------------------------------------------------
// IRLS loop (src/beta.cpp:25-51) with active-gene compaction
// ------------------------------------------------------------------
// ------------------------------------------------------------------
// tile autotuner
// ------------------------------------------------------------------
// Each engine has a tile knob whose best value depends on the shape: genes
// per thread of the register engine (GT), the waves a slice-major step of
// the design-group engine is spread over (its gene tile), the minimum
// waves of the wide tensor-core pass (its cell segments).  On the first
// loop of a shape bucket (pass kind, engine, p, count type, log2 n,
// log2 G, half-octaves of the density) in this process, each candidate
// plan runs the loop's first pass once untimed and once timed (CUDA events
// on the context stream, all genes active); the fastest is kept for the
// bucket.  The candidates leave every gene's result unchanged except for
// the register and wide engines, whose FP32 segment sums can round
// differently (well inside the parity bars).  DEVIL_AUTOTUNE=0 keeps the
// heuristic defaults.
struct TuneKey {
    int kind, engine, P, u16, nb, gb, db;
    bool operator<(const TuneKey& o) const {
        return std::tie(kind, engine, P, u16, nb, gb, db) < std::tie(o.kind, o.engine, o.P, o.u16, o.nb, o.gb, o.db);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, PassPlan> g_tune;

bool autotune_enabled() {
    const char* e = getenv("DEVIL_AUTOTUNE");
    return !(e && *e && atoi(e) == 0);
}

std::vector<PassPlan> tune_candidates(devil_ctx* ctx, const DevProblem& dp, const PassPlan& base) {
    std::vector<PassPlan> c{base};
    if (base.plain) return c;
    if (base.engine == ENGINE_REG && (base.kind == PASS_IRLS || base.kind == PASS_MLE)) {
        if (getenv(base.kind == PASS_IRLS ? "DEVIL_IRLS_GT" : "DEVIL_MLE_GT")) return c;  // set by hand
        for (int gt : {base.GT / 2, base.GT * 2}) {
            if (gt < 1 || !reg_gt_supported(base.kind, dp.P, gt)) continue;
            PassPlan p = base;
            p.GT = gt;
            c.push_back(p);
        }
    } else if (base.engine == ENGINE_GRP) {
        const int bit = base.kind == PASS_IRLS ? 1 : (base.kind == PASS_MLE ? 2 : 0);
        if (ctx->grp_slices & bit) {
            for (int w : {2, 6}) {
                PassPlan p = base;
                p.waves = w;
                c.push_back(p);
            }
        }
    } else if (base.engine == ENGINE_TCW) {
        PassPlan p = base;
        p.waves = 4;
        c.push_back(p);
    }
    return c;
}

// the plan for a loop's passes; act / n_act list the n0 genes of its first pass
PassPlan autotune(devil_ctx* ctx, const DevProblem& dp, const PassPlan& base, const int32_t* act,
                  const int32_t* n_act, int64_t n0, const PassParamsAny& prm, int form) {
    if (!autotune_enabled() || n0 < 256) return base;
    const double dens = dp.nnz > 0 ? (double)dp.nnz / ((double)dp.G * (double)dp.n) : 1e-9;
    const TuneKey key{(int)base.kind, (int)base.engine, dp.P, dp.val_u16,
                      (int)std::floor(std::log2((double)dp.n)), (int)std::floor(std::log2((double)dp.G)),
                      (int)std::floor(-2.0 * std::log2(dens))};
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
    const std::vector<PassPlan> cands = tune_candidates(ctx, dp, base);
    PassPlan best = base;
    if (cands.size() > 1) {
        const int was_profiling = ctx->profiling;
        ctx->profiling = 0;
        cudaEvent_t t0, t1;
        CK(cudaEventCreate(&t0));
        CK(cudaEventCreate(&t1));
        double best_ms = 0.0;
        for (size_t i = 0; i < cands.size(); ++i) {
            const PassPlan& pl = cands[i];
            const int tiles = (int)((n0 + pl.GT - 1) / pl.GT);
            const int nseg = choose_nseg(ctx, dp, pl, tiles, form);
            const PassBuffers pb = pass_buffers(ctx, pl.kind, dp.P, (size_t)nseg * tiles * pl.GT);
            float ms = 0.f;
            for (int rep = 0; rep < 2; ++rep) {
                CK(cudaEventRecord(t0, ctx->stream));
                launch_pass(ctx, dp, pl.kind, pl, nseg, tiles, dp.fine_bound, dp.fine_ptr, dp.nfine + 1, act,
                            n_act, nullptr, pb, prm);
                CK(cudaEventRecord(t1, ctx->stream));
                CK(cudaEventSynchronize(t1));
                CK(cudaEventElapsedTime(&ms, t0, t1));
            }
            // a candidate replaces the default only when clearly faster
            if (i == 0 || ms < 0.97 * best_ms) {
                best = pl;
                best_ms = ms;
            }
            if (ctx->debug) fprintf(stderr, "[devil] tune kind %d engine %d GT %d waves %d: %.3f ms\n",
                                    (int)pl.kind, (int)pl.engine, pl.GT, pl.waves, ms);
        }
        CK(cudaEventDestroy(t0));
        CK(cudaEventDestroy(t1));
        ctx->profiling = was_profiling;
    }
    g_tune[key] = best;
    return best;
}

// entries per slice below which a gene of a slice-major pass takes eight
// lanes instead of a warp: IRLS (DEVIL_LIGHT_ENTRIES overrides
// kLightEntries) and MLE (DEVIL_LIGHT_ENTRIES_MLE, kLightEntriesMle)
int light_entries(bool mle = false) {
    static const int v[2] = {
        [] {
            const char* e = getenv("DEVIL_LIGHT_ENTRIES");
            return (e && *e) ? std::max(0, atoi(e)) : kLightEntries;
        }(),
        [] {
            const char* e = getenv("DEVIL_LIGHT_ENTRIES_MLE");
            return (e && *e) ? std::max(0, atoi(e)) : kLightEntriesMle;
        }()};
    return v[mle ? 1 : 0];
}

// One IRLS loop over the n0 genes listed in the "act0" workspace (their
// iteration counts and status start at 0); returns the pass launches.
int64_t irls_loop(devil_ctx* ctx, const DevProblem& dp, const PassPlan& plan0, double* beta, float* beta_f,
                  const float* k, int32_t* iters, int32_t* status, int max_iter, double eps, int form,
                  int64_t n0) {
    cudaStream_t st = ctx->stream;
    const int64_t G = dp.G;
    int32_t* act[2] = {ws<int32_t>(ctx, "act0", G), ws<int32_t>(ctx, "act1", G)};
    int32_t* cnt = ws<int32_t>(ctx, "cnt", 4);
    LAUNCH(launch_set_i32(cnt, (int32_t)n0, st));
    LAUNCH(launch_set_i32(cnt + 1, 0, st));
    PassParamsAny prm{beta_f, beta, k, nullptr, nullptr};
    const PassPlan plan = autotune(ctx, dp, plan0, act[0], cnt, n0, prm, form);
    PassBuffers pb = pass_buffers(ctx, PASS_IRLS, dp.P, max_slot_segs(ctx, dp, plan, form));
    // slice-major passes over the genes in decreasing order of entries
    // (act0 = dp.grp.order): the genes below kLightEntries entries per slice
    // on average take eight lanes each
    const bool sliced = plan.engine == ENGINE_GRP && (ctx->grp_slices & 1);
    int32_t* nheavy = ws<int32_t>(ctx, "cnt_heavy", 2);
    const int32_t thr = (int32_t)std::min<int64_t>((int64_t)light_entries() * dp.grp.S, INT32_MAX);
    if (sliced) LAUNCH(launch_count_at_least(dp.grp.skey, n0, thr, nheavy, st));
    // copies of an earlier loop still in flight would overwrite the mirror
    CK(cudaStreamSynchronize(st));
    const int LAG = 2;
    int64_t launched = 0;
    for (int t = 0; t < max_iter; ++t) {
        const int cur = t & 1, nxt = cur ^ 1;
        // active-gene count after iteration t - 1 - LAG, the last one the
        // host has waited for (an upper bound: blocks beyond the current
        // count exit at once).  Each iteration mirrors its count into its own
        // slot, so the grid sizes -- and the segment sums they set -- do not
        // depend on how far the device has run ahead.
        const int64_t hint = t <= LAG ? n0 : ctx->mapped_host_at(t - 1 - LAG);
        if (hint <= 0) break;
        const int tiles = (int)((hint + plan.GT - 1) / plan.GT);
        const int nseg = choose_nseg(ctx, dp, plan, tiles, form);
        // (after the first pass the step kernel keeps the genes' exp(x_u . beta))
        launch_pass(ctx, dp, PASS_IRLS, plan, nseg, tiles, dp.fine_bound, dp.fine_ptr,
                    dp.nfine + 1, act[cur], cnt + cur, cnt + nxt, pb, prm, 0, sliced ? nheavy + cur : nullptr,
                    sliced && t > 0);
        ++launched;
        const bool part_f64 = plan.engine != ENGINE_REG && plan.engine != ENGINE_TC && plan.engine != ENGINE_TCW;
        if (sliced) {
            // slice-major pass: the assembly is part of the step
            GrpGeom gg = grp_geom(dp);
            gg.act = act[cur];
            gg.n_act = cnt + cur;
            gg.gsum = ws<double>(ctx, "grp_gsum", (size_t)tiles * gg.S * 2);
            gg.rowexp = ws<double>(ctx, "grp_rowexp", (size_t)G * gg.U);
            // the genes that go on keep the order of the list (decreasing
            // entries: the pass's work order)
            int8_t* keep = ws<int8_t>(ctx, "keep", G);
            LAUNCH(launch_grp_irls_finalize(gg, (int)hint, act[nxt], cnt + nxt, beta, beta_f, iters,
                                            status, max_iter, eps, k, st, keep));
            LAUNCH(launch_compact_kept(act[cur], cnt + cur, 0, keep, act[nxt], cnt + nxt, st, dp.grp.wkey, thr,
                                       nheavy + nxt, ctx->mapped_dev + (t & 3)));
        } else {
            LAUNCH(launch_irls_finalize(pb.partW, part_f64, nseg, tiles * plan.GT, dp.P, act[cur],
                                        cnt + cur, (int)hint, act[nxt], cnt + nxt, beta, beta_f,
                                        iters, status, max_iter, eps, k, st));
            LAUNCH(launch_copy_i32_to_host_mapped(cnt + nxt, ctx->mapped_dev + (t & 3), st));
        }
        CK(cudaEventRecord(ctx->ev[t & 3], st));
        if (t >= LAG) CK(cudaEventSynchronize(ctx->ev[(t - LAG) & 3]));
    }
    return launched;
}

// beta_fit for every gene (src/beta.cpp:25-51).  On the tensor-core engine
// of p = 5..32 (FP32-level Hessian and score) a gene whose fit ends with a
// coefficient beyond +-8 is fitted again from beta_0 on the CUDA-core engine
// (FP64 per cell above p = 8): such a gene has a group of cells without
// counts, its intercept and group coefficients drift apart step after step
// along a nearly flat direction of the likelihood, and along that path
// FP32-level rounding moves the iterate where the FP64 path would not
// (|d beta| 2e-4 after 183 steps at |beta| ~ 15).  On continuous designs the
// engine stays within 2e-6 of the FP64 oracle at every iteration count up
// to max_iter.  DEVIL_TCW_RESCUE_BETA sets the coefficient bound;
// DEVIL_TCW_RESCUE=s also refits every gene that took more than s steps.
int tcw_rescue_steps(int max_iter) {
    const char* e = getenv("DEVIL_TCW_RESCUE");
    return (e && *e) ? atoi(e) : max_iter;
}
double tcw_rescue_beta() {
    const char* e = getenv("DEVIL_TCW_RESCUE_BETA");
    return (e && *e) ? atof(e) : 8.0;
}

void run_irls(devil_ctx* ctx, const DevProblem& dp, double* beta, float* beta_f, const float* k,
              int32_t* iters, int32_t* status, int max_iter, double eps, int form) {
    cudaStream_t st = ctx->stream;
    const int64_t G = dp.G;
    CK(cudaMemsetAsync(iters, 0, G * sizeof(int32_t), st));
    CK(cudaMemsetAsync(status, 0, G * sizeof(int32_t), st));
    if (G == 0 || max_iter <= 0) return;
    const PassPlan plan = plan_for(PASS_IRLS, dp, form);
    if (plan.GT <= 0) fail(ctx, DEVIL_ERR_UNSUPPORTED, "p = %d unsupported", dp.P);
    const int limit = tcw_rescue_steps(max_iter);
    const bool rescue = plan.engine == ENGINE_TCW;
    double* beta0 = nullptr;
    if (rescue) {
        beta0 = ws<double>(ctx, "irls_beta0", (size_t)G * dp.P);
        CK(cudaMemcpyAsync(beta0, beta, (size_t)G * dp.P * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    if (plan.engine == ENGINE_GRP && (ctx->grp_slices & 1))
        CK(cudaMemcpyAsync(ws<int32_t>(ctx, "act0", G), dp.grp.order, G * sizeof(int32_t),
                           cudaMemcpyDeviceToDevice, st));  // decreasing entries
    else
        LAUNCH(launch_iota(ws<int32_t>(ctx, "act0", G), G, st));
    const int64_t launched = irls_loop(ctx, dp, plan, beta, beta_f, k, iters, status, max_iter, eps, form, G);
    if (ctx->profiling) {
        prof_collect(ctx);
        prof_add_bytes(ctx, dp, PASS_IRLS, iters, launched, plan);
    }
    ctx->irls_rescued = 0;
    if (!rescue) return;
    int32_t* act0 = ws<int32_t>(ctx, "act0", G);
    int32_t* flag = ws<int32_t>(ctx, "irls_rescue_flag", G);
    int32_t* cnt = ws<int32_t>(ctx, "cnt", 4);
    LAUNCH(launch_set_i32(cnt + 2, 0, st));
    LAUNCH(launch_irls_rescue_select(iters, G, limit, tcw_rescue_beta(), beta0, dp.P, beta, beta_f, iters,
                                     status, act0, cnt + 2, flag, st));
    int32_t nr = 0;
    CK(cudaMemcpyAsync(&nr, cnt + 2, sizeof nr, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    ctx->irls_rescued = nr;
    if (nr == 0) return;
    const PassPlan p2 = plan_for(PASS_IRLS, dp, form, false);
    const int64_t l2 = irls_loop(ctx, dp, p2, beta, beta_f, k, iters, status, max_iter, eps, form, nr);
    ctx->last_engine[PASS_IRLS] = (int)plan.engine;  // the fit's engine (the rescue is counted apart)
    if (ctx->profiling) {
        // the rescue loop's passes: the rescued genes' iteration counts
        int32_t* passes = ws<int32_t>(ctx, "irls_rescue_passes", G);
        LAUNCH(launch_mask_i32(iters, flag, G, passes, st));
        prof_collect(ctx);
        prof_add_bytes(ctx, dp, PASS_IRLS, passes, l2, p2);
    }
}

// MOM theta for all genes (src/mom_overdispersion.cpp)
void run_mom(devil_ctx* ctx, const DevProblem& dp, const float* beta_f, const double* beta_d,
             double* theta, int form) {
    if (dp.G == 0) return;
    const PassPlan plan = plan_for(PASS_MOM, dp, form);
    int32_t* cnt = nullptr;
    const int32_t* act = all_genes(ctx, dp, &cnt, plan.engine == ENGINE_GRP);  // (mom_finalize maps slots)
    const int tiles = (int)((dp.G + plan.GT - 1) / plan.GT);
    const int nseg = choose_nseg(ctx, dp, plan, tiles, form);
    PassBuffers pb = pass_buffers(ctx, PASS_MOM, dp.P, (size_t)nseg * tiles * plan.GT);
    PassParamsAny prm{beta_f, beta_d, nullptr, nullptr, nullptr};
    launch_pass(ctx, dp, PASS_MOM, plan, nseg, tiles, dp.fine_bound, dp.fine_ptr,
                dp.nfine + 1, act, cnt, nullptr, pb, prm);
    LAUNCH(launch_mom_finalize(pb.partS, nseg, tiles * plan.GT, act, cnt, (int)dp.G, dp.n, dp.P,
                               theta, ctx->stream));
    if (ctx->profiling) {
        prof_collect(ctx);
        int32_t* ones = ws<int32_t>(ctx, "prof_ones", dp.G);
        LAUNCH(launch_fill_i32(ones, 1, dp.G, ctx->stream));
        prof_add_bytes(ctx, dp, PASS_MOM, ones, 1, plan);
    }
}

// MLE theta (R/overdispersion.R:25-115)
void run_mle(devil_ctx* ctx, const DevProblem& dp, const float* beta_f, const double* beta_d,
             const double* start_hint, double* theta,
             int32_t* newton_iters, int max_iter, int cox_reid, int form) {
    cudaStream_t st = ctx->stream;
    const int64_t G = dp.G;
    if (G == 0) return;
    PassPlan plan = plan_for(PASS_MLE, dp, form);
    if (plan.GT <= 0) fail(ctx, DEVIL_ERR_UNSUPPORTED, "p = %d unsupported for MLE", dp.P);
    MleState s;
    s.x = ws<double>(ctx, "mle_x", G);
    s.lo = ws<double>(ctx, "mle_lo", G);
    s.hi = ws<double>(ctx, "mle_hi", G);
    s.it = newton_iters ? newton_iters : ws<int32_t>(ctx, "mle_it", G);
    s.phase = ws<int32_t>(ctx, "mle_phase", G);
    s.theta = theta;
    s.dx = ws<double>(ctx, "mle_dx", G);
    s.dxold = ws<double>(ctx, "mle_dxold", G);
    s.start_hint = start_hint;
    int32_t* act[2] = {ws<int32_t>(ctx, "act0", G), ws<int32_t>(ctx, "act1", G)};
    int32_t* cnt = ws<int32_t>(ctx, "cnt", 4);
    LAUNCH(launch_set_i32(cnt, 0, st));
    LAUNCH(launch_set_i32(cnt + 1, 0, st));
    // slice-major passes: the active genes stay in decreasing order of entries
    const bool ordered = plan.engine == ENGINE_GRP && (ctx->grp_slices & 2);
    // (and those below kLightEntriesMle entries per slice take eight lanes each)
    int32_t* nheavy = ws<int32_t>(ctx, "cnt_heavy", 2);
    const int32_t thr = ordered ? (int32_t)std::min<int64_t>((int64_t)light_entries(true) * dp.grp.S, INT32_MAX) : 0;
    if (ordered) s.keep = ws<int8_t>(ctx, "keep", G);
    LAUNCH(launch_mle_init(dp.stats, G, dp.n, s, act[0], cnt, st));
    if (ordered)
        LAUNCH(launch_compact_kept(dp.grp.order, nullptr, G, s.keep, act[0], cnt, st, dp.grp.wkey, thr, nheavy));
    PassParamsAny prm{beta_f, beta_d, nullptr, s.x, nullptr};
    plan = autotune(ctx, dp, plan, act[0], cnt, G, prm, form);
    PassBuffers pb = pass_buffers(ctx, PASS_MLE, dp.P, max_slot_segs(ctx, dp, plan, form));
    // copies of an earlier loop still in flight would overwrite the mirror
    CK(cudaStreamSynchronize(st));
    const int LAG = 2;
    int64_t launched = 0;
    // one far-left evaluation plus at most max_iter Newton evaluations
    for (int t = 0; t <= max_iter; ++t) {
        const int cur = t & 1, nxt = cur ^ 1;
        // (the count after iteration t - 1 - LAG, as in irls_loop)
        const int64_t hint = t <= LAG ? G : ctx->mapped_host_at(t - 1 - LAG);
        if (hint <= 0) break;
        const int tiles = (int)((hint + plan.GT - 1) / plan.GT);
        const int nseg = choose_nseg(ctx, dp, plan, tiles, form);
        // (beta is fixed during the MLE loop: exp(x_u . beta) from its first pass)
        launch_pass(ctx, dp, PASS_MLE, plan, nseg, tiles, dp.fine_bound,
                    dp.fine_ptr, dp.nfine + 1, act[cur], cnt + cur, cnt + nxt, pb, prm, 0,
                    ordered ? nheavy + cur : nullptr, ordered && t > 0);
        ++launched;
        const bool part_f64 = plan.engine != ENGINE_REG && plan.engine != ENGINE_TC && plan.engine != ENGINE_TCW;
        // the exclusive-column (one-hot) structure of a grouped design
        // shortens the Cox-Reid terms
        const bool structured = plan.engine == ENGINE_GRP && dp.grp.nA > 0;
        LAUNCH(launch_mle_finalize(pb.partW, part_f64, pb.partS, nseg, tiles * plan.GT, dp.P, dp.stats, dp.n,
                                   act[cur], cnt + cur, (int)hint, act[nxt], cnt + nxt, s, max_iter,
                                   cox_reid, nullptr, st, structured ? dp.grp.nA : 0,
                                   structured ? dp.grp.colA : nullptr, structured ? dp.grp.colD : nullptr));
        // (the compaction mirrors the count for the host; otherwise a kernel does)
        if (ordered)
            LAUNCH(launch_compact_kept(act[cur], cnt + cur, 0, s.keep, act[nxt], cnt + nxt, st, dp.grp.wkey, thr,
                                       nheavy + nxt, ctx->mapped_dev + (t & 3)));
        else
            LAUNCH(launch_copy_i32_to_host_mapped(cnt + nxt, ctx->mapped_dev + (t & 3), st));
        CK(cudaEventRecord(ctx->ev[t & 3], st));
        if (t >= LAG) CK(cudaEventSynchronize(ctx->ev[(t - LAG) & 3]));
    }
    if (ctx->profiling) {
        prof_collect(ctx);
        // genes take part in phase-0 plus one pass per Newton step
        int32_t* np1 = ws<int32_t>(ctx, "prof_mle_passes", G);
        LAUNCH(launch_mle_passes(s.it, s.phase, dp.stats, G, np1, st));
        prof_add_bytes(ctx, dp, PASS_MLE, np1, launched, plan);
    }
}

// bread + clustered meat + sandwich for all genes
void run_sandwich(devil_ctx* ctx, const DevProblem& dp, const float* beta_f, const double* beta_d,
                  const double* theta,
                  const int32_t* ends_host, int n_clusters, double* bread, double* sandwich,
                  double* meat, int form) {
    cudaStream_t st = ctx->stream;
    if (dp.G == 0) return;
    PassPlan plan = plan_for(PASS_SANDWICH, dp, form);
    // the grouped sandwich needs the cells keyed by cluster too
    if (plan.engine == ENGINE_GRP && n_clusters > 0 && dp.grp.C != n_clusters) {
        DevProblem plain = dp;
        plain.grp.active = false;
        plan = plan_for(PASS_SANDWICH, plain, form);
    }
    if (plan.GT <= 0) fail(ctx, DEVIL_ERR_UNSUPPORTED, "p = %d unsupported", dp.P);
    int32_t* cnt = nullptr;
    // (sandwich_finalize maps slots to genes)
    const int32_t* act = all_genes(ctx, dp, &cnt, plan.engine == ENGINE_GRP && n_clusters <= 0);
    const int tiles = (int)((dp.G + plan.GT - 1) / plan.GT);
    PassParamsAny prm{beta_f, beta_d, nullptr, nullptr, theta};
    if (plan.engine == ENGINE_GRP && n_clusters > 0) {
        // one output segment per cluster (fine groups = (design row, cluster))
        for (int b = 0; b < n_clusters; ++b) {
            const int64_t prev = b ? ends_host[b - 1] : 0;
            if (ends_host[b] < prev || ends_host[b] > dp.n)
                fail(ctx, DEVIL_ERR_ARG, "cluster ends must be non-decreasing and <= n");
        }
        if (ends_host[n_clusters - 1] != dp.n)
            fail(ctx, DEVIL_ERR_ARG, "last cluster end must equal the number of cells");
        const int nseg = n_clusters;
        int32_t* segc = ws<int32_t>(ctx, "sw_segc", nseg);
        LAUNCH(launch_iota(segc, nseg, st));
        PassBuffers pb = pass_buffers(ctx, PASS_SANDWICH, dp.P, (size_t)nseg * tiles);
        launch_pass(ctx, dp, PASS_SANDWICH, plan, nseg, tiles, nullptr, nullptr, 0, act, cnt,
                    nullptr, pb, prm, 1);
        LAUNCH(launch_sandwich_finalize(pb.partWd(), nseg, tiles, dp.P, segc, n_clusters, dp.n, act,
                                        cnt, (int)dp.G, bread, sandwich, meat, st));
        if (ctx->profiling) {
            prof_collect(ctx);
            int32_t* ones = ws<int32_t>(ctx, "prof_ones", dp.G);
            LAUNCH(launch_fill_i32(ones, 1, dp.G, st));
            prof_add_bytes(ctx, dp, PASS_SANDWICH, ones, 1, plan);
        }
        return;
    }
    if (n_clusters <= 0) {
        const int nseg = choose_nseg(ctx, dp, plan, tiles, form);
        PassBuffers pb = pass_buffers(ctx, PASS_SANDWICH, dp.P, (size_t)nseg * tiles * plan.GT);
        launch_pass(ctx, dp, PASS_SANDWICH, plan, nseg, tiles, dp.fine_bound,
                    dp.fine_ptr, dp.nfine + 1, act, cnt, nullptr, pb, prm);
        LAUNCH(launch_sandwich_finalize(pb.partWd(), nseg, tiles * plan.GT, dp.P, nullptr, 0, dp.n,
                                        act, cnt, (int)dp.G, bread, nullptr, nullptr, st));
        if (ctx->profiling) {
            prof_collect(ctx);
            int32_t* ones = ws<int32_t>(ctx, "prof_ones", dp.G);
            LAUNCH(launch_fill_i32(ones, 1, dp.G, st));
            prof_add_bytes(ctx, dp, PASS_SANDWICH, ones, 1, plan);
        }
        return;
    }
    // cluster-aligned segments: every cluster block split into pieces of
    // at most L cells (1-based exclusive ends, R/main.R:193)
    const int64_t n = dp.n;
    int want = (ctx->sm_count * 2 + tiles - 1) / tiles;
    int64_t L = std::max<int64_t>(1024, (n + want - 1) / std::max(1, want));
    std::vector<int32_t> hb{0};
    std::vector<int32_t> hc;
    int64_t start = 0;
    for (int b = 0; b < n_clusters; ++b) {
        int64_t end = ends_host[b];
        if (end < start || end > n) fail(ctx, DEVIL_ERR_ARG, "cluster ends must be non-decreasing and <= n");
        if (end == start) continue;
        int64_t pieces = (end - start + L - 1) / L;
        for (int64_t q = 1; q <= pieces; ++q) {
            hb.push_back((int32_t)(start + ((end - start) * q) / pieces));
            hc.push_back(b);
        }
        start = end;
    }
    if (start != n) fail(ctx, DEVIL_ERR_ARG, "last cluster end must equal the number of cells");
    const int nseg = (int)hc.size();
    int32_t* bound = ws<int32_t>(ctx, "sw_bound", hb.size());
    int32_t* segc = ws<int32_t>(ctx, "sw_segc", hc.size());
    h2d(ctx, bound, hb.data(), hb.size());
    h2d(ctx, segc, hc.data(), hc.size());
    int64_t* segptr = ws<int64_t>(ctx, "sw_segptr", (size_t)dp.G * hb.size());
    LAUNCH(launch_segptr(dp.rowptr, dp.col, dp.G, bound, (int)hb.size(), segptr, st));
    PassBuffers pb = pass_buffers(ctx, PASS_SANDWICH, dp.P, (size_t)nseg * tiles * plan.GT);
    launch_pass(ctx, dp, PASS_SANDWICH, plan, nseg, tiles, bound, segptr, (int)hb.size(), act,
                cnt, nullptr, pb, prm);
    LAUNCH(launch_sandwich_finalize(pb.partWd(), nseg, tiles * plan.GT, dp.P, segc, n_clusters, dp.n,
                                    act, cnt, (int)dp.G, bread, sandwich, meat, st));
    CK(cudaStreamSynchronize(st));  // host vectors hb/hc go out of scope
    if (ctx->profiling) {
        prof_collect(ctx);
        int32_t* ones = ws<int32_t>(ctx, "prof_ones", dp.G);
        LAUNCH(launch_fill_i32(ones, 1, dp.G, st));
        prof_add_bytes(ctx, dp, PASS_SANDWICH, ones, 1, plan);
    }
}

// a bounded wait inside a kernel gave up (the kernel skipped its writes)
void check_kernel_err(devil_ctx* ctx) {
    int32_t* err = ws<int32_t>(ctx, "kernel_err", 1);
    int32_t h = 0;
    CK(cudaMemcpyAsync(&h, err, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h) {
        CK(cudaMemsetAsync(err, 0, sizeof(int32_t), ctx->stream));
        fail(ctx, DEVIL_ERR_CUDA, "a staged copy wait timed out inside a pass kernel");
    }
}

// Gauss-Hermite rule (weight exp(-x^2)) of order m: eigenvalues of the
// Jacobi matrix (zero diagonal, off-diagonal sqrt(k/2)) by bisection on
// Sturm counts, weights sqrt(pi) / sum_k q_k(x)^2 over the orthonormal
// Hermite polynomials q_k (Golub-Welsch, as src/new_overdispersion.cpp:22-47)
void gauss_hermite_rule(int m, double* x, double* w) {
    const double hi0 = std::sqrt(2.0 * m) + 1.0;
    for (int j = 0; j < m; ++j) {
        double lo = -hi0, hi = hi0;
        for (int it = 0; it < 200; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (mid <= lo || mid >= hi) break;
            int below = 0;
            double d = 1.0;
            for (int i = 0; i < m; ++i) {
                d = -mid - (i ? 0.5 * i / d : 0.0);
                if (d == 0.0) d = -1e-300;
                below += d < 0.0;
            }
            if (below > j) hi = mid; else lo = mid;
        }
        const double xj = 0.5 * (lo + hi);
        double qm = 0.0, q = 1.0, sum = 1.0;
        for (int k = 0; k + 1 < m; ++k) {
            const double qn = (xj * q - (k ? std::sqrt(0.5 * k) : 0.0) * qm) / std::sqrt(0.5 * (k + 1));
            qm = q;
            q = qn;
            sum += q * q;
        }
        x[j] = xj;
        w[j] = std::sqrt(M_PI) / sum;
    }
}

// overdispersion = "new" (fit_overdispersion_cppp) for every gene at the
// fitted beta; the reference's stop() conditions fail the whole call, as
// they fail fit_devil in R (R/main.R:443-454 under bplapply)
void run_new_od(devil_ctx* ctx, const DevProblem& dp, const double* beta_d, double* theta,
                int32_t* iters, int max_iter, double eps) {
    if (dp.G == 0) return;
    cudaStream_t st = ctx->stream;
    const int m = 16;  // newton_max, also the Gauss-Hermite order (src/new_overdispersion.cpp:310)
    double hx[16], hw[16];
    gauss_hermite_rule(m, hx, hw);
    double* gx = ws<double>(ctx, "nod_gx", m);
    double* gw = ws<double>(ctx, "nod_gw", m);
    h2d(ctx, gx, hx, m);
    h2d(ctx, gw, hw, m);
    double* xcs = ws<double>(ctx, "nod_xcolsum", dp.P);
    int32_t* err = ws<int32_t>(ctx, "nod_err", dp.G);
    NodArgs a{};
    a.G = dp.G;
    a.n = dp.n;
    a.P = dp.P;
    a.xs = dp.xs;
    a.Xd = dp.Xdrm;
    a.off = dp.off;
    a.xcolsum = xcs;
    a.rowptr = dp.rowptr;
    a.col = dp.col;
    a.val = dp.val;
    a.val_u16 = dp.val_u16;
    a.beta = beta_d;
    a.stats = dp.stats;
    a.max_iter = max_iter;
    a.eps = eps;
    a.gh_m = m;
    a.max_newton = m;
    a.gx = gx;
    a.gw = gw;
    a.theta = theta;
    a.iters = iters;
    a.err = err;
    LAUNCH(launch_new_od(a, dp.Xcm, xcs, st));
    std::vector<int32_t> he(dp.G);
    CK(cudaMemcpyAsync(he.data(), err, dp.G * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));  // also keeps hx/hw alive until the copies ran
    for (int64_t g = 0; g < dp.G; ++g) {
        if (!he[g]) continue;
        static const char* msg[] = {"", "kappa update requires C1 > n",
                                    "Mode-finding failed: h''(mu0) >= 0 or non-finite.",
                                    "GH quadrature underflow.", "kappa residual not finite at start."};
        fail(ctx, DEVIL_ERR_NUMERIC, "%s (gene %lld)", msg[he[g] >= 1 && he[g] <= 4 ? he[g] : 0],
             (long long)g);
    }
}

struct FitBuffers {
    double* beta;
    float* beta_f;
    float* k;
    double* theta0;
    double* theta;
    double* theta_mom;
    int32_t* iters;
    int32_t* status;
    int32_t* titers;
    double* bread;
    double* sandwich;
    double* meat;
};

// cpu_fit order: theta_0 -> beta | theta_0 -> theta | beta -> bread, meat
void fit_pipeline(devil_ctx* ctx, DevProblem& dp, const int32_t* ends_host, int n_clusters,
                  const devil_fit_opts* o, FitBuffers& fb) {
    cudaStream_t st = ctx->stream;
    const int64_t G = dp.G;
    const int P = dp.P;
    dp.precision = o->precision;
    dbg_mark(ctx, "groups");
    LAUNCH(launch_theta0(dp.stats, dp.off, G, dp.n, o->has_init_overdispersion,
                         o->init_overdispersion, fb.theta0, fb.k, st));
    double* ginv = ws<double>(ctx, "ginv", (size_t)P * P);
    int32_t* err = ws<int32_t>(ctx, "qr_err", 1);
    if (!o->init_beta_rough) {
        double* part = ws<double>(ctx, "xtx_part", (size_t)xtx_blocks(dp.n) * P * (P + 1) / 2);
        LAUNCH(launch_xtx_inverse(dp.Xcm, dp.n, P, part, ginv, err, st));
        int32_t herr = 0;
        CK(cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr) fail(ctx, DEVIL_ERR_SINGULAR, "design matrix is rank deficient");
    }
    if (dp.grp.active && !o->init_beta_rough) {
        GrpGeom gg = grp_geom(dp);
        int32_t* cnt = nullptr;
        gg.act = all_genes(ctx, dp, &cnt);
        gg.n_act = cnt;
        gg.reset_next = nullptr;
        gg.gsum = ws<double>(ctx, "grp_gsum", (size_t)G * gg.S);
        gg.rowexp = ws<double>(ctx, "grp_rowexp", (size_t)G * gg.U);
        double* zb = ws<double>(ctx, "grp_zero_beta", (size_t)G * P);
        CK(cudaMemsetAsync(zb, 0, (size_t)G * P * sizeof(double), st));
        LAUNCH(launch_grp_init_beta(gg, dp.val_u16, zb, ginv, G, grp_slices_tile(G, gg.S, ctx->sm_count),
                                    fb.beta, fb.beta_f, st));
    }
    else
        LAUNCH(launch_init_beta(dp.rowptr, dp.col, dp.val, dp.val_u16, dp.Xdrm, dp.xs, dp.off,
                                ws<double>(ctx, "inv_sf", dp.n), ginv, dp.stats, G, dp.n, P,
                                o->init_beta_rough, fb.beta, fb.beta_f, st));
    const double eps = (double)(float)o->tolerance;
    dbg_mark(ctx, "init");
    run_irls(ctx, dp, fb.beta, fb.beta_f, fb.k, fb.iters, fb.status, o->max_iter, eps, o->form);
    dbg_mark(ctx, "irls");
    double* tm = nullptr;
    if (fb.theta_mom || o->overdispersion == DEVIL_OD_MOM || o->overdispersion == DEVIL_OD_MLE) {
        // MOM theta: the requested estimate, or the Newton start for MLE
        tm = fb.theta_mom ? fb.theta_mom
                          : (o->overdispersion == DEVIL_OD_MOM ? fb.theta : ws<double>(ctx, "mom_start", G));
        run_mom(ctx, dp, fb.beta_f, fb.beta, tm, o->form);
        if (o->overdispersion == DEVIL_OD_MOM && tm != fb.theta)
            CK(cudaMemcpyAsync(fb.theta, tm, G * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    dbg_mark(ctx, "mom");
    // theta_iters: NA for "old"/"MLE", 0 for MOM and FALSE (R/main.R:424-461)
    if (o->overdispersion == DEVIL_OD_MLE) {
        run_mle(ctx, dp, fb.beta_f, fb.beta, tm, fb.theta, nullptr, o->max_iter, 1, o->form);
        LAUNCH(launch_fill_i32(fb.titers, INT32_MIN, G, st));
    } else if (o->overdispersion == DEVIL_OD_NEW) {
        run_new_od(ctx, dp, fb.beta, fb.theta, fb.titers, o->max_iter, o->tolerance);
    } else {
        if (o->overdispersion == DEVIL_OD_NONE) CK(cudaMemsetAsync(fb.theta, 0, G * sizeof(double), st));
        LAUNCH(launch_fill_i32(fb.titers, 0, G, st));
    }
    dbg_mark(ctx, "mle");
    run_sandwich(ctx, dp, fb.beta_f, fb.beta, fb.theta, ends_host, n_clusters, fb.bread,
                 n_clusters > 0 ? fb.sandwich : nullptr, n_clusters > 0 ? fb.meat : nullptr,
                 o->form);
    dbg_mark(ctx, "sandwich");
    check_kernel_err(ctx);
    dbg_report(ctx);
}

void alloc_fit_buffers(devil_ctx* ctx, int64_t G, int P, bool theta_mom, bool clusters,
                       FitBuffers& fb) {
    fb.beta = ws<double>(ctx, "beta", (size_t)G * P);
    fb.beta_f = ws<float>(ctx, "beta_f", (size_t)G * P);
    fb.k = ws<float>(ctx, "k", G);
    fb.theta0 = ws<double>(ctx, "theta0", G);
    fb.theta = ws<double>(ctx, "theta", G);
    fb.theta_mom = theta_mom ? ws<double>(ctx, "theta_mom", G) : nullptr;
    fb.iters = ws<int32_t>(ctx, "iters", G);
    fb.status = ws<int32_t>(ctx, "status", G);
    fb.titers = ws<int32_t>(ctx, "titers", G);
    fb.bread = ws<double>(ctx, "bread", (size_t)G * P * P);
    fb.sandwich = clusters ? ws<double>(ctx, "sandwich", (size_t)G * P * P) : nullptr;
    fb.meat = clusters ? ws<double>(ctx, "meat_out", (size_t)G * P * P) : nullptr;
}

void validate_opts(devil_ctx* ctx, const devil_fit_opts* o) {
    if (!o) fail(ctx, DEVIL_ERR_ARG, "opts is NULL");
    if (o->overdispersion < 0 || o->overdispersion > 3)
        fail(ctx, DEVIL_ERR_UNSUPPORTED, "overdispersion mode %d not supported", o->overdispersion);
    if (o->form != DEVIL_FORM_CHOSEN && o->form != DEVIL_FORM_PLAIN)
        fail(ctx, DEVIL_ERR_ARG, "unknown form %d", o->form);
    if (o->precision == DEVIL_PREC_TC_BF16X3)
        fail(ctx, DEVIL_ERR_UNSUPPORTED,
             "precision tc_bf16x3 is not provided; DEVIL_PREC_TC_TF32 (split TF32) reaches FP32 accuracy");
    if (o->precision != DEVIL_PREC_FP32 && o->precision != DEVIL_PREC_TC_TF32)
        fail(ctx, DEVIL_ERR_ARG, "unknown precision %d", o->precision);
}

template <class F>
int guarded(devil_ctx* ctx, F&& f) {
    if (!ctx) return DEVIL_ERR_ARG;
    try {
        CK(cudaSetDevice(ctx->device));
        f();
        return DEVIL_OK;
    } catch (const Fail& e) {
        // drain what the failed call queued before the next call reuses
        // the context's workspace (the error message is kept)
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        return e.code;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        return DEVIL_ERR_ARG;
    }
}

}  // namespace

// ====================================================================
// public API
// ====================================================================
extern "C" {

const char* devil_version(void) { return "devil_b200 0.1.0 (sm_100a)"; }

void devil_fit_opts_default(devil_fit_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->max_iter = 200;
    o->tolerance = 1e-3;
    o->overdispersion = DEVIL_OD_MOM;
    o->size_factors = DEVIL_SF_NONE;
    o->form = DEVIL_FORM_CHOSEN;
}

int devil_ctx_create(int device, devil_ctx** out) {
    if (!out) return DEVIL_ERR_ARG;
    *out = nullptr;
    devil_ctx* ctx = new devil_ctx();
    ctx->device = device;
    int rc = guarded(ctx, [&] {
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        CK(cudaHostAlloc(&ctx->mapped_host, sizeof(int32_t) * 4, cudaHostAllocMapped));
        CK(cudaHostGetDevicePointer((void**)&ctx->mapped_dev, ctx->mapped_host, 0));
        for (auto& e : ctx->ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
        // the TMA-staged engine is opt-in: with CSR loads per chunk exposed it
        // measured slower than the register engine on the sparse workload
        const char* ut = getenv("DEVIL_TMA");
        ctx->use_tma = (ut && atoi(ut)) ? 1 : 0;
        // the design-group engine is on unless DEVIL_GROUPS=0 (A/B timing)
        const char* ug = getenv("DEVIL_GROUPS");
        ctx->use_groups = (ug && !atoi(ug)) ? 0 : 1;
        const char* gsl = getenv("DEVIL_GRP_SLICES");
        ctx->grp_slices = gsl ? (atoi(gsl) & 15) : 15;
        const char* dbg = getenv("DEVIL_DEBUG");
        ctx->debug = (dbg && atoi(dbg)) ? 1 : 0;
        int32_t* err = ws<int32_t>(ctx, "kernel_err", 1);
        CK(cudaMemset(err, 0, sizeof(int32_t)));
    });
    if (rc != DEVIL_OK) {
        fprintf(stderr, "devil_ctx_create: %s\n", ctx->err.c_str());
        devil_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return DEVIL_OK;
}

int devil_ctx_destroy(devil_ctx* ctx) {
    if (!ctx) return DEVIL_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->bufs)
        if (kv.second.p) cudaFree(kv.second.p);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->mapped_host) cudaFreeHost(ctx->mapped_host);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return DEVIL_OK;
}

const char* devil_last_error(const devil_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
void* devil_ctx_stream(devil_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
int devil_ctx_synchronize(devil_ctx* ctx) {
    return guarded(ctx, [&] { CK(cudaStreamSynchronize(ctx->stream)); });
}
int64_t devil_ctx_launch_count(const devil_ctx* ctx) { return ctx ? ctx->launches : 0; }

int devil_ctx_set_profiling(devil_ctx* ctx, int enable) {
    return guarded(ctx, [&] {
        prof_collect(ctx);
        ctx->profiling = enable ? 1 : 0;
        for (int k = 0; k < 4; ++k) {
            ctx->prof_launches[k] = 0;
            ctx->prof_ms[k] = 0.0;
            ctx->prof_bytes[k] = 0.0;
            ctx->prof_tc_flops[k] = 0.0;
        }
    });
}

int devil_ctx_engine(const devil_ctx* ctx, int pass_kind) {
    if (!ctx || pass_kind < 0 || pass_kind > 3) return -1;
    return ctx->last_engine[pass_kind];
}

int devil_ctx_profile(devil_ctx* ctx, int pass_kind, int64_t* launches, double* ms,
                      double* alg_bytes) {
    return guarded(ctx, [&] {
        if (pass_kind < 0 || pass_kind > 3) fail(ctx, DEVIL_ERR_ARG, "pass kind 0..3");
        prof_collect(ctx);
        if (launches) *launches = ctx->prof_launches[pass_kind];
        if (ms) *ms = ctx->prof_ms[pass_kind];
        if (alg_bytes) *alg_bytes = ctx->prof_bytes[pass_kind];
    });
}

int64_t devil_ctx_irls_rescued(const devil_ctx* ctx) { return ctx ? ctx->irls_rescued : -1; }

int devil_ctx_profile_tc(devil_ctx* ctx, int pass_kind, double* tc_flops) {
    return guarded(ctx, [&] {
        if (pass_kind < 0 || pass_kind > 3) fail(ctx, DEVIL_ERR_ARG, "pass kind 0..3");
        if (tc_flops) *tc_flops = ctx->prof_tc_flops[pass_kind];
    });
}

int devil_fit(devil_ctx* ctx, const devil_counts* counts, const double* X, int p,
              const int32_t* cluster_ends, int n_clusters, const devil_fit_opts* opts,
              devil_fit_result* res) {
    return guarded(ctx, [&] {
        validate_opts(ctx, opts);
        check_counts(ctx, counts);
        if (!X || !res || !res->beta || !res->theta || !res->beta_iters)
            fail(ctx, DEVIL_ERR_ARG, "X and result beta/theta/beta_iters are required");
        if (n_clusters > 0 && !cluster_ends) fail(ctx, DEVIL_ERR_ARG, "cluster_ends is NULL");
        DevProblem dp;
        dbg_mark(ctx, "start");
        upload_counts(ctx, counts, dp);
        dbg_mark(ctx, "upload");
        prepare_design(ctx, dp, X, p, false);
        dbg_mark(ctx, "design");
        compute_offsets(ctx, dp, opts->size_factors, opts->size_factor_values, nullptr, opts->offset);
        dbg_mark(ctx, "offsets");
        build_groups(ctx, dp, cluster_ends, n_clusters, opts->form);
        FitBuffers fb;
        alloc_fit_buffers(ctx, dp.G, p, res->theta_mom && opts->compute_theta_mom, n_clusters > 0, fb);
        fit_pipeline(ctx, dp, cluster_ends, n_clusters, opts, fb);
        const int64_t G = dp.G;
        d2h(ctx, res->beta, fb.beta, (size_t)G * p);
        d2h(ctx, res->theta, fb.theta, G);
        d2h(ctx, res->beta_iters, fb.iters, G);
        d2h(ctx, res->status, fb.status, G);
        d2h(ctx, res->bread, fb.bread, (size_t)G * p * p);
        if (n_clusters > 0) {
            d2h(ctx, res->sandwich, fb.sandwich, (size_t)G * p * p);
            d2h(ctx, res->meat, fb.meat, (size_t)G * p * p);
        }
        if (fb.theta_mom) d2h(ctx, res->theta_mom, fb.theta_mom, G);
        d2h(ctx, res->size_factors, dp.sf, dp.n);
        d2h(ctx, res->offset_vector, dp.off, dp.n);
        CK(cudaStreamSynchronize(ctx->stream));
        if (res->theta_iters) {
            CK(cudaMemcpy(res->theta_iters, fb.titers, G * sizeof(int32_t), cudaMemcpyDeviceToHost));
        }
    });
}

int devil_fit_batch(devil_ctx* ctx, int n_problems, const devil_problem* problems,
                    const devil_fit_opts* opts, devil_fit_result* results, int workers) {
    if (!ctx) return DEVIL_ERR_ARG;
    if (n_problems < 0 || (n_problems > 0 && (!problems || !results)) || !opts) {
        ctx->err = "devil_fit_batch: need problems, results and opts";
        return DEVIL_ERR_ARG;
    }
    if (n_problems == 0) return DEVIL_OK;
    workers = std::max(1, std::min(std::min(workers, 8), n_problems));
    std::vector<devil_ctx*> wc(workers, nullptr);
    for (int w = 0; w < workers; ++w) {
        const int rc = devil_ctx_create(ctx->device, &wc[w]);
        if (rc != DEVIL_OK) {
            for (auto* c : wc)
                if (c) devil_ctx_destroy(c);
            ctx->err = "devil_fit_batch: could not create a worker context";
            return rc;
        }
    }
    std::vector<int> rcs(n_problems, DEVIL_OK);
    std::vector<std::string> msgs(n_problems);
    std::atomic<int> next(0);
    auto work = [&](int w) {
        for (int i = next.fetch_add(1); i < n_problems; i = next.fetch_add(1)) {
            const devil_problem& pr = problems[i];
            rcs[i] = devil_fit(wc[w], &pr.counts, pr.X, pr.p, pr.cluster_ends, pr.n_clusters, opts,
                               &results[i]);
            if (rcs[i] != DEVIL_OK) msgs[i] = devil_last_error(wc[w]);
        }
    };
    std::vector<std::thread> th;
    for (int w = 1; w < workers; ++w) th.emplace_back(work, w);
    work(0);
    for (auto& t : th) t.join();
    for (auto* c : wc) devil_ctx_destroy(c);
    for (int i = 0; i < n_problems; ++i)
        if (rcs[i] != DEVIL_OK) {
            ctx->err = "problem " + std::to_string(i) + ": " + msgs[i];
            return rcs[i];
        }
    return DEVIL_OK;
}

int devil_fit_device(devil_ctx* ctx, const devil_counts* counts_dev, const double* X_dev, int p,
                     const int32_t* cluster_ends_host, int n_clusters, const devil_fit_opts* opts,
                     devil_fit_result* r) {
    return guarded(ctx, [&] {
        validate_opts(ctx, opts);
        if (!counts_dev || !X_dev || !r || !r->beta || !r->theta || !r->beta_iters)
            fail(ctx, DEVIL_ERR_ARG, "counts, X and result beta/theta/beta_iters are required");
        DevProblem dp;
        dbg_mark(ctx, "start");
        use_device_counts(ctx, counts_dev, dp);
        dbg_mark(ctx, "validate");
        prepare_design(ctx, dp, X_dev, p, true);
        dbg_mark(ctx, "design");
        compute_offsets(ctx, dp, opts->size_factors, nullptr, opts->size_factor_values, opts->offset);
        dbg_mark(ctx, "offsets");
        build_groups(ctx, dp, cluster_ends_host, n_clusters, opts->form);
        FitBuffers fb;
        alloc_fit_buffers(ctx, dp.G, p, r->theta_mom && opts->compute_theta_mom, n_clusters > 0, fb);
        // write straight into the caller's device buffers where given
        fb.beta = r->beta;
        fb.theta = r->theta;
        fb.iters = r->beta_iters;
        if (r->status) fb.status = r->status;
        if (r->bread) fb.bread = r->bread;
        if (r->sandwich && n_clusters > 0) fb.sandwich = r->sandwich;
        if (r->meat && n_clusters > 0) fb.meat = r->meat;
        if (r->theta_mom && opts->compute_theta_mom) fb.theta_mom = r->theta_mom;
        if (r->theta_iters) fb.titers = r->theta_iters;
        fit_pipeline(ctx, dp, cluster_ends_host, n_clusters, opts, fb);
        if (r->size_factors)
            CK(cudaMemcpyAsync(r->size_factors, dp.sf, dp.n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        if (r->offset_vector)
            CK(cudaMemcpyAsync(r->offset_vector, dp.off, dp.n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    });
}

int devil_fit_async(devil_ctx* ctx, void* stream, const devil_counts* counts_dev, const double* X_dev,
                    int p, const int32_t* cluster_ends_host, int n_clusters,
                    const devil_fit_opts* opts, devil_fit_result* r) {
    if (!ctx) return DEVIL_ERR_ARG;
    cudaStream_t own = ctx->stream;
    if (stream) ctx->stream = static_cast<cudaStream_t>(stream);
    const int rc = devil_fit_device(ctx, counts_dev, X_dev, p, cluster_ends_host, n_clusters, opts, r);
    ctx->stream = own;
    return rc;
}

// ------------------------------------------------------------------
int devil_test_de_device(devil_ctx* ctx, int64_t G, int p, const double* beta_dev,
                         const double* bread_dev, const double* sandwich_dev, int64_t n_samples,
                         const double* contrast_host, int adjust_method, double max_lfc,
                         double* pval_dev, double* adj_dev, double* lfc_dev) {
    return guarded(ctx, [&] {
        if (p < 1 || p > 64 || !contrast_host) fail(ctx, DEVIL_ERR_ARG, "bad p or contrast");
        if (adjust_method < 0 || adjust_method > DEVIL_ADJ_HOMMEL) fail(ctx, DEVIL_ERR_UNSUPPORTED, "adjust method");
        double* c = ws<double>(ctx, "contrast", p);
        h2d(ctx, c, contrast_host, p);
        LAUNCH(launch_test_pvalues(G, p, beta_dev, bread_dev, sandwich_dev, (double)(n_samples - 2), c,
                                   max_lfc, pval_dev, lfc_dev, ctx->stream));
        size_t tb = p_adjust_temp_bytes(G);
        void* tmp = ws<char>(ctx, "padj_tmp", tb);
        LAUNCH(launch_p_adjust(G, pval_dev, adjust_method, adj_dev, tmp, tb, ctx->stream));
        ctx->launches += 2;
        CK(cudaStreamSynchronize(ctx->stream));  // contrast upload source
    });
}

int devil_test_de(devil_ctx* ctx, int64_t G, int p, const double* beta, const double* bread,
                  const double* sandwich, int64_t n_samples, const double* contrast,
                  int adjust_method, double max_lfc, double* pval, double* adj_pval, double* lfc) {
    return guarded(ctx, [&] {
        if (!beta || !bread || !pval || !adj_pval || !lfc) fail(ctx, DEVIL_ERR_ARG, "null argument");
        double* b = ws<double>(ctx, "t_beta", (size_t)G * p);
        double* br = ws<double>(ctx, "t_bread", (size_t)G * p * p);
        double* sw = sandwich ? ws<double>(ctx, "t_sw", (size_t)G * p * p) : nullptr;
        double* pv = ws<double>(ctx, "t_p", G);
        double* pa = ws<double>(ctx, "t_pa", G);
        double* lf = ws<double>(ctx, "t_lfc", G);
        h2d(ctx, b, beta, (size_t)G * p);
        h2d(ctx, br, bread, (size_t)G * p * p);
        if (sw) h2d(ctx, sw, sandwich, (size_t)G * p * p);
        int rc = devil_test_de_device(ctx, G, p, b, br, sw, n_samples, contrast, adjust_method,
                                      max_lfc, pv, pa, lf);
        if (rc != DEVIL_OK) throw Fail{rc};
        d2h(ctx, pval, pv, G);
        d2h(ctx, adj_pval, pa, G);
        d2h(ctx, lfc, lf, G);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_p_adjust(devil_ctx* ctx, int64_t m, const double* p, int method, double* out) {
    return guarded(ctx, [&] {
        if (method < 0 || method > DEVIL_ADJ_HOMMEL) fail(ctx, DEVIL_ERR_UNSUPPORTED, "adjust method");
        double* pd = ws<double>(ctx, "pa_in", m);
        double* od = ws<double>(ctx, "pa_out", m);
        h2d(ctx, pd, p, m);
        size_t tb = p_adjust_temp_bytes(m);
        void* tmp = ws<char>(ctx, "padj_tmp", tb);
        LAUNCH(launch_p_adjust(m, pd, method, od, tmp, tb, ctx->stream));
        d2h(ctx, out, od, m);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_p_adjust_device(devil_ctx* ctx, int64_t m, const double* p_dev, int method,
                          double* out_dev) {
    return guarded(ctx, [&] {
        if (method < 0 || method > DEVIL_ADJ_HOMMEL) fail(ctx, DEVIL_ERR_UNSUPPORTED, "adjust method");
        size_t tb = p_adjust_temp_bytes(m);
        void* tmp = ws<char>(ctx, "padj_tmp", tb);
        LAUNCH(launch_p_adjust(m, p_dev, method, out_dev, tmp, tb, ctx->stream));
    });
}

// ------------------------------------------------------------------
// single steps
// ------------------------------------------------------------------
int devil_calculate_sf(devil_ctx* ctx, const devil_counts* counts, int method, double* sf) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        if (method != DEVIL_SF_NORMED_SUM && method != DEVIL_SF_PSINORM)
            fail(ctx, DEVIL_ERR_ARG, "'arg' should be one of \"normed_sum\", \"psinorm\"");
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        compute_offsets(ctx, dp, method, nullptr, nullptr, 0.0);
        d2h(ctx, sf, dp.sf, dp.n);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

static void upload_offsets(devil_ctx* ctx, DevProblem& dp, const double* offv_host) {
    dp.sf = ws<double>(ctx, "sf", dp.n);
    dp.off = ws<double>(ctx, "off", dp.n);
    dp.off_f = ws<float>(ctx, "off_f", dp.n + 16);
    CK(cudaMemsetAsync(dp.off_f + dp.n, 0, 16 * sizeof(float), ctx->stream));
    h2d(ctx, dp.off, offv_host, dp.n);
    LAUNCH(launch_double_to_float(dp.off, dp.off_f, dp.n, ctx->stream));
}
static void upload_sf_as_offsets(devil_ctx* ctx, DevProblem& dp, const double* sf_host) {
    compute_offsets(ctx, dp, DEVIL_SF_GIVEN, sf_host, nullptr, 0.0);
}

int devil_estimate_dispersion(devil_ctx* ctx, const devil_counts* counts,
                              const double* offset_vector, double* theta0) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        dp.stats = ws<double>(ctx, "stats", (size_t)dp.G * 6);
        LAUNCH(launch_gene_stats(dp.rowptr, dp.val, dp.val_u16, dp.G, dp.n, dp.stats, ctx->stream));
        upload_offsets(ctx, dp, offset_vector);
        double* th = ws<double>(ctx, "theta0", dp.G);
        float* k = ws<float>(ctx, "k", dp.G);
        LAUNCH(launch_theta0(dp.stats, dp.off, dp.G, dp.n, 0, 0.0, th, k, ctx->stream));
        d2h(ctx, theta0, th, dp.G);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_init_beta(devil_ctx* ctx, const devil_counts* counts, const double* X, int p,
                    const double* offset_vector, int rough, double* beta0) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        prepare_design(ctx, dp, X, p, false);
        upload_offsets(ctx, dp, offset_vector);
        double* ginv = ws<double>(ctx, "ginv", (size_t)p * p);
        int32_t* err = ws<int32_t>(ctx, "qr_err", 1);
        if (!rough) {
            double* part = ws<double>(ctx, "xtx_part", (size_t)xtx_blocks(dp.n) * p * (p + 1) / 2);
            LAUNCH(launch_xtx_inverse(dp.Xcm, dp.n, p, part, ginv, err, ctx->stream));
            int32_t herr = 0;
            CK(cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            if (herr) fail(ctx, DEVIL_ERR_SINGULAR, "design matrix is rank deficient");
        }
        double* b = ws<double>(ctx, "beta", (size_t)dp.G * p);
        float* bf = ws<float>(ctx, "beta_f", (size_t)dp.G * p);
        LAUNCH(launch_init_beta(dp.rowptr, dp.col, dp.val, dp.val_u16, dp.Xdrm, dp.xs, dp.off,
                                ws<double>(ctx, "inv_sf", dp.n), ginv, dp.stats, dp.G, dp.n, p,
                                rough, b, bf, ctx->stream));
        d2h(ctx, beta0, b, (size_t)dp.G * p);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_beta_fit(devil_ctx* ctx, const devil_counts* counts, const double* X, int p,
                   const double* beta0, const double* offset_vector, const double* theta0,
                   int max_iter, double eps, int form, double* beta, int32_t* iters) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        prepare_design(ctx, dp, X, p, false);
        upload_offsets(ctx, dp, offset_vector);
        build_groups(ctx, dp, nullptr, 0, form);
        const int64_t G = dp.G;
        double* b = ws<double>(ctx, "beta", (size_t)G * p);
        float* bf = ws<float>(ctx, "beta_f", (size_t)G * p);
        double* th = ws<double>(ctx, "theta0", G);
        float* k = ws<float>(ctx, "k", G);
        h2d(ctx, b, beta0, (size_t)G * p);
        h2d(ctx, th, theta0, G);
        LAUNCH(launch_double_to_float(b, bf, (size_t)G * p, ctx->stream));
        // k = 1/theta0 with theta0 rounded to float (src/beta.cpp:25-28)
        std::vector<float> hk(G);
        for (int64_t g = 0; g < G; ++g) hk[g] = (float)(1.0 / (double)(float)theta0[g]);
        h2d(ctx, k, hk.data(), G);
        int32_t* it = ws<int32_t>(ctx, "iters", G);
        int32_t* stt = ws<int32_t>(ctx, "status", G);
        run_irls(ctx, dp, b, bf, k, it, stt, max_iter, (double)(float)eps, form);
        check_kernel_err(ctx);
        d2h(ctx, beta, b, (size_t)G * p);
        d2h(ctx, iters, it, G);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

static void upload_beta(devil_ctx* ctx, const DevProblem& dp, const double* beta, float** bf_out,
                        double** bd_out) {
    double* b = ws<double>(ctx, "beta", (size_t)dp.G * dp.P);
    float* bf = ws<float>(ctx, "beta_f", (size_t)dp.G * dp.P);
    h2d(ctx, b, beta, (size_t)dp.G * dp.P);
    LAUNCH(launch_double_to_float(b, bf, (size_t)dp.G * dp.P, ctx->stream));
    *bf_out = bf;
    *bd_out = b;
}

int devil_estimate_mom_dispersion(devil_ctx* ctx, const devil_counts* counts, const double* X,
                                  int p, const double* beta, const double* size_factors,
                                  double* theta) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        prepare_design(ctx, dp, X, p, false);
        upload_sf_as_offsets(ctx, dp, size_factors);
        build_groups(ctx, dp, nullptr, 0, DEVIL_FORM_CHOSEN);
        float* bf;
        double* bd;
        upload_beta(ctx, dp, beta, &bf, &bd);
        double* th = ws<double>(ctx, "theta", dp.G);
        run_mom(ctx, dp, bf, bd, th, DEVIL_FORM_CHOSEN);
        d2h(ctx, theta, th, dp.G);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_fit_dispersion(devil_ctx* ctx, const devil_counts* counts, const double* X, int p,
                         const double* beta, const double* offset_vector, int max_iter, int cox_reid,
                         double* theta, int32_t* newton_iters) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        prepare_design(ctx, dp, X, p, false);
        upload_offsets(ctx, dp, offset_vector);
        build_groups(ctx, dp, nullptr, 0, DEVIL_FORM_CHOSEN);
        float* bf;
        double* bd;
        upload_beta(ctx, dp, beta, &bf, &bd);
        double* th = ws<double>(ctx, "theta", dp.G);
        int32_t* it = ws<int32_t>(ctx, "mle_iters_out", dp.G);
        // MOM at beta (size factors exp(offset)) seeds the Newton search
        double* tm = ws<double>(ctx, "mom_start", dp.G);
        run_mom(ctx, dp, bf, bd, tm, DEVIL_FORM_CHOSEN);
        run_mle(ctx, dp, bf, bd, tm, th, it, max_iter, cox_reid, DEVIL_FORM_CHOSEN);
        check_kernel_err(ctx);
        d2h(ctx, theta, th, dp.G);
        d2h(ctx, newton_iters, it, dp.G);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_fit_overdispersion_new(devil_ctx* ctx, const devil_counts* counts, const double* X,
                                 int p, const double* beta, const double* offset_vector,
                                 int max_iter, double eps_theta, double* theta,
                                 int32_t* kappa_iters) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        if (!X || !beta || !offset_vector || !theta) fail(ctx, DEVIL_ERR_ARG, "missing argument");
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        prepare_design(ctx, dp, X, p, false);
        upload_offsets(ctx, dp, offset_vector);
        float* bf;
        double* bd;
        upload_beta(ctx, dp, beta, &bf, &bd);
        double* th = ws<double>(ctx, "theta", dp.G);
        int32_t* it = ws<int32_t>(ctx, "nod_iters_out", dp.G);
        run_new_od(ctx, dp, bd, th, it, max_iter, eps_theta);
        d2h(ctx, theta, th, dp.G);
        d2h(ctx, kappa_iters, it, dp.G);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_compute_hessian(devil_ctx* ctx, const devil_counts* counts, const double* X, int p,
                          const double* beta, const double* overdispersion,
                          const double* size_factors, double* bread) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        prepare_design(ctx, dp, X, p, false);
        upload_sf_as_offsets(ctx, dp, size_factors);
        build_groups(ctx, dp, nullptr, 0, DEVIL_FORM_CHOSEN);
        float* bf;
        double* bd;
        upload_beta(ctx, dp, beta, &bf, &bd);
        double* th = ws<double>(ctx, "theta", dp.G);
        h2d(ctx, th, overdispersion, dp.G);
        double* br = ws<double>(ctx, "bread", (size_t)dp.G * p * p);
        run_sandwich(ctx, dp, bf, bd, th, nullptr, 0, br, nullptr, nullptr, DEVIL_FORM_CHOSEN);
        d2h(ctx, bread, br, (size_t)dp.G * p * p);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_compute_clustered_meat(devil_ctx* ctx, const devil_counts* counts, const double* X,
                                 int p, const double* beta, const double* overdispersion,
                                 const double* size_factors, const int32_t* cluster_ends,
                                 int n_clusters, double* meat) {
    return guarded(ctx, [&] {
        check_counts(ctx, counts);
        if (n_clusters < 1 || !cluster_ends) fail(ctx, DEVIL_ERR_ARG, "need cluster ends");
        DevProblem dp;
        upload_counts(ctx, counts, dp);
        prepare_design(ctx, dp, X, p, false);
        upload_sf_as_offsets(ctx, dp, size_factors);
        build_groups(ctx, dp, cluster_ends, n_clusters, DEVIL_FORM_CHOSEN);
        float* bf;
        double* bd;
        upload_beta(ctx, dp, beta, &bf, &bd);
        double* th = ws<double>(ctx, "theta", dp.G);
        h2d(ctx, th, overdispersion, dp.G);
        double* br = ws<double>(ctx, "bread", (size_t)dp.G * p * p);
        double* mt = ws<double>(ctx, "meat", (size_t)dp.G * p * p);
        run_sandwich(ctx, dp, bf, bd, th, cluster_ends, n_clusters, br, nullptr, mt, DEVIL_FORM_CHOSEN);
        d2h(ctx, meat, mt, (size_t)dp.G * p * p);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

int devil_nb_adjoint(devil_ctx* ctx, int64_t n, const double* y, const double* eta,
                     double log_theta, double* loglik, double* d_eta, double* d_log_theta) {
    return guarded(ctx, [&] {
        if (n < 0 || !y || !eta) fail(ctx, DEVIL_ERR_ARG, "null argument");
        double* yd = ws<double>(ctx, "adj_y", n);
        double* ed = ws<double>(ctx, "adj_eta", n);
        double* l = ws<double>(ctx, "adj_l", n);
        double* de = ws<double>(ctx, "adj_de", n);
        double* dt = ws<double>(ctx, "adj_dt", n);
        h2d(ctx, yd, y, n);
        h2d(ctx, ed, eta, n);
        LAUNCH(launch_nb_adjoint(n, yd, ed, log_theta, l, de, dt, ctx->stream));
        d2h(ctx, loglik, l, n);
        d2h(ctx, d_eta, de, n);
        d2h(ctx, d_log_theta, dt, n);
        CK(cudaStreamSynchronize(ctx->stream));
    });
}

// ------------------------------------------------------------------
// cluster handling on the host (R's factor / is.unsorted / rle / order)
// ------------------------------------------------------------------
int devil_cluster_blocks(int64_t n, const int64_t* clusters, int32_t* levels, int32_t* ends,
                         int* n_blocks) {
    if (n < 0 || (n > 0 && (!clusters || !levels || !ends)) || !n_blocks) return DEVIL_ERR_ARG;
    std::unordered_map<int64_t, int32_t> lev;
    lev.reserve(64);
    for (int64_t c = 0; c < n; ++c) {
        auto it = lev.find(clusters[c]);
        int32_t v;
        if (it == lev.end()) {
            v = (int32_t)lev.size() + 1;
            lev.emplace(clusters[c], v);
        } else {
            v = it->second;
        }
        levels[c] = v;
    }
    for (int64_t c = 1; c < n; ++c)
        if (levels[c] < levels[c - 1]) return DEVIL_ERR_UNSORTED;
    int nb = 0;
    for (int64_t c = 0; c < n; ++c)
        if (c == n - 1 || levels[c + 1] != levels[c]) ends[nb++] = (int32_t)(c + 1);
    *n_blocks = nb;
    return DEVIL_OK;
}

int devil_group_order(int64_t n, const int64_t* clusters, int64_t* order) {
    if (n < 0 || (n > 0 && (!clusters || !order))) return DEVIL_ERR_ARG;
    std::unordered_map<int64_t, int32_t> lev;
    std::vector<int32_t> levels(n);
    for (int64_t c = 0; c < n; ++c) {
        auto it = lev.find(clusters[c]);
        if (it == lev.end()) {
            int32_t v = (int32_t)lev.size();
            lev.emplace(clusters[c], v);
            levels[c] = v;
        } else {
            levels[c] = it->second;
        }
    }
    std::vector<int64_t> cnt(lev.size() + 1, 0);
    for (int64_t c = 0; c < n; ++c) cnt[levels[c] + 1]++;
    for (size_t i = 1; i < cnt.size(); ++i) cnt[i] += cnt[i - 1];
    for (int64_t c = 0; c < n; ++c) order[cnt[levels[c]]++] = c;  // stable counting sort
    return DEVIL_OK;
}

}  // extern "C"
