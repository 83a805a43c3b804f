// IRLS cell pass with the Hessian's dense part on the tensor cores (sm_100a
// tcgen05, kind::tf32), p <= 4.
//
// One IRLS pass accumulates, per gene, outer0 = sum_c r_c z_c over every
// cell (z_c = the products x_i x_j of the cell's design row, r_c = 1/(mu_c
// + k)) plus corrections at the gene's nonzeros, and vec0 = sum mu r x - ...
// (PassIRLS in passes.cuh; src/beta.cpp:35-42).  For a tile of 128 genes
// and a chunk of 32 cells the dense part is the product
//     D[128 genes x 16] += R[128 genes x 32 cells] * Z[16 x 32 cells]^T
// with R computed by the CUDA cores (exp, reciprocal) and Z (the products,
// padded to 16 rows) precomputed once per fit.  R and Z are staged in
// shared memory in the canonical K-major layout without swizzle, one
// thread issues the MMAs, D lives in tensor memory (128 lanes x FP32
// columns) and is read back with tcgen05.ld at the end.
//
// Precision: an FP32 value v enters as two TF32 numbers, hi = rna(v) and
// lo = rna(v - hi) (10-bit mantissas each), so R Z^T is computed as
//     (R_hi + R_lo) [Z_hi; Z_lo]^T   (two MMAs with N = 32)
// whose four partial products sum to R Z^T with a relative error near
// 2^-21 per term, FP32 accumulation.  A single TF32 rounding is not enough:
// for weakly expressed genes r = 1/(mu + k) is almost the same in every
// cell, its rounding error does not average out, and a Hessian wrong by
// 2^-11 changes the path of slowly converging IRLS runs.  The score
// (vec0), which fixes the solution, stays on the CUDA cores in FP32, as do
// the nonzero corrections.
//
// Pipeline per block: two shared-memory stages (R and Z of a chunk); before
// a stage is rewritten the block waits for the commit of the MMAs that read
// it (mbarrier, bounded wait).  All waits are bounded: on expiry the block
// records an error, skips its output, drains and frees its tensor memory.
#include "internal.h"
#include "tc_common.cuh"

#include <cstdlib>

namespace devil {

namespace {

constexpr int kTcM = 128;                      // genes per block tile (MMA M)
constexpr int kTcZ = 16;                       // product rows, zero padded
constexpr int kTcN = 2 * kTcZ;                 // MMA N: Z_hi rows then Z_lo rows
constexpr int kTcKC = 32;                      // cells per chunk (4 K-steps of 8)
constexpr int kTcNT = 256;                     // threads per block
constexpr int kTcABytes = kTcM * kTcKC * 4;    // one R_hi or R_lo stage, 16 KB
constexpr int kTcBBytes = kTcN * kTcKC * 4;    // one Z stage, 4 KB
constexpr int kTcStage = 2 * kTcABytes;        // R_hi and R_lo of one chunk
// input stages (4, filled two chunks ahead by cp.async): Z of the chunk, its
// 32 design rows (<= 4 floats each) and offsets
constexpr int kTcInX = kTcBBytes;              // 4096
constexpr int kTcInOff = kTcInX + kTcKC * 16;  // 4608
constexpr int kTcInBytes = kTcInOff + kTcKC * 4;
constexpr int kTcSmem = 2 * kTcStage + 4 * kTcInBytes;  // 82.5 KB
// D is accumulated in runs of kTcRun chunks (128 cells) and each run is
// added into FP32 registers: a long accumulation inside tensor memory loses
// low-order bits of every addend once the sum is much larger than it, a
// bias that would grow with the cell count.  Runs alternate between two
// regions of 64 columns (D_hi: R_hi [Z_hi; Z_lo], D_lo: R_lo [Z_hi; Z_lo]),
// so one region is read while the MMAs of the next run fill the other.
constexpr int kTcRun = 4;
constexpr uint32_t kTcRegion = 2 * kTcN;       // columns of one region
constexpr uint32_t kTcCols = 2 * kTcRegion;    // 128 columns allocated

static_assert(kTcN * kTcKC / 4 == kTcNT, "one 16-byte piece of Z per thread and chunk");
static_assert(kTcKC / 4 == kTcNT / 32, "one quad of cells per warp and chunk");

constexpr uint32_t kIdesc = tf32_idesc(kTcM, kTcN);

DEV void tc_mma(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t accumulate) {
    tc_mma_n(tmem, ad, bd, accumulate, kIdesc);
}

// add two of the four 16-column parts of one region (rows of this warp's
// lanes): parts 0, 1 (R_hi against Z_hi, Z_lo) or parts 2, 3 (R_lo)
DEV void tc_drain(uint32_t taddr, float* h) {
#pragma unroll
    for (int part = 0; part < 2; ++part) {
        float t[16];
        tc_ld16(taddr + (uint32_t)(16 * part), t);
#pragma unroll
        for (int a = 0; a < 16; ++a) h[a] += t[a];
    }
}

template <int P, class VT>
__global__ void __launch_bounds__(kTcNT) tc_irls_kernel(PassGeom geo, PassIRLS::Params prm,
                                                       const float4* __restrict__ zimg) {
    constexpr int NE = P * (P + 1) / 2;
    constexpr int NA = NE + P;
    constexpr int PP = P <= 1 ? 1 : (P <= 2 ? 2 : 4);
    static_assert(NE <= kTcZ, "products fit the MMA's N");
    static_assert((8 * kTcM * P + kTcM * NA + kTcM * 16) * 4 <= kTcStage,
                  "the final reductions fit the first R stage");
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tslot;
    __shared__ int abort_flag;

    if (geo.reset_next && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *geo.reset_next = 0;
    const int nact = *geo.n_act;
    const int tile = blockIdx.y;
    if (tile * kTcM >= nact) return;
    const int seg = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const VT* __restrict__ val = static_cast<const VT*>(geo.val);

    // dense phase: this thread's genes are tile slots 32 j + lane, j = 0..3
    float beta[4][P];
    float kk[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int slot = tile * kTcM + 32 * j + lane;
        if (slot >= nact) slot = tile * kTcM;  // duplicate a valid gene; not written
        const int g = __ldg(geo.act + slot);
#pragma unroll
        for (int i = 0; i < P; ++i) beta[j][i] = __ldg(prm.beta + (int64_t)g * P + i) * kLog2e;
        kk[j] = __ldg(prm.k + g);
    }
    const int nfs = geo.nbound - 1;
    const int b0 = (int)(((int64_t)seg * nfs) / geo.nseg);
    const int b1 = (int)(((int64_t)(seg + 1) * nfs) / geo.nseg);
    const int c0 = __ldg(geo.bound + b0), c1 = __ldg(geo.bound + b1);

    // inputs of chunk kc into input stage kc & 3: Z (8 quads x 32 rows x 16
    // bytes, already in stage order), the 32 design rows and the offsets.
    // Chunks never straddle a segment end except the last one of the cells
    // (segment ends are multiples of 2048 cells, or n): rows and offsets of
    // cells at or beyond c1 are zero-filled, so those cells add x = 0 to the
    // score and meet Z = 0 (the image is zero past n) in the Hessian.
    auto in_stage = [&](int s) { return tc_smem + 2 * kTcStage + s * kTcInBytes; };
    auto fetch_inputs = [&](int kc) {
        unsigned char* ib = in_stage(kc & 3);
        const int cs = c0 + kc * kTcKC;
        cp_async<16>(ib + tid * 16, zimg + (int64_t)(cs >> 2) * kTcN + tid);
        constexpr int NX = kTcKC * PP / 4;  // 16-byte pieces of the design rows
        constexpr int CPX = 4 / PP;         // cells per piece
        if (tid < NX) {
            const int cell = cs + tid * CPX;
            const int valid = min(max(c1 - cell, 0), CPX);
            cp_async_zfill(ib + kTcInX + tid * 16, valid ? (const void*)(geo.X + (int64_t)cell * PP) : geo.X,
                           (uint32_t)(valid * PP * 4));
        } else if (tid >= 64 && tid < 64 + kTcKC / 4) {
            const int pc = tid - 64;
            const int cell = cs + 4 * pc;
            const int valid = min(max(c1 - cell, 0), 4);
            cp_async_zfill(ib + kTcInOff + pc * 16, valid ? (const void*)(geo.off + cell) : geo.off,
                           (uint32_t)(valid * 4));
        }
    };
    const int nchunk0 = (c1 - c0 + kTcKC - 1) / kTcKC;
    if (nchunk0 > 0) fetch_inputs(0);
    cp_async_commit();
    if (nchunk0 > 1) fetch_inputs(1);
    cp_async_commit();
    cp_async_wait<1>();  // chunk 0 has landed (visible to all after the barrier below)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");

    if (tid == 0) {
        abort_flag = 0;
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tslot)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;

    float vacc[4][P];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < P; ++i) vacc[j][i] = 0.f;
    // Hessian row of slot 32 (warp & 3) + lane: the drained runs; warps 0..3
    // add the R_hi columns, warps 4..7 the R_lo columns of the same rows
    float hacc[16];
#pragma unroll
    for (int a = 0; a < 16; ++a) hacc[a] = 0.f;
    const uint32_t lanes = ((uint32_t)(32 * (warp & 3)) << 16) + (warp < 4 ? 0u : (uint32_t)kTcN);
    int drained = 0;  // runs added into hacc (the same in every thread)

    const int nchunk = (c1 - c0 + kTcKC - 1) / kTcKC;
    int issued = 0;  // chunks whose MMAs were committed (the same in every thread)
    for (int k = 0; k < nchunk; ++k) {
        const int st = k & 1;
        // chunk k - 2 has completed: R stage st and input stage (k + 2) & 3
        // are free again
        bool ok = true;
        if (k >= 2) {
            ok = mbar_wait_bounded(&bars[st], (uint32_t)(((k >> 1) - 1) & 1));
            if (!ok) atomicExch(&abort_flag, 1);
        }
        ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld below is warp-collective
        // when chunk k - 2 closed a run, read that run's region (the MMAs in
        // flight write the other one)
        if (k >= 2 && (k - 2) % kTcRun == kTcRun - 1) {
            if (ok) tc_drain(tmem + lanes + kTcRegion * (uint32_t)(drained & 1), hacc);
            ++drained;
        }
        if (k + 2 < nchunk) fetch_inputs(k + 2);
        cp_async_commit();  // one group per chunk, empty past the end
        unsigned char* sAh = tc_smem + st * kTcStage;
        unsigned char* sAl = sAh + kTcABytes;
        const unsigned char* ib = in_stage(k & 3);
        const float* xs = reinterpret_cast<const float*>(ib + kTcInX);
        const float* os = reinterpret_cast<const float*>(ib + kTcInOff);
        // R of the chunk: warp w fills quad w for all 128 genes
        {
            const int q = warp;
            float rv[4][4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                float x[P];
#pragma unroll
                for (int i = 0; i < P; ++i) x[i] = xs[(4 * q + t) * PP + i];
                const float o = os[4 * q + t] * kLog2e;
                float e[4] = {o, o, o, o};
#pragma unroll
                for (int i = 0; i < P; ++i) {
                    fma_x2(e[0], e[1], x[i], beta[0][i], beta[1][i]);
                    fma_x2(e[2], e[3], x[i], beta[2][i], beta[3][i]);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float mu = ex2_approx(e[j]);
                    const float r = rcp_approx(mu + kk[j]);
                    const float w = mu * r;
                    if constexpr (P >= 2) {
#pragma unroll
                        for (int i = 0; i + 1 < P; i += 2) fma_x2(vacc[j][i], vacc[j][i + 1], w, x[i], x[i + 1]);
                    }
                    if constexpr (P & 1) vacc[j][P - 1] = fmaf(w, x[P - 1], vacc[j][P - 1]);
                    rv[j][t] = r;
                }
            }
            // r = hi + lo exactly: hi keeps the TF32 bits of r, lo = r - hi
            // (the tensor core reads lo's leading 10 mantissa bits)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float hi[4], lo[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    hi[t] = __uint_as_float(__float_as_uint(rv[j][t]) & 0xFFFFE000u);
                    lo[t] = rv[j][t] - hi[t];
                }
                const int off = stage_off(32 * j + lane, q, kTcM);
                *reinterpret_cast<float4*>(sAh + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
                *reinterpret_cast<float4*>(sAl + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
            }
        }
        cp_async_wait<1>();  // this thread's copies for chunk k + 1 have landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();  // the drain's tensor-memory reads precede later MMAs
        __syncthreads();
        if (abort_flag) break;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t dreg = tmem + kTcRegion * (uint32_t)((k / kTcRun) & 1);
            const uint32_t sB = smem_u32(ib);
#pragma unroll
            for (int s = 0; s < kTcKC / 8; ++s) {
                const uint32_t acc = (k % kTcRun != 0 || s > 0) ? 1u : 0u;
                const uint64_t bd = umma_desc(sB + s * 2 * kTcN * 16, kTcN * 16, 128);
                const uint64_t ah = umma_desc(smem_u32(sAh) + s * 2 * kTcM * 16, kTcM * 16, 128);
                const uint64_t al = umma_desc(smem_u32(sAl) + s * 2 * kTcM * 16, kTcM * 16, 128);
                tc_mma(dreg, ah, bd, acc);                   // R_hi [Z_hi; Z_lo]
                tc_mma(dreg + (uint32_t)kTcN, al, bd, acc);  // R_lo [Z_hi; Z_lo]
            }
            tc_commit(&bars[st]);
        }
        issued = k + 1;
    }
    cp_async_wait<0>();  // no copy may land after the stages are reused below
    // the last commit completes after every MMA of the block; wait for it
    // on the error path too, so that no MMA is in flight when the tensor
    // memory is freed
    if (issued > 0 &&
        !mbar_wait_bounded(&bars[(issued - 1) & 1], (uint32_t)(((issued - 1) >> 1) & 1)))
        atomicExch(&abort_flag, 1);
    tc_fence_after();
    __syncthreads();  // abort_flag is final for the block from here on
    // runs not drained inside the loop (at most the last two, in different
    // regions); every MMA has completed
    if (!abort_flag) {
        const int runs = (issued + kTcRun - 1) / kTcRun;
        for (; drained < runs; ++drained)
            tc_drain(tmem + lanes + kTcRegion * (uint32_t)(drained & 1), hacc);
    }
    __syncthreads();

    // score partials of the 8 warps, then the nonzero corrections; both in
    // the (now idle) first R stage
    float* red = reinterpret_cast<float*>(tc_smem);  // [8 warps][128 slots][P]
    float* spar = red + 8 * kTcM * P;                 // [128 slots][NA]
    float* hlo = spar + kTcM * NA;                    // [128 slots][16]: R_lo columns
    if (warp >= 4) {
#pragma unroll
        for (int a = 0; a < 16; ++a) hlo[(32 * (warp - 4) + lane) * 16 + a] = hacc[a];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < P; ++i) red[(warp * kTcM + 32 * j + lane) * P + i] = vacc[j][i];

    // nonzero corrections (PassIRLS::sparse): warp w takes slots w, w + 8, ...
    for (int sidx = warp; sidx < kTcM; sidx += 8) {
        int slot = tile * kTcM + sidx;
        if (slot >= nact) slot = tile * kTcM;
        const int g = __ldg(geo.act + slot);
        float bg[P];
#pragma unroll
        for (int i = 0; i < P; ++i) bg[i] = __ldg(prm.beta + (int64_t)g * P + i) * kLog2e;
        const float kg = __ldg(prm.k + g), rk = 1.f / kg;
        float acc[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) acc[a] = 0.f;
        const int64_t* sp = geo.segptr + (int64_t)g * geo.nbound;
        const int64_t e0 = __ldg(sp + b0), e1 = __ldg(sp + b1);
        constexpr int SU = 4;  // entries in flight per lane
        for (int64_t eb = e0 + lane; eb < e1; eb += 32 * SU) {
            int cc[SU];
            float yy[SU];
            bool ok[SU];
#pragma unroll
            for (int u = 0; u < SU; ++u) {
                const int64_t e = eb + 32 * u;
                ok[u] = e < e1;
                cc[u] = ok[u] ? __ldg(geo.col + e) : c0;
                yy[u] = ok[u] ? load_val(val, e) : 0.f;
            }
            float xr[SU][P], ol[SU];
#pragma unroll
            for (int u = 0; u < SU; ++u) {
                load_row<P, PP>(geo.X, cc[u], xr[u]);
                ol[u] = __ldg(geo.off + cc[u]);
            }
#pragma unroll
            for (int u = 0; u < SU; ++u) {
                if (!ok[u]) continue;
                float el = ol[u] * kLog2e;
#pragma unroll
                for (int i = 0; i < P; ++i) el = fmaf(xr[u][i], bg[i], el);
                const float mu = ex2_approx(el);
                const float r = rcp_approx(mu + kg);
                const float yr = yy[u] * r;
                const float wh = yr * rk;  // rk scales H only, not the score
#pragma unroll
                for (int jj = 0; jj < P; ++jj)
#pragma unroll
                    for (int ii = 0; ii <= jj; ++ii)
                        acc[tri_index(ii, jj)] = fmaf(wh, xr[u][ii] * xr[u][jj], acc[tri_index(ii, jj)]);
#pragma unroll
                for (int i = 0; i < P; ++i) acc[NE + i] = fmaf(-yr, xr[u][i], acc[NE + i]);
            }
        }
#pragma unroll
        for (int a = 0; a < NA; ++a) acc[a] = warp_sum(acc[a]);
        if (lane == 0) {
#pragma unroll
            for (int a = 0; a < NA; ++a) spar[sidx * NA + a] = acc[a];
        }
    }
    __syncthreads();

    // outputs: warps 0..3 read the Hessian rows of slots 32 w + lane
    if (warp < 4) {
        const int sidx = 32 * warp + lane;
        float h[16];
#pragma unroll
        for (int a = 0; a < 16; ++a) h[a] = hacc[a] + hlo[sidx * 16 + a];
        const int slot = tile * kTcM + sidx;
        if (slot < nact && !abort_flag) {
            float* out = static_cast<float*>(geo.partW) + ((int64_t)seg * geo.slot_stride + slot) * NA;
#pragma unroll
            for (int a = 0; a < NE; ++a) out[a] = h[a] + spar[sidx * NA + a];
#pragma unroll
            for (int i = 0; i < P; ++i) {
                float v = spar[sidx * NA + NE + i];
#pragma unroll
                for (int w = 0; w < 8; ++w) v += red[(w * kTcM + sidx) * P + i];
                out[NE + i] = v;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols)
                     : "memory");
    if (abort_flag && tid == 0) atomicExch(geo.err, 1);
}

// ---------------------------------------------------------------------
// MLE pass (PassMLE in passes.cuh; src/overdispersion.cpp:95-242): the
// Cox-Reid matrices b = X' diag(w) X, db = X' diag(-w^2) X and
// d2b = X' diag(2 w^3) X (w = mu / (1 + mu theta)) on the tensor cores.
// A tile is 32 genes; the MMA's 128 rows are the three weights of the 32
// genes (rows 32 b + gene, b = 0, 1, 2) and 32 zero rows.  One thread per
// (gene, quad of cells) computes the weights and the two FP32 scalar sums
// of the dense terms; the nonzero terms (FP64, per-gene digamma tables)
// run after the cell loop, a warp per gene.  Per K-step two MMAs:
//     D[0..31]  += R_hi [Z_hi; Z_lo]      (N = 32)
//     D[0..15]  += R_lo  Z_hi              (N = 16; R_lo Z_lo ~ 2^-22 dropped)
// so a run region is 32 columns and the Hessian-like sums are columns
// 0..15 plus 16..31.
// ---------------------------------------------------------------------
constexpr int kMleG = 32;                    // genes per tile
constexpr uint32_t kMleRegion = kTcN;        // 32 columns per run region
constexpr uint32_t kMleCols = 2 * kMleRegion;
constexpr uint32_t kIdesc16 = tf32_idesc(kTcM, kTcZ);

struct ScalAcc {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    template <int K>
    DEV void scal(double v) { s[K] += v; }
};

// per-warp table of psi(v + a) - psi(a) and psi1(v + a) - psi1(a),
// v = 0..kPsiTab-1 (prefix sums of 1/(a+j) and -1/(a+j)^2)
DEV void warp_psi_table(double a, double* d1, double* d2) {
    const int lane = threadIdx.x & 31;
    double c1 = 0.0, c2 = 0.0;
    for (int base = 0; base < kPsiTab; base += 32) {
        const int v = base + lane;
        const double t = v == 0 ? 0.0 : 1.0 / (a + (v - 1));
        double s1 = t, s2 = -t * t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double u1 = __shfl_up_sync(0xffffffffu, s1, o);
            const double u2 = __shfl_up_sync(0xffffffffu, s2, o);
            if (lane >= o) {
                s1 += u1;
                s2 += u2;
            }
        }
        d1[v] = c1 + s1;
        d2[v] = c2 + s2;
        c1 += __shfl_sync(0xffffffffu, s1, 31);
        c2 += __shfl_sync(0xffffffffu, s2, 31);
    }
    __syncwarp();
}

template <int P, class VT>
__global__ void __launch_bounds__(kTcNT) tc_mle_kernel(PassGeom geo, PassMLE::Params prm,
                                                      const float4* __restrict__ zimg) {
    constexpr int NE = P * (P + 1) / 2;
    constexpr int NA = 3 * NE + 2;
    constexpr int PP = P <= 1 ? 1 : (P <= 2 ? 2 : 4);
    static_assert(NE <= kTcZ, "products fit the MMA's N");
    // epilogue scratch in the first R stage: dense scalar sums, the R_lo
    // halves of the drained rows, nonzero sums, digamma tables
    constexpr int kFs = 0;                               // float [8][32][2]
    constexpr int kHlo = kFs + 8 * kMleG * 2 * 4;        // float [3][32][16]
    constexpr int kSpar = kHlo + 3 * kMleG * 16 * 4;     // double [32][4]
    constexpr int kPsi = kSpar + kMleG * 4 * 8;          // double [8 warps][2][kPsiTab]
    static_assert(kPsi + 8 * 2 * kPsiTab * 8 <= kTcStage, "epilogue scratch fits the first R stage");
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tslot;
    __shared__ int abort_flag;

    if (geo.reset_next && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *geo.reset_next = 0;
    const int nact = *geo.n_act;
    const int tile = blockIdx.y;
    if (tile * kMleG >= nact) return;
    const int seg = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const VT* __restrict__ val = static_cast<const VT*>(geo.val);

    // dense phase: gene = tile slot lane, cells = quad `warp` of each chunk
    int slot0 = tile * kMleG + lane;
    if (slot0 >= nact) slot0 = tile * kMleG;  // duplicate a valid gene; not written
    const int gene = __ldg(geo.act + slot0);
    float beta[P];
#pragma unroll
    for (int i = 0; i < P; ++i) beta[i] = __ldg(prm.beta + (int64_t)gene * P + i) * kLog2e;
    const float thf = (float)exp(__ldg(prm.log_theta + gene));
    const int nfs = geo.nbound - 1;
    const int b0 = (int)(((int64_t)seg * nfs) / geo.nseg);
    const int b1 = (int)(((int64_t)(seg + 1) * nfs) / geo.nseg);
    const int c0 = __ldg(geo.bound + b0), c1 = __ldg(geo.bound + b1);

    auto in_stage = [&](int s) { return tc_smem + 2 * kTcStage + s * kTcInBytes; };
    auto fetch_inputs = [&](int kc) {
        unsigned char* ib = in_stage(kc & 3);
        const int cs = c0 + kc * kTcKC;
        cp_async<16>(ib + tid * 16, zimg + (int64_t)(cs >> 2) * kTcN + tid);
        constexpr int NX = kTcKC * PP / 4;
        constexpr int CPX = 4 / PP;
        if (tid < NX) {
            const int cell = cs + tid * CPX;
            const int valid = min(max(c1 - cell, 0), CPX);
            cp_async_zfill(ib + kTcInX + tid * 16, valid ? (const void*)(geo.X + (int64_t)cell * PP) : geo.X,
                           (uint32_t)(valid * PP * 4));
        } else if (tid >= 64 && tid < 64 + kTcKC / 4) {
            const int pc = tid - 64;
            const int cell = cs + 4 * pc;
            const int valid = min(max(c1 - cell, 0), 4);
            cp_async_zfill(ib + kTcInOff + pc * 16, valid ? (const void*)(geo.off + cell) : geo.off,
                           (uint32_t)(valid * 4));
        }
    };
    const int nchunk = (c1 - c0 + kTcKC - 1) / kTcKC;
    if (nchunk > 0) fetch_inputs(0);
    cp_async_commit();
    if (nchunk > 1) fetch_inputs(1);
    cp_async_commit();
    // rows 96..127 (no weight) stay zero in both stages
    for (int i = tid; i < 2 * 2 * kMleG * (kTcKC / 4); i += kTcNT) {
        const int buf = i / (kMleG * (kTcKC / 4)), r = i % (kMleG * (kTcKC / 4));
        const int q = r / kMleG, row = 3 * kMleG + r % kMleG;
        *reinterpret_cast<float4*>(tc_smem + buf * kTcABytes + stage_off(row, q, kTcM)) =
            make_float4(0.f, 0.f, 0.f, 0.f);
    }
    cp_async_wait<1>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");

    if (tid == 0) {
        abort_flag = 0;
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tslot)),
                     "r"(kMleCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;

    float fs0 = 0.f, fs1 = 0.f;
    // drained rows: warp w (w & 3 = weight b < 3) owns row 32 b + lane,
    // columns 0..15 (warps 0..3) or 16..31 (warps 4..7)
    float hacc[16];
#pragma unroll
    for (int a = 0; a < 16; ++a) hacc[a] = 0.f;
    const bool drains = (warp & 3) < 3;
    const uint32_t lanes = ((uint32_t)(32 * (warp & 3)) << 16) + (warp < 4 ? 0u : (uint32_t)kTcZ);
    int drained = 0;
    int issued = 0;
    for (int k = 0; k < nchunk; ++k) {
        const int st = k & 1;
        bool ok = true;
        if (k >= 2) {
            ok = mbar_wait_bounded(&bars[st], (uint32_t)(((k >> 1) - 1) & 1));
            if (!ok) atomicExch(&abort_flag, 1);
        }
        ok = __all_sync(0xffffffffu, ok);
        if (k >= 2 && (k - 2) % kTcRun == kTcRun - 1) {
            if (drains && ok) {
                float t[16];
                tc_ld16(tmem + lanes + kMleRegion * (uint32_t)(drained & 1), t);
#pragma unroll
                for (int a = 0; a < 16; ++a) hacc[a] += t[a];
            }
            ++drained;
        }
        if (k + 2 < nchunk) fetch_inputs(k + 2);
        cp_async_commit();
        unsigned char* sAh = tc_smem + st * kTcStage;
        unsigned char* sAl = sAh + kTcABytes;
        const unsigned char* ib = in_stage(k & 3);
        const float* xs = reinterpret_cast<const float*>(ib + kTcInX);
        const float* os = reinterpret_cast<const float*>(ib + kTcInOff);
        const int cs = c0 + k * kTcKC;
        {
            const int q = warp;
            float wv[3][4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                float x[P];
#pragma unroll
                for (int i = 0; i < P; ++i) x[i] = xs[(4 * q + t) * PP + i];
                float e = os[4 * q + t] * kLog2e;
#pragma unroll
                for (int i = 0; i < P; ++i) e = fmaf(x[i], beta[i], e);
                const float mu = ex2_approx(e);
                // PassMLE::dense
                const float xx = mu * thf;
                const float r = rcp_approx(1.f + xx);
                const float w = mu * r;
                wv[0][t] = w;
                wv[1][t] = -w * w;
                wv[2][t] = 2.f * w * w * w;
                // zero-filled cells past the last one meet Z = 0 in the
                // MMAs but would add to these sums
                if (cs + 4 * q + t < c1) {
                    fs0 += nb_ll_term<float>(xx, r);
                    fs1 += w * xx * r;
                }
            }
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                float hi[4], lo[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    hi[t] = __uint_as_float(__float_as_uint(wv[b][t]) & 0xFFFFE000u);
                    lo[t] = wv[b][t] - hi[t];
                }
                const int off = stage_off(kMleG * b + lane, q, kTcM);
                *reinterpret_cast<float4*>(sAh + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
                *reinterpret_cast<float4*>(sAl + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
            }
        }
        cp_async_wait<1>();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        if (abort_flag) break;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t dreg = tmem + kMleRegion * (uint32_t)((k / kTcRun) & 1);
            const uint32_t sB = smem_u32(ib);
#pragma unroll
            for (int s = 0; s < kTcKC / 8; ++s) {
                const uint32_t acc = (k % kTcRun != 0 || s > 0) ? 1u : 0u;
                const uint64_t bd = umma_desc(sB + s * 2 * kTcN * 16, kTcN * 16, 128);
                const uint64_t ah = umma_desc(smem_u32(sAh) + s * 2 * kTcM * 16, kTcM * 16, 128);
                const uint64_t al = umma_desc(smem_u32(sAl) + s * 2 * kTcM * 16, kTcM * 16, 128);
                tc_mma(dreg, ah, bd, acc);                // R_hi [Z_hi; Z_lo]
                tc_mma_n(dreg, al, bd, 1u, kIdesc16);     // R_lo Z_hi (the first 16 rows of B)
            }
            tc_commit(&bars[st]);
        }
        issued = k + 1;
    }
    cp_async_wait<0>();
    if (issued > 0 &&
        !mbar_wait_bounded(&bars[(issued - 1) & 1], (uint32_t)(((issued - 1) >> 1) & 1)))
        atomicExch(&abort_flag, 1);
    tc_fence_after();
    __syncthreads();
    if (!abort_flag) {
        const int runs = (issued + kTcRun - 1) / kTcRun;
        for (; drained < runs; ++drained)
            if (drains) {
                float t[16];
                tc_ld16(tmem + lanes + kMleRegion * (uint32_t)(drained & 1), t);
#pragma unroll
                for (int a = 0; a < 16; ++a) hacc[a] += t[a];
            }
    }
    __syncthreads();

    float* fsr = reinterpret_cast<float*>(tc_smem + kFs);
    float* hlo = reinterpret_cast<float*>(tc_smem + kHlo);
    double* spar = reinterpret_cast<double*>(tc_smem + kSpar);
    double* psi = reinterpret_cast<double*>(tc_smem + kPsi) + warp * 2 * kPsiTab;
    fsr[(warp * kMleG + lane) * 2 + 0] = fs0;
    fsr[(warp * kMleG + lane) * 2 + 1] = fs1;
    if (warp >= 4 && drains) {
#pragma unroll
        for (int a = 0; a < 16; ++a) hlo[((warp - 4) * kMleG + lane) * 16 + a] = hacc[a];
    }

    // nonzero terms (PassMLE::sparse, FP64): warp w takes genes w, w + 8, ...
    for (int gi = warp; gi < kMleG; gi += 8) {
        int slot = tile * kMleG + gi;
        if (slot >= nact) slot = tile * kMleG;
        const int g = __ldg(geo.act + slot);
        const double th = exp(__ldg(prm.log_theta + g));
        const double a = 1.0 / th;
        warp_psi_table(a, psi, psi + kPsiTab);
        PassMLE::Gene G{th, a, (float)th, PsiTable{psi, psi + kPsiTab, digamma_d(a), trigamma_d(a)}};
        float bg[P];
#pragma unroll
        for (int i = 0; i < P; ++i) bg[i] = __ldg(prm.beta + (int64_t)g * P + i) * kLog2e;
        ScalAcc acc;
        const int64_t* sp = geo.segptr + (int64_t)g * geo.nbound;
        const int64_t e0 = __ldg(sp + b0), e1 = __ldg(sp + b1);
        for (int64_t eb = e0 + lane; eb < e1; eb += 64) {
            int cc[2];
            float yy[2];
            bool okk[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int64_t e = eb + 32 * u;
                okk[u] = e < e1;
                cc[u] = okk[u] ? __ldg(geo.col + e) : c0;
                yy[u] = okk[u] ? load_val(val, e) : 0.f;
            }
            float xr[2][P], ol[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                load_row<P, PP>(geo.X, cc[u], xr[u]);
                ol[u] = __ldg(geo.off + cc[u]);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (!okk[u]) continue;
                float el = ol[u] * kLog2e;
#pragma unroll
                for (int i = 0; i < P; ++i) el = fmaf(xr[u][i], bg[i], el);
                PassMLE::sparse<float>(G, ex2_approx(el), yy[u], acc);
            }
        }
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) acc.s[k2] = warp_sum(acc.s[k2]);
        if (lane == 0) {
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) spar[gi * 4 + k2] = acc.s[k2];
        }
        __syncwarp();  // the table is rebuilt for the next gene
    }
    __syncthreads();

    const int slot = tile * kMleG + lane;
    if (slot < nact && !abort_flag) {
        float* out = static_cast<float*>(geo.partW) + ((int64_t)seg * geo.slot_stride + slot) * NA;
        if (warp < 3) {  // weight b = warp: b, db, d2b
#pragma unroll
            for (int a = 0; a < NE; ++a) out[warp * NE + a] = hacc[a] + hlo[(warp * kMleG + lane) * 16 + a];
        } else if (warp == 3) {
            float f0 = 0.f, f1 = 0.f;
#pragma unroll
            for (int w = 0; w < 8; ++w) {
                f0 += fsr[(w * kMleG + lane) * 2 + 0];
                f1 += fsr[(w * kMleG + lane) * 2 + 1];
            }
            out[3 * NE + 0] = f0;
            out[3 * NE + 1] = f1;
            double* outs = geo.partS + ((int64_t)seg * geo.slot_stride + slot) * 4;
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) outs[k2] = spar[lane * 4 + k2];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMleCols)
                     : "memory");
    if (abort_flag && tid == 0) atomicExch(geo.err, 1);
}

// Z image: for every quad of 4 cells, 32 rows of 4 TF32 values: rows
// 0..15 the high parts of the products x_i x_j (packed upper-triangle
// order, then zeros), rows 16..31 the low parts; cells at or beyond n are
// zero
__global__ void tc_zimg_kernel(const float* Xrm, int xs, int64_t n, int P, int64_t nq, float4* zimg) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nq * kTcN;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = t / kTcN;
        const int prow = (int)(t - q * kTcN);
        const bool low = prow >= kTcZ;
        const int row = low ? prow - kTcZ : prow;
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        int ii = -1, jj = -1;
        for (int b = 0, idx = 0; b < P && ii < 0; ++b)
            for (int a = 0; a <= b; ++a, ++idx)
                if (idx == row) {
                    ii = a;
                    jj = b;
                    break;
                }
        if (ii >= 0) {
            for (int u = 0; u < 4; ++u) {
                const int64_t c = 4 * q + u;
                if (c < n) {
                    const float z = __fmul_rn(Xrm[c * xs + ii], Xrm[c * xs + jj]);
                    const float hi = to_tf32(z);
                    v[u] = low ? to_tf32(z - hi) : hi;
                }
            }
        }
        zimg[t] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

template <int P>
cudaError_t run_tc(const PassLaunch& L, const float4* zimg) {
    if (L.GT != kTcM) return cudaErrorInvalidValue;
    dim3 grid(L.nseg, L.ntiles);
    PassIRLS::Params prm{L.prm.beta, L.prm.beta_d, L.prm.k};
    cudaError_t e;
    if (L.val_u16) {
        auto k = tc_irls_kernel<P, uint16_t>;
        e = raise_dyn_smem(k, kTcSmem);
        if (e != cudaSuccess) return e;
        if (L.occ_out) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, k, kTcNT, kTcSmem);
        k<<<grid, kTcNT, kTcSmem, L.stream>>>(L.geo, prm, zimg);
    } else {
        auto k = tc_irls_kernel<P, float>;
        e = raise_dyn_smem(k, kTcSmem);
        if (e != cudaSuccess) return e;
        if (L.occ_out) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, k, kTcNT, kTcSmem);
        k<<<grid, kTcNT, kTcSmem, L.stream>>>(L.geo, prm, zimg);
    }
    return cudaGetLastError();
}

template <int P>
cudaError_t run_tc_mle(const PassLaunch& L, const float4* zimg) {
    if (L.GT != kMleG) return cudaErrorInvalidValue;
    dim3 grid(L.nseg, L.ntiles);
    PassMLE::Params prm{L.prm.beta, L.prm.beta_d, L.prm.log_theta};
    cudaError_t e;
    if (L.val_u16) {
        auto k = tc_mle_kernel<P, uint16_t>;
        e = raise_dyn_smem(k, kTcSmem);
        if (e != cudaSuccess) return e;
        if (L.occ_out) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, k, kTcNT, kTcSmem);
        k<<<grid, kTcNT, kTcSmem, L.stream>>>(L.geo, prm, zimg);
    } else {
        auto k = tc_mle_kernel<P, float>;
        e = raise_dyn_smem(k, kTcSmem);
        if (e != cudaSuccess) return e;
        if (L.occ_out) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, k, kTcNT, kTcSmem);
        k<<<grid, kTcNT, kTcSmem, L.stream>>>(L.geo, prm, zimg);
    }
    return cudaGetLastError();
}

}  // namespace

int tc_max_p() { return 4; }
int tc_tile_genes(PassKind k) { return k == PASS_MLE ? kMleG : kTcM; }
int tc_chunk_cells() { return kTcKC; }

// Opt-in (DEVIL_TC=1): at p <= 4 the register engine is faster on B200.
// Its outer products already run as packed FP32x2 FMAs (5 instructions per
// gene and cell at p = 4); this engine saves them but spends about as much
// on the hi/lo split, the shared-memory stores and the per-chunk
// synchronisation (measured: IRLS 171 ms vs 133 ms per step on the
// 20,000 x 100,000 benchmark fit).
bool tc_enabled(PassKind k) {
    if (k == PASS_MLE) {
        const char* e = getenv("DEVIL_TC_MLE");
        return e && atoi(e) == 1;
    }
    if (k != PASS_IRLS) return false;
    const char* e = getenv("DEVIL_TC");
    return e && atoi(e) == 1;
}

int64_t tc_zimg_quads(int64_t n) { return (n + kTcKC - 1) / kTcKC * (kTcKC / 4); }
int64_t tc_zimg_float4s(int64_t n) { return tc_zimg_quads(n) * kTcN; }

cudaError_t launch_tc_zimg(const float* Xrm, int xs, int64_t n, int P, float4* zimg, cudaStream_t st) {
    if (P < 1 || P > 4) return cudaErrorInvalidValue;
    const int64_t nq = tc_zimg_quads(n);
    if (nq == 0) return cudaSuccess;
    tc_zimg_kernel<<<(unsigned)std::min<int64_t>((nq * kTcN + 255) / 256, 148 * 16), 256, 0, st>>>(
        Xrm, xs, n, P, nq, zimg);
    return cudaGetLastError();
}

// L.GT = 128 genes per tile; the grid has L.ntiles rows of blocks
cudaError_t launch_tc_pass(const PassLaunch& L, const float4* zimg) {
    if (L.xs_pad != (L.P <= 1 ? 1 : (L.P <= 2 ? 2 : 4))) return cudaErrorInvalidValue;
    if (L.kind == PASS_MLE) {
        switch (L.P) {
            case 1: return run_tc_mle<1>(L, zimg);
            case 2: return run_tc_mle<2>(L, zimg);
            case 3: return run_tc_mle<3>(L, zimg);
            case 4: return run_tc_mle<4>(L, zimg);
        }
        return cudaErrorInvalidValue;
    }
    if (L.kind != PASS_IRLS) return cudaErrorInvalidValue;
    switch (L.P) {
        case 1: return run_tc<1>(L, zimg);
        case 2: return run_tc<2>(L, zimg);
        case 3: return run_tc<3>(L, zimg);
        case 4: return run_tc<4>(L, zimg);
    }
    return cudaErrorInvalidValue;
}

}  // namespace devil
