// IRLS and dispersion (MLE) passes with the per-gene p x p contractions on
// the tensor cores (sm_100a tcgen05, kind::tf32) for designs of p = 5..32
// columns that do not collapse to a few distinct rows (continuous
// covariates).  The IRLS form is described here; the MLE form (the Cox-Reid
// matrices) is described at tcw_pass_kernel.
//
// beta_fit (src/beta.cpp:35-42) needs per gene g and IRLS step
//     H_g = sum_c hw_gc z_c,   z_c = the products x_ci x_cj (i <= j),
//     s_g = sum_c sw_gc x_c,
// with r = 1/(mu + k), hw = r (1 + y / k), sw = (mu - y) r (PassIRLS in
// passes.cuh: the dense terms of every cell plus the nonzero corrections).
// Over a tile of 128 genes and a chunk of 32 cells the Hessian part is the
// product
//     D[128 genes x NBLK products] += HW[128 x 32 cells] Z[NBLK x 32 cells]^T
// with NE = p (p + 1) / 2 products split over gridDim.z blocks of at most
// 176 columns (p = 32: three blocks of 176).  The counts enter the weights
// directly: the pass reads a dense image of the counts (gene rows of
// npad cells, uint16 or float), so no separate nonzero pass is needed.
//
// Per chunk the CUDA cores compute eta = off + x beta (FP32, packed FMAs),
// mu (ex2), r (rcp), the weights, and the chunk's products z = x_i x_j;
// HW and Z enter as split TF32 pairs (v = hi + lo) and the MMA sums
//     HW_hi Z_hi + HW_lo Z_hi + HW_hi Z_lo
// (3 x TF32: about 2^-21 relative per term, the hi x lo terms of both
// operands kept; lo x lo, ~2^-22, dropped).  The score, which fixes the
// solution, stays on the CUDA cores in FP32 (block z = 0).
//
// Accumulation: D accumulates a run of 8 chunks (256 cells) in tensor
// memory; the run is then added in FP32 on the CUDA cores into a running
// total (tensor-memory columns T.., T = 128 or 256, tcgen05.ld / add /
// tcgen05.st), so no tensor-core accumulation spans more than 256 terms.
// A block allocates 2 T columns: two blocks of a small product count
// (T = 128) can share an SM's 512 columns.
//
// Pipeline: cp.async brings the chunk's design rows (transposed: feature
// rows of 32 cells), offsets and count rows two chunks ahead (ring of 3);
// the operand stages (HW_hi, HW_lo, Z_hi, Z_lo) are double-buffered and a
// stage is rewritten only after the MMAs that read it have completed
// (mbarrier, bounded wait).  A run is added to the total after the next
// chunk's CUDA-core work, so that work overlaps the run's last MMAs.  On a
// bounded wait's expiry the block records an error, skips its output,
// drains its MMAs (bounded) and frees its tensor memory.
#include "internal.h"
#include "tc_common.cuh"

#include <algorithm>

namespace devil {

namespace {

constexpr int kWM = 128;                  // genes per tile: MMA M, tensor-memory lanes
constexpr int kWKC = 32;                  // cells per chunk (4 K-steps of 8 TF32)
constexpr int kWNT = 256;                 // threads per block
constexpr int kWNmax = 176;               // product columns per block at most
constexpr int kWRun = 8;                  // chunks per tensor-memory run (256 cells)
constexpr int kWA = kWM * kWKC * 4;       // one of HW_hi, HW_lo: 16 KB
constexpr int kWRing = 3;                 // input ring depth

constexpr int op_bytes(int nblk) { return 2 * kWA + 2 * nblk * kWKC * 4; }
template <class VT, int GTn>
constexpr int in_bytes(int XS) { return XS * kWKC * 4 + kWKC * 4 + GTn * kWKC * (int)sizeof(VT); }
constexpr int kMleG = 32;                             // genes per tile of the MLE pass
constexpr int kPsiBytes = kMleG * 2 * kPsiTab * 8;    // their psi tables
template <class VT, bool MLE>
constexpr int tcw_smem(int XS, int nblk) {
    return 2 * op_bytes(nblk) + kWRing * in_bytes<VT, MLE ? kMleG : kWM>(XS) + (MLE ? kPsiBytes : 0);
}

static_assert(tcw_smem<float, false>(32, kWNmax) <= 227 * 1024, "stages fit the shared memory of one block");
static_assert(tcw_smem<float, true>(32, kWNmax) <= 227 * 1024, "stages fit the shared memory of one block");

// (a0, a1) += (b0, b1) * (c0, c1) as one packed FP32x2 FMA
DEV void fma2(float& a0, float& a1, float b0, float b1, float c0, float c1) {
    uint64_t acc, bb, cc;
    asm("mov.b64 %0, {%1, %2};" : "=l"(acc) : "f"(a0), "f"(a1));
    asm("mov.b64 %0, {%1, %2};" : "=l"(bb) : "f"(b0), "f"(b1));
    asm("mov.b64 %0, {%1, %2};" : "=l"(cc) : "f"(c0), "f"(c1));
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(bb), "l"(cc));
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a0), "=f"(a1) : "l"(acc));
}

// counts of cells 4q..4q+3 of gene row gr in a count stage of R rows
template <int R>
DEV void load_counts(const uint16_t* ys, int q, int gr, float* y) {
    // piece (gene, 8 cells) at ((q >> 1) * R + gene) * 16; this quad is its half q & 1
    const uint2 h = *reinterpret_cast<const uint2*>(
        reinterpret_cast<const unsigned char*>(ys) + (((q >> 1) * R + gr) * 16 + (q & 1) * 8));
    y[0] = (float)(h.x & 0xFFFFu);
    y[1] = (float)(h.x >> 16);
    y[2] = (float)(h.y & 0xFFFFu);
    y[3] = (float)(h.y >> 16);
}
template <int R>
DEV void load_counts(const float* ys, int q, int gr, float* y) {
    const float4 v = *reinterpret_cast<const float4*>(
        reinterpret_cast<const unsigned char*>(ys) + (q * R + gr) * 16);
    y[0] = v.x;
    y[1] = v.y;
    y[2] = v.z;
    y[3] = v.w;
}

// add the run (columns [c0, c1) of this warp's 32 lanes) into the total
// at column offset tot
DEV void tcw_drain(uint32_t tmem, uint32_t lanes, uint32_t tot, int c0, int c1, bool first) {
    for (int c = c0; c < c1; c += 8) {
        float v[8];
        tc_ld8(tmem + lanes + (uint32_t)c, v);
        if (!first) {
            float t[8];
            tc_ld8(tmem + lanes + tot + (uint32_t)c, t);
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] += t[u];
        }
        tc_st8(tmem + lanes + tot + (uint32_t)c, v);
    }
    tc_wait_st();
}

DEV void store_split(unsigned char* sA, int row, int q, const float* v) {
    float hi[4], lo[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) tf32_split(v[c], hi[c], lo[c]);
    *reinterpret_cast<float4*>(sA + stage_off(row, q, kWM)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<float4*>(sA + kWA + stage_off(row, q, kWM)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
}

// The IRLS pass (MLE = false): 128 genes per tile, A row = gene, weight
// r (1 + y / k); thread = (gene row tid % 128, cells of quads 4 h .. 4 h + 3
// with h = tid / 128), the score in registers.
// The dispersion pass (MLE = true; PassMLE in passes.cuh,
// src/overdispersion.cpp:95-242): 32 genes per tile, A rows 32 b + gene
// carry the Cox-Reid weights w, -w^2, 2 w^3 (b = 0, 1, 2; rows 96..127
// zero); thread = (gene tid % 32, quad tid / 32); the two FP32 scalar sums
// and, at the gene's nonzeros, the four FP64 sums with per-gene psi tables,
// all in block z = 0.
template <int XS, class VT, bool MLE>
__global__ void __launch_bounds__(kWNT, 1) tcw_pass_kernel(PassGeom geo, PassParamsAny prm, TcwGeom tw) {
    constexpr int GTn = MLE ? kMleG : kWM;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tslot;
    __shared__ int abort_flag;
    __shared__ int16_t ptab[kWNmax];  // product row -> i | j << 8 (-1: padding)
    __shared__ double psia[MLE ? kMleG : 1];

    if (geo.reset_next && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0)
        *geo.reset_next = 0;
    const int nact = *geo.n_act;
    const int tile = blockIdx.y;
    if (tile * GTn >= nact) return;
    const int seg = blockIdx.x;
    const int zb = blockIdx.z;
    const int nblk = tw.nblk;
    const uint32_t tot = nblk <= 128 ? 128u : 256u;  // column of the running total
    const uint32_t ncols = 2 * tot;                  // columns allocated
    const int tid = threadIdx.x, warp = tid >> 5;
    const int gi = tid & (GTn - 1);  // this thread's gene within the tile
    const int hh = tid >> 7;         // IRLS: half of the chunk's cells (and of the drained columns)
    const bool extra = zb == 0;      // block z = 0 adds the score / scalar sums

    int slot = tile * GTn + gi;
    const bool valid_slot = slot < nact;
    if (!valid_slot) slot = tile * GTn;  // duplicate a valid gene; not written
    const int g = __ldg(geo.act + slot);
    float bt[XS];
#pragma unroll
    for (int i = 0; i < XS; ++i) bt[i] = i < tw.P ? __ldg(prm.beta + (int64_t)g * tw.P + i) * kLog2e : 0.f;
    float kk = 0.f, rk = 0.f, thf = 0.f;
    double theta = 0.0, aa = 0.0;
    if constexpr (MLE) {
        theta = exp(prm.log_theta[g]);
        aa = 1.0 / theta;
        thf = (float)theta;
    } else {
        kk = __ldg(prm.k + g);
        rk = 1.f / kk;
    }

    for (int r = tid; r < nblk; r += kWNT) {
        const int gp = zb * nblk + r;
        int16_t v = -1;
        if (gp < tw.NE) {
            int j = 0;
            while ((j + 1) * (j + 2) / 2 <= gp) ++j;
            const int i = gp - j * (j + 1) / 2;
            v = (int16_t)(i | (j << 8));
        }
        ptab[r] = v;
    }

    // this block's cells: fine segments [b0, b1) (multiples of 32 cells up
    // to n; the last chunk reads the padding of the images past n)
    const int nfs = geo.nbound - 1;
    const int b0 = (int)(((int64_t)seg * nfs) / geo.nseg);
    const int b1 = (int)(((int64_t)(seg + 1) * nfs) / geo.nseg);
    const int64_t k0 = __ldg(geo.bound + b0) / kWKC;
    const int64_t k1 = (__ldg(geo.bound + b1) + kWKC - 1) / kWKC;
    const int nchunk = (int)(k1 - k0);

    const int OPB = op_bytes(nblk);
    constexpr int INB = in_bytes<VT, GTn>(XS);
    auto op = [&](int s) { return smem + s * OPB; };
    auto in_slot = [&](int s) { return smem + 2 * OPB + s * INB; };
    const VT* __restrict__ yrow = static_cast<const VT*>(tw.ydense) + (int64_t)g * tw.ld;

    // MLE: the tile's psi tables (scratch in the first operand stage), then
    // the zero rows 96..127 of both A stages
    PsiTable tab{nullptr, nullptr, 0.0, 0.0};
    if constexpr (MLE) {
        double* psitab = reinterpret_cast<double*>(smem + 2 * OPB + kWRing * INB);
        if (tid < kMleG) psia[tid] = aa;
        __syncthreads();
        build_psi_tables(kMleG, psia, psitab, reinterpret_cast<double*>(smem));
        tab.d1 = psitab + (gi * 2 + 0) * kPsiTab;
        tab.d2 = psitab + (gi * 2 + 1) * kPsiTab;
        if (extra) {
            tab.pa = digamma_d(aa);
            tab.ta = trigamma_d(aa);
        }
        for (int t = tid; t < 2 * 2 * 32 * 8; t += kWNT) {
            const int s = t >> 9, hl = (t >> 8) & 1, row = 96 + ((t >> 3) & 31), q = t & 7;
            *reinterpret_cast<float4*>(op(s) + hl * kWA + stage_off(row, q, kWM)) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }

    auto fetch = [&](int kc) {
        unsigned char* ib = in_slot(kc % kWRing);
        const int64_t cs = (k0 + kc) * kWKC;
        for (int idx = tid; idx < XS * 8 + 8; idx += kWNT) {
            if (idx < XS * 8) {
                const int i = idx >> 3, q = idx & 7;
                cp_async<16>(ib + stage_off(i, q, XS), tw.xt + (int64_t)i * tw.npad + cs + 4 * q);
            } else {
                const int q = idx - XS * 8;
                cp_async<16>(ib + XS * kWKC * 4 + 16 * q, tw.offp + cs + 4 * q);
            }
        }
        unsigned char* yb = ib + XS * kWKC * 4 + kWKC * 4;
        constexpr int CPP = 16 / (int)sizeof(VT);  // cells per piece
        constexpr int NPG = kWKC / CPP;            // pieces per gene row
        if constexpr (MLE) {
            // piece (gene tid % 32, p = tid / 32)
            if (tid < kMleG * NPG) {
                const int p = tid >> 5;
                cp_async<16>(yb + (p * kMleG + gi) * 16, yrow + cs + p * CPP);
            }
        } else {
#pragma unroll
            for (int u = 0; u < NPG / 2; ++u) {
                const int p = hh + 2 * u;  // piece index within the row
                cp_async<16>(yb + (p * kWM + gi) * 16, yrow + cs + p * CPP);
            }
        }
    };

    if (nchunk > 0) fetch(0);
    cp_async_commit();
    if (nchunk > 1) fetch(1);
    cp_async_commit();

    if (tid == 0) {
        abort_flag = 0;
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tslot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    const uint32_t lanes = (uint32_t)(32 * (warp & 3)) << 16;
    const int dc0 = hh * (nblk / 2), dc1 = dc0 + nblk / 2;  // this warp's drained columns
    const uint32_t idesc = tf32_idesc(kWM, nblk);

    // IRLS score: cells (0, 1) and (2, 3) of each quad; MLE: the FP32 and
    // FP64 scalar sums
    float va[MLE ? 1 : XS], vb[MLE ? 1 : XS];
    float fs[2] = {0.f, 0.f};
    double sc[4] = {0.0, 0.0, 0.0, 0.0};
    if constexpr (!MLE) {
#pragma unroll
        for (int i = 0; i < XS; ++i) va[i] = vb[i] = 0.f;
    }

    int issued = 0;   // chunks whose MMAs were committed (uniform)
    int drained = 0;  // runs added into the total (uniform)
    for (int k = 0; k < nchunk; ++k) {
        const int st = k & 1;
        bool ok = true;
        // chunk k - 2's MMAs have completed: operand stage st is free
        if (k >= 2) ok = mbar_wait_bounded(&bars[st], (uint32_t)(((k - 2) >> 1) & 1));
        if (!ok) atomicExch(&abort_flag, 1);
        if (k + 2 < nchunk) fetch(k + 2);
        cp_async_commit();
        cp_async_wait<2>();  // this thread's copies of chunk k have landed
        __syncthreads();     // ... and everyone's
        if (abort_flag) break;

        const unsigned char* ib = in_slot(k % kWRing);
        const float4* x4 = reinterpret_cast<const float4*>(ib);
        const float4* o4 = reinterpret_cast<const float4*>(ib + XS * kWKC * 4);
        const VT* ys = reinterpret_cast<const VT*>(ib + XS * kWKC * 4 + kWKC * 4);
        unsigned char* sA = op(st);
        // the weights of this thread's gene at its cells
#pragma unroll
        for (int qi = 0; qi < (MLE ? 1 : 4); ++qi) {
            const int q = MLE ? warp : 4 * hh + qi;
            const float4 o = o4[q];
            float e0 = o.x * kLog2e, e1 = o.y * kLog2e, e2 = o.z * kLog2e, e3 = o.w * kLog2e;
#pragma unroll
            for (int i = 0; i < XS; ++i) {
                const float4 x = x4[q * XS + i];
                fma_x2(e0, e1, bt[i], x.x, x.y);
                fma_x2(e2, e3, bt[i], x.z, x.w);
            }
            float y[4];
            load_counts<GTn>(ys, q, gi, y);
            const float e[4] = {e0, e1, e2, e3};
            if constexpr (MLE) {
                float w1[4], w2[4], w3[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float mu = ex2_approx(e[c]);
                    const float xx = mu * thf;
                    const float r = rcp_r(1.f + xx);
                    const float w = mu * r;
                    w1[c] = w;
                    w2[c] = -w * w;
                    w3[c] = 2.f * w * w * w;
                    if (extra) {
                        fs[0] += nb_ll_term<float>(xx, r);
                        fs[1] += w * xx * r;
                        if (y[c] > 0.f) {
                            const double m = mu, yy = y[c];
                            const double den = 1.0 + m * theta;
                            double rr = (double)rcp_approx((float)den);
                            rr = rr + rr * (1.0 - den * rr);
                            sc[0] += yy * theta * rr;
                            sc[1] += yy * rr * rr;
                            double d1, d2;
                            psi_diffs_tab(yy, aa, tab, d1, d2);
                            sc[2] += d1;
                            sc[3] += d2;
                        }
                    }
                }
                store_split(sA, gi, q, w1);
                store_split(sA, 32 + gi, q, w2);
                store_split(sA, 64 + gi, q, w3);
            } else {
                float hw[4], sw[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float mu = ex2_approx(e[c]);
                    const float r = rcp_approx(mu + kk);
                    const float yr = y[c] * r;
                    hw[c] = fmaf(yr, rk, r);    // r + y r / k
                    sw[c] = fmaf(mu, r, -yr);   // (mu - y) r
                }
                store_split(sA, gi, q, hw);
                if (extra) {
#pragma unroll
                    for (int i = 0; i < XS; ++i) {
                        const float4 x = x4[q * XS + i];
                        fma2(va[i], vb[i], sw[0], sw[2], x.x, x.z);
                        fma2(va[i], vb[i], sw[1], sw[3], x.y, x.w);
                    }
                }
            }
        }
        // the chunk's products of this block, split
        {
            unsigned char* sB = sA + 2 * kWA;
            int row = tid % nblk, q = tid / nblk;
            for (; q < 8;) {
                const int pr = ptab[row];
                float4 hz = make_float4(0.f, 0.f, 0.f, 0.f), lz = hz;
                if (pr >= 0) {
                    const float4 xi = x4[q * XS + (pr & 0xFF)];
                    const float4 xj = x4[q * XS + (pr >> 8)];
                    tf32_split(xi.x * xj.x, hz.x, lz.x);
                    tf32_split(xi.y * xj.y, hz.y, lz.y);
                    tf32_split(xi.z * xj.z, hz.z, lz.z);
                    tf32_split(xi.w * xj.w, hz.w, lz.w);
                }
                *reinterpret_cast<float4*>(sB + stage_off(row, q, nblk)) = hz;
                *reinterpret_cast<float4*>(sB + nblk * kWKC * 4 + stage_off(row, q, nblk)) = lz;
                row += kWNT;
                while (row >= nblk) {
                    row -= nblk;
                    ++q;
                }
            }
        }
        fence_async_smem();
        // chunk k - 1 closed a run: add it into the total once its MMAs
        // have completed (the work above overlapped them)
        if (k > 0 && k % kWRun == 0) {
            bool okd = mbar_wait_bounded(&bars[(k - 1) & 1], (uint32_t)(((k - 1) >> 1) & 1));
            okd = __all_sync(0xffffffffu, okd);
            if (okd) {
                tc_fence_after();
                tcw_drain(tmem, lanes, tot, dc0, dc1, drained == 0);
            } else {
                atomicExch(&abort_flag, 1);
            }
            ++drained;
        }
        tc_fence_before();
        __syncthreads();
        if (abort_flag) break;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a_hi = smem_u32(sA), a_lo = a_hi + kWA;
            const uint32_t b_hi = a_hi + 2 * kWA, b_lo = b_hi + (uint32_t)(nblk * kWKC * 4);
#pragma unroll
            for (int s = 0; s < kWKC / 8; ++s) {
                const uint32_t acc = (k % kWRun != 0 || s > 0) ? 1u : 0u;
                const uint64_t ah = umma_desc(a_hi + s * 2 * kWM * 16, kWM * 16, 128);
                const uint64_t al = umma_desc(a_lo + s * 2 * kWM * 16, kWM * 16, 128);
                const uint64_t bh = umma_desc(b_hi + s * 2 * nblk * 16, nblk * 16, 128);
                const uint64_t bl = umma_desc(b_lo + s * 2 * nblk * 16, nblk * 16, 128);
                tc_mma_n(tmem, ah, bh, acc, idesc);
                tc_mma_n(tmem, al, bh, 1u, idesc);
                tc_mma_n(tmem, ah, bl, 1u, idesc);
            }
            tc_commit(&bars[st]);
        }
        issued = k + 1;
    }
    cp_async_wait<0>();
    // the last commit completes after every MMA of the block; wait for it on
    // the error path too, so that no MMA is in flight when the tensor memory
    // is freed
    if (issued > 0 &&
        !mbar_wait_bounded(&bars[(issued - 1) & 1], (uint32_t)(((issued - 1) >> 1) & 1)))
        atomicExch(&abort_flag, 1);
    tc_fence_after();
    __syncthreads();  // abort_flag is final from here on
    const bool good = !abort_flag;
    if (good && issued > 0) tcw_drain(tmem, lanes, tot, dc0, dc1, drained == 0);  // the last run
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    // the Hessian-like columns of this warp's lanes: IRLS rows = genes;
    // MLE rows 32 b + gene (b = warp % 4 < 3)
    {
        const int b = MLE ? (warp & 3) : 0;
        const int lg = MLE ? (tid & 31) : gi;  // gene of this thread's tensor-memory lane
        const bool write = good && tile * GTn + lg < nact && (!MLE || b < 3);
        float* out = static_cast<float*>(geo.partW) + ((int64_t)seg * geo.slot_stride + tile * GTn + lg) * tw.NA +
                     b * tw.NE;
        for (int c = dc0; c < dc1; c += 8) {
            float v[8];
            if (issued > 0) {
                tc_ld8(tmem + lanes + tot + (uint32_t)c, v);
            } else {
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = 0.f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int gp = zb * nblk + c + u;
                if (write && c + u < nblk && gp < tw.NE) out[gp] = v[u];
            }
        }
    }
    if (extra) {
        const bool write = good && valid_slot;
        float* out = static_cast<float*>(geo.partW) + ((int64_t)seg * geo.slot_stride + tile * GTn + gi) * tw.NA;
        if constexpr (MLE) {
            // the 8 quads' sums of each gene, added in quad order
            float* fred = reinterpret_cast<float*>(smem);                  // [8][32][2]
            double* dred = reinterpret_cast<double*>(smem + 8 * 32 * 2 * 4);  // [8][32][4]
            fred[(warp * 32 + gi) * 2 + 0] = fs[0];
            fred[(warp * 32 + gi) * 2 + 1] = fs[1];
#pragma unroll
            for (int j = 0; j < 4; ++j) dred[(warp * 32 + gi) * 4 + j] = sc[j];
            __syncthreads();
            if (warp == 0 && write) {
                float f0 = 0.f, f1 = 0.f;
                double d[4] = {0.0, 0.0, 0.0, 0.0};
                for (int w = 0; w < 8; ++w) {
                    f0 += fred[(w * 32 + gi) * 2 + 0];
                    f1 += fred[(w * 32 + gi) * 2 + 1];
#pragma unroll
                    for (int j = 0; j < 4; ++j) d[j] += dred[(w * 32 + gi) * 4 + j];
                }
                out[3 * tw.NE + 0] = f0;
                out[3 * tw.NE + 1] = f1;
                double* os = geo.partS + ((int64_t)seg * geo.slot_stride + tile * GTn + gi) * 4;
#pragma unroll
                for (int j = 0; j < 4; ++j) os[j] = d[j];
            }
        } else {
            // the two halves of the cells: half 1 hands its sums to half 0
            // through the (idle) first operand stage
            float* red = reinterpret_cast<float*>(smem);  // [128 genes][XS]
            if (hh == 1) {
#pragma unroll
                for (int i = 0; i < XS; ++i) red[gi * XS + i] = va[i] + vb[i];
            }
            __syncthreads();
            if (hh == 0 && write) {
#pragma unroll
                for (int i = 0; i < XS; ++i)
                    if (i < tw.P) out[tw.NE + i] = va[i] + vb[i] + red[gi * XS + i];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                     : "memory");
    if (abort_flag && tid == 0) atomicExch(geo.err, 1);
}

template <int XS, class VT, bool MLE>
cudaError_t run_tcw(const PassLaunch& L, const TcwGeom& tw) {
    auto k = tcw_pass_kernel<XS, VT, MLE>;
    const int smem = tcw_smem<VT, MLE>(XS, tw.nblk);
    cudaError_t e = raise_dyn_smem(k, smem);
    if (e != cudaSuccess) return e;
    if (L.occ_out) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, k, kWNT, smem);
    dim3 grid(L.nseg, L.ntiles, tcw_blocks(L.P));
    k<<<grid, kWNT, smem, L.stream>>>(L.geo, L.prm, tw);
    return cudaGetLastError();
}

template <class VT, bool MLE>
cudaError_t run_tcw_xs(const PassLaunch& L, const TcwGeom& tw) {
    switch (L.xs_pad) {
        case 8: return run_tcw<8, VT, MLE>(L, tw);
        case 12: return run_tcw<12, VT, MLE>(L, tw);
        case 16: return run_tcw<16, VT, MLE>(L, tw);
        case 20: return run_tcw<20, VT, MLE>(L, tw);
        case 24: return run_tcw<24, VT, MLE>(L, tw);
        case 28: return run_tcw<28, VT, MLE>(L, tw);
        case 32: return run_tcw<32, VT, MLE>(L, tw);
    }
    return cudaErrorInvalidValue;
}

// count rows of the dense image: one warp per gene
template <class VT>
__global__ void tcw_dense_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                 const VT* __restrict__ val, int64_t G, int64_t ld, VT* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < G;
         g += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        VT* row = out + g * ld;
        for (int64_t e = rowptr[g] + lane; e < rowptr[g + 1]; e += 32) row[col[e]] = val[e];
    }
}

// feature rows of the design (zero past n and past p) and the offsets:
// -1e30 past n, so that mu = 0 there and the padding cells of the last
// chunk add nothing to any sum (the products and the score vanish with
// x = 0 as well, the dispersion pass's scalar sums only with mu = 0)
__global__ void tcw_xt_kernel(const float* __restrict__ Xrm, int xs, int64_t n, int64_t npad,
                              const float* __restrict__ off, float* __restrict__ xt, float* __restrict__ offp) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)(xs + 1) * npad;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / npad);
        const int64_t c = t - (int64_t)i * npad;
        if (i < xs) xt[t] = c < n ? Xrm[c * xs + i] : 0.f;
        else offp[c] = c < n ? off[c] : -1e30f;
    }
}

__global__ void irls_rescue_kernel(const int32_t* iters_in, int64_t G, int limit, double beta_limit,
                                   const double* __restrict__ beta0, int P, double* beta, float* beta_f,
                                   int32_t* iters, int32_t* status, int32_t* act, int32_t* cnt, int32_t* flag) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G; g += (int64_t)gridDim.x * blockDim.x) {
        double bmax = 0.0;
        for (int i = 0; i < P; ++i) bmax = fmax(bmax, fabs(beta[g * P + i]));
        const bool slow = iters_in[g] > limit || !(bmax <= beta_limit);
        flag[g] = slow ? 1 : 0;
        if (!slow) continue;
        act[atomicAdd(cnt, 1)] = (int32_t)g;
        for (int i = 0; i < P; ++i) {
            const double b = beta0[g * P + i];
            beta[g * P + i] = b;
            beta_f[g * P + i] = (float)b;
        }
        iters[g] = 0;
        status[g] = 0;
    }
}

__global__ void mask_i32_kernel(const int32_t* v, const int32_t* flag, int64_t G, int32_t* out) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G; g += (int64_t)gridDim.x * blockDim.x)
        out[g] = flag[g] ? v[g] : 0;
}

}  // namespace

cudaError_t launch_irls_rescue_select(const int32_t* iters_in, int64_t G, int limit, double beta_limit,
                                      const double* beta0, int P, double* beta, float* beta_f, int32_t* iters,
                                      int32_t* status, int32_t* act, int32_t* cnt, int32_t* flag, cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    irls_rescue_kernel<<<(unsigned)std::min<int64_t>((G + 255) / 256, 1024), 256, 0, st>>>(
        iters_in, G, limit, beta_limit, beta0, P, beta, beta_f, iters, status, act, cnt, flag);
    return cudaGetLastError();
}

cudaError_t launch_mask_i32(const int32_t* v, const int32_t* flag, int64_t G, int32_t* out, cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    mask_i32_kernel<<<(unsigned)std::min<int64_t>((G + 255) / 256, 1024), 256, 0, st>>>(v, flag, G, out);
    return cudaGetLastError();
}

int tcw_blocks(int P) {
    const int ne = P * (P + 1) / 2;
    return (ne + kWNmax - 1) / kWNmax;
}
int tcw_nblk(int P) {
    const int ne = P * (P + 1) / 2, nb = tcw_blocks(P);
    return ((ne + nb - 1) / nb + 15) / 16 * 16;
}
int64_t tcw_npad(int64_t n) { return (n + kWKC - 1) / kWKC * kWKC; }
bool tcw_supported(int P, int xs) { return P >= 5 && P <= 32 && xs >= 8 && xs <= 32 && xs % 4 == 0; }

cudaError_t launch_tcw_prepare(const int64_t* rowptr, const int32_t* col, const void* val, int val_u16,
                               int64_t G, int64_t n, const float* Xrm, int xs, const float* off,
                               const TcwGeom& tw, cudaStream_t st) {
    const size_t esz = val_u16 ? 2 : 4;
    cudaError_t e = cudaMemsetAsync(const_cast<void*>(tw.ydense), 0, (size_t)G * tw.ld * esz, st);
    if (e != cudaSuccess) return e;
    if (G > 0) {
        const unsigned blocks = (unsigned)std::min<int64_t>((G * 32 + 255) / 256, 148 * 32);
        if (val_u16)
            tcw_dense_kernel<uint16_t><<<blocks, 256, 0, st>>>(rowptr, col, static_cast<const uint16_t*>(val), G,
                                                              tw.ld, static_cast<uint16_t*>(const_cast<void*>(tw.ydense)));
        else
            tcw_dense_kernel<float><<<blocks, 256, 0, st>>>(rowptr, col, static_cast<const float*>(val), G, tw.ld,
                                                           static_cast<float*>(const_cast<void*>(tw.ydense)));
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const int64_t tot = (int64_t)(xs + 1) * tw.npad;
    tcw_xt_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 148 * 16), 256, 0, st>>>(
        Xrm, xs, n, tw.npad, off, const_cast<float*>(tw.xt), const_cast<float*>(tw.offp));
    return cudaGetLastError();
}

int tcw_tile_genes(PassKind k) { return k == PASS_MLE ? kMleG : kWM; }

// L.GT = tcw_tile_genes(L.kind) genes per tile; grid (L.nseg, L.ntiles, tcw_blocks(P))
cudaError_t launch_tcw_pass(const PassLaunch& L, const TcwGeom& tw) {
    if ((L.kind != PASS_IRLS && L.kind != PASS_MLE) || L.GT != tcw_tile_genes(L.kind) ||
        !tcw_supported(L.P, L.xs_pad))
        return cudaErrorInvalidValue;
    TcwGeom t = tw;
    t.NA = pass_na(L.kind, L.P);
    if (L.occ_out) t.nblk = tcw_nblk(L.P);
    else if (tw.nblk != tcw_nblk(L.P) || tw.NE != L.P * (L.P + 1) / 2 || tw.P != L.P)
        return cudaErrorInvalidValue;
    if (L.kind == PASS_MLE)
        return L.val_u16 ? run_tcw_xs<uint16_t, true>(L, t) : run_tcw_xs<float, true>(L, t);
    return L.val_u16 ? run_tcw_xs<uint16_t, false>(L, t) : run_tcw_xs<float, false>(L, t);
}

}  // namespace devil
