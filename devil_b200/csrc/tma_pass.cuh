// Register engine with TMA staging of the design rows (sm_100a).
//
// Same reductions as reg_pass_kernel (GT genes per CTA in registers, p <= 8,
// FP32 per-cell terms) but each fine segment ("chunk") of the design matrix
// X (row-major floats) and of the offsets is copied into shared memory by a
// 1-D bulk tensor-memory-access copy (cp.async.bulk, completion counted on
// an mbarrier), double-buffered so the copy of chunk k+1 overlaps the
// arithmetic of chunk k.  The dense loop and the nonzero corrections then
// read design rows from shared memory: no dependent global gathers remain,
// only the streamed CSR entries.  Requirements (checked by the host): chunk
// starts are multiples of 16 cells and X / offsets are padded by 16 rows so
// every copy starts 16-byte aligned and spans a multiple of 16 bytes.
// mbarrier waits are bounded; on timeout the kernel flags geo.err and
// returns without writing partial sums.
#pragma once
#include "passes.cuh"

namespace devil {

DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

DEV void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
DEV void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
DEV void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// 1-D bulk copy global -> shared (this CTA), completion on bar
DEV void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
constexpr uint32_t kWaitTries = 1u << 22;
DEV bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitTries; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// chunk capacity in cells for a row stride PP (floats)
template <int PP>
struct TmaChunk {
    static constexpr int CH = PP <= 4 ? 2048 : 1024;
    static constexpr int STAGE_FLOATS = CH * PP + CH;  // rows then offsets
};

template <int P, int PP, int GT, int NT, class Pass, class VT>
__global__ void __launch_bounds__(NT) tma_pass_kernel(PassGeom geo, typename Pass::Params prm) {
    static_assert(!Pass::F64, "TMA engine carries FP32 passes");
    constexpr int NE = P * (P + 1) / 2;
    constexpr int NA = Pass::NW * NE + Pass::NV * P + Pass::NF;
    constexpr int NS = Pass::NS;
    constexpr int NAc = NA > 0 ? NA : 1;
    constexpr int NSc = NS > 0 ? NS : 1;
    constexpr int CH = TmaChunk<PP>::CH;
    constexpr int SF = TmaChunk<PP>::STAGE_FLOATS;
    using AW = typename Pass::AW;
    using AS = typename Pass::AS;

    extern __shared__ __align__(128) float tma_smem[];  // [2][SF]
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int abort_flag;

    if (geo.reset_next && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *geo.reset_next = 0;
    const int nact = *geo.n_act;
    const int tile = blockIdx.y;
    if (tile * GT >= nact) return;
    const int seg = blockIdx.x;
    const VT* __restrict__ val = static_cast<const VT*>(geo.val);
    const int nfs = geo.nbound - 1;
    const int b0 = (int)(((int64_t)seg * nfs) / geo.nseg);
    const int b1 = (int)(((int64_t)(seg + 1) * nfs) / geo.nseg);

    // thread 0 issues every copy and tracks which stages have one in flight
    // (and the phase parity it completes) for the abort path
    bool inflight[2] = {false, false};
    uint32_t use_count[2] = {0u, 0u};
    // issue the copy of fine segment b into stage st
    auto issue = [&](int b, int st) {
        inflight[st] = true;
        const int cb = __ldg(geo.bound + b), ce = __ldg(geo.bound + b + 1);
        const int cells4 = ((ce - cb) + 3) & ~3;
        const uint32_t bx = (uint32_t)(cells4 * PP * 4), bo = (uint32_t)(cells4 * 4);
        float* xs = tma_smem + st * SF;
        mbar_arrive_expect_tx(&bars[st], bx + bo);
        bulk_g2s(xs, geo.X + (int64_t)cb * PP, bx, &bars[st]);
        bulk_g2s(xs + CH * PP, geo.off + cb, bo, &bars[st]);
    };
    if (threadIdx.x == 0) {
        abort_flag = 0;
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && b0 < b1) issue(b0, 0);

    int gid[GT];
    float beta[GT][P];
    typename Pass::Gene gp[GT];
#pragma unroll
    for (int j = 0; j < GT; ++j) {
        int slot = tile * GT + j;
        if (slot >= nact) slot = tile * GT;  // duplicate a valid gene; not written
        int g = __ldg(geo.act + slot);
        gid[j] = g;
#pragma unroll
        for (int i = 0; i < P; ++i) beta[j][i] = __ldg(prm.beta + (int64_t)g * P + i) * kLog2e;
        gp[j] = Pass::load(prm, g);
    }
    if constexpr (Pass::TABLES) {
        __shared__ double psitab[GT * 2 * kPsiTab];
        __shared__ double psiscr[GT * kPsiTab];
        __shared__ double psia[GT];
        if (threadIdx.x < GT) {
#pragma unroll
            for (int j = 0; j < GT; ++j)
                if (j == (int)threadIdx.x) psia[j] = gp[j].a;
        }
        __syncthreads();
        build_psi_tables(GT, psia, psitab, psiscr);
#pragma unroll
        for (int j = 0; j < GT; ++j) {
            gp[j].tab.d1 = psitab + (j * 2 + 0) * kPsiTab;
            gp[j].tab.d2 = psitab + (j * 2 + 1) * kPsiTab;
            gp[j].tab.pa = digamma_d(gp[j].a);
            gp[j].tab.ta = trigamma_d(gp[j].a);
        }
    }

    AW aw[GT][NAc];
    AS as[GT][NSc];
#pragma unroll
    for (int j = 0; j < GT; ++j) {
#pragma unroll
        for (int a = 0; a < NAc; ++a) aw[j][a] = 0;
#pragma unroll
        for (int s2 = 0; s2 < NSc; ++s2) as[j][s2] = 0;
    }

    constexpr int UNR = (Pass::NS > 0) ? 2 : 4;
    for (int b = b0, k = 0; b < b1; ++b, ++k) {
        const int st = k & 1;
        if (threadIdx.x == 0 && b + 1 < b1) issue(b + 1, st ^ 1);
        if (!mbar_wait_bounded(&bars[st], (uint32_t)((k >> 1) & 1))) {
            atomicExch(&abort_flag, 1);
        } else if (threadIdx.x == 0) {
            inflight[st] = false;
            ++use_count[st];
        }
        __syncthreads();
        if (abort_flag) break;
        const float* xs = tma_smem + st * SF;
        const float* os = xs + CH * PP;
        const int cb = __ldg(geo.bound + b), ce = __ldg(geo.bound + b + 1);
        const int ncell = ce - cb;
        // dense: every cell of the chunk for every gene of the tile
        for (int cl = threadIdx.x; cl < ncell; cl += NT) {
            float x[P];
            if constexpr (PP == 4) {
                float4 v = *reinterpret_cast<const float4*>(xs + cl * 4);
                float t4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int i = 0; i < P; ++i) x[i] = t4[i];
            } else {
#pragma unroll
                for (int i = 0; i < P; ++i) x[i] = xs[cl * PP + i];
            }
            const float o = os[cl] * kLog2e;
            float zz[NE];
#pragma unroll
            for (int jj = 0; jj < P; ++jj)
#pragma unroll
                for (int ii = 0; ii <= jj; ++ii) zz[tri_index(ii, jj)] = x[ii] * x[jj];
#pragma unroll
            for (int j = 0; j < GT; ++j) {
                float e = o;
#pragma unroll
                for (int i = 0; i < P; ++i) e = fmaf(x[i], beta[j][i], e);
                float mu = ex2_approx(e);
                RegAcc<P, NAc, NSc, AW, AS, float> acc{aw[j], as[j], x, zz};
                Pass::template dense<float>(gp[j], mu, acc);
            }
        }
        // nonzero corrections: CSR entries of this chunk, design rows from smem
#pragma unroll
        for (int j = 0; j < GT; ++j) {
            const int64_t* sp = geo.segptr + (int64_t)gid[j] * geo.nbound;
            const int64_t e0 = __ldg(sp + b), e1 = __ldg(sp + b + 1);
            for (int64_t eb = e0 + threadIdx.x; eb < e1; eb += (int64_t)UNR * NT) {
                int cl[UNR];
                float yy[UNR];
                bool ok[UNR];
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
                    const int64_t e = eb + (int64_t)u * NT;
                    ok[u] = e < e1;
                    cl[u] = ok[u] ? __ldg(geo.col + e) - cb : 0;
                    yy[u] = ok[u] ? load_val(val, e) : 0.f;
                }
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
                    if (!ok[u]) continue;
                    float x[P];
#pragma unroll
                    for (int i = 0; i < P; ++i) x[i] = xs[cl[u] * PP + i];
                    float el = os[cl[u]] * kLog2e;
#pragma unroll
                    for (int i = 0; i < P; ++i) el = fmaf(x[i], beta[j][i], el);
                    float mu = ex2_approx(el);
                    float zz[NE];
#pragma unroll
                    for (int jj = 0; jj < P; ++jj)
#pragma unroll
                        for (int ii = 0; ii <= jj; ++ii) zz[tri_index(ii, jj)] = x[ii] * x[jj];
                    RegAcc<P, NAc, NSc, AW, AS, float> acc{aw[j], as[j], x, zz};
                    Pass::template sparse<float>(gp[j], mu, yy[u], acc);
                }
            }
        }
        __syncthreads();  // stage st is reused by the copy issued next iteration
    }
    if (abort_flag) {
        // let copies still in flight land before the CTA's shared memory goes
        if (threadIdx.x == 0) {
            for (int st = 0; st < 2; ++st)
                if (inflight[st]) mbar_wait_bounded(&bars[st], use_count[st] & 1u);
            atomicExch(geo.err, 1);
        }
        return;
    }

    // block reduction: warp shuffles, then across warps through shared memory
    constexpr int NWARP = NT / 32;
    __shared__ AW redW[NWARP][GT * NAc];
    __shared__ AS redS[NWARP][GT * NSc];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < GT; ++j) {
        if constexpr (NA > 0) {
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                AW v = warp_sum(aw[j][a]);
                if (lane == 0) redW[warp][j * NAc + a] = v;
            }
        }
        if constexpr (NS > 0) {
#pragma unroll
            for (int s2 = 0; s2 < NS; ++s2) {
                AS v = warp_sum(as[j][s2]);
                if (lane == 0) redS[warp][j * NSc + s2] = v;
            }
        }
    }
    __syncthreads();
    if constexpr (NA > 0) {
        for (int t = threadIdx.x; t < GT * NA; t += NT) {
            int j = t / NA, a = t - j * NA;
            int slot = tile * GT + j;
            if (slot >= nact) continue;
            AW s2 = 0;
#pragma unroll
            for (int w = 0; w < NWARP; ++w) s2 += redW[w][j * NAc + a];
            static_cast<AW*>(geo.partW)[((int64_t)seg * geo.slot_stride + slot) * NA + a] = s2;
        }
    }
    if constexpr (NS > 0) {
        for (int t = threadIdx.x; t < GT * NS; t += NT) {
            int j = t / NS, s2 = t - j * NS;
            int slot = tile * GT + j;
            if (slot >= nact) continue;
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < NWARP; ++w) v += (double)redS[w][j * NSc + s2];
            geo.partS[((int64_t)seg * geo.slot_stride + slot) * NS + s2] = v;
        }
    }
}

}  // namespace devil
