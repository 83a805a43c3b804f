// Instantiations of the shared-memory engine (any p <= 32) for every pass.
#include "internal.h"

namespace devil {

int gen_default_gt(PassKind k, int P) {
    const int na = pass_na(k, P), ns = pass_ns(k);
    for (int gt = 8; gt >= 1; gt >>= 1) {
        if ((gt * na + kGenNT - 1) / kGenNT <= kGenKMAX && gt * ns <= kGenNT) return gt;
    }
    return 0;  // p too large for this engine
}

// FP32 staging (the plain form) only for the passes with FP32 per-cell
// arithmetic; MOM and bread/meat stay FP64 in every form
bool gen_f32_staging(PassKind k, int plain) {
    return plain && (k == PASS_IRLS || k == PASS_MLE);
}

size_t gen_smem_bytes(PassKind k, int P, int GT, int plain) {
    const int ns = pass_ns(k), nwv = pass_nw(k) + pass_nv(k) + pass_nf(k);
    const size_t wt = gen_f32_staging(k, plain) ? 4 : 8;
    const int TC = kGenNT / GT;
    const int XS = (P + 1) | 1;
    size_t b = gen_wt_offset(ns, GT);
    b += (size_t)TC * XS * wt;                 // xsm
    b += (size_t)nwv * kGenNT * wt;            // wts
    b += (size_t)kGenNT * 4;                   // ys
    b += (size_t)GT * P * 4;                   // betas
    return b + 16;
}

template <class Pass>
static typename Pass::Params params_of(const PassParamsAny& a);
template <> PassIRLS::Params params_of<PassIRLS>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.k}; }
template <> PassMOM::Params params_of<PassMOM>(const PassParamsAny& a) { return {a.beta, a.beta_d}; }
template <> PassMLE::Params params_of<PassMLE>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.log_theta}; }
template <> PassSandwich::Params params_of<PassSandwich>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.theta}; }

template <class Pass, bool F32W, class K>
static cudaError_t go(const PassLaunch& L, K* k, size_t smem) {
    // static shared memory (psi tables) counts against the 48 KB default
    cudaError_t e = raise_dyn_smem(k, smem);
    if (e != cudaSuccess) return e;
    if (L.occ_out) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, k, kGenNT, smem);
    dim3 grid(L.nseg, L.ntiles);
    k<<<grid, kGenNT, smem, L.stream>>>(L.geo, params_of<Pass>(L.prm), L.P, L.GT);
    return cudaGetLastError();
}

template <class Pass>
static cudaError_t run(const PassLaunch& L) {
    const size_t smem = gen_smem_bytes(L.kind, L.P, L.GT, L.plain);
    if constexpr (!Pass::F64) {
        if (gen_f32_staging(L.kind, L.plain))
            return L.val_u16 ? go<Pass, true>(L, gen_pass_kernel<Pass, uint16_t, true>, smem)
                             : go<Pass, true>(L, gen_pass_kernel<Pass, float, true>, smem);
    }
    return L.val_u16 ? go<Pass, false>(L, gen_pass_kernel<Pass, uint16_t, false>, smem)
                     : go<Pass, false>(L, gen_pass_kernel<Pass, float, false>, smem);
}

cudaError_t launch_gen_pass(const PassLaunch& L) {
    if (L.P < 1 || L.P > 32) return cudaErrorInvalidValue;
    if (L.GT < 1 || (L.GT * pass_na(L.kind, L.P) + kGenNT - 1) / kGenNT > kGenKMAX)
        return cudaErrorInvalidValue;
    switch (L.kind) {
        case PASS_IRLS: return run<PassIRLS>(L);
        case PASS_MOM: return run<PassMOM>(L);
        case PASS_MLE: return run<PassMLE>(L);
        case PASS_SANDWICH: return run<PassSandwich>(L);
    }
    return cudaErrorInvalidValue;
}

}  // namespace devil
