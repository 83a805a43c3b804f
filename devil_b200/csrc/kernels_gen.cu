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

size_t gen_smem_bytes(PassKind k, int P, int GT) {
    const int ns = pass_ns(k), nwv = pass_nw(k) + pass_nv(k) + pass_nf(k);
    const size_t wt = 8;  // FP64 staging for every pass
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

template <class Pass>
static cudaError_t run(const PassLaunch& L) {
    const size_t smem = gen_smem_bytes(L.kind, L.P, L.GT);
    dim3 grid(L.nseg, L.ntiles);
    auto prm = params_of<Pass>(L.prm);
    cudaError_t e;
    if (L.val_u16) {
        auto k = gen_pass_kernel<Pass, uint16_t>;
        // static shared memory (psi tables) counts against the 48 KB default
        e = raise_dyn_smem(k, smem);
        if (e != cudaSuccess) return e;
        if (L.occ_out) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, k, kGenNT, smem);
        k<<<grid, kGenNT, smem, L.stream>>>(L.geo, prm, L.P, L.GT);
    } else {
        auto k = gen_pass_kernel<Pass, float>;
        e = raise_dyn_smem(k, smem);
        if (e != cudaSuccess) return e;
        if (L.occ_out) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, k, kGenNT, smem);
        k<<<grid, kGenNT, smem, L.stream>>>(L.geo, prm, L.P, L.GT);
    }
    return cudaGetLastError();
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
