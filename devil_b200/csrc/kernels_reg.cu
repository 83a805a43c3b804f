// Instantiations of the register engine (p <= 8) for every pass.
#include "internal.h"
#include "tma_pass.cuh"

namespace devil {

constexpr int kRegNT = 256;

int reg_max_p() { return 8; }

int tma_chunk_cells(int xs) { return xs <= 4 ? TmaChunk<4>::CH : TmaChunk<8>::CH; }

int reg_default_gt(PassKind k, int P) {
    switch (k) {
        case PASS_IRLS: return P <= 6 ? 4 : 2;
        case PASS_SANDWICH: return P <= 2 ? 8 : (P <= 4 ? 4 : (P <= 6 ? 2 : 1));
        case PASS_MOM: return 8;
        case PASS_MLE: return 1;
    }
    return 1;
}

bool reg_gt_supported(PassKind k, int P, int GT) {
    if (P < 1 || P > 8) return false;
    if (k == PASS_IRLS) {
        int mx = P <= 4 ? 8 : (P <= 6 ? 4 : 2);
        return GT == 1 || GT == 2 || (GT == 4 && mx >= 4) || (GT == 8 && mx >= 8);
    }
    if (k == PASS_MLE) return GT == 1 || GT == (P <= 2 ? 4 : (P <= 4 ? 2 : 1));
    return GT == reg_default_gt(k, P);
}

template <PassKind K> struct PassOf;
template <> struct PassOf<PASS_IRLS> { using T = PassIRLS; };
template <> struct PassOf<PASS_MOM> { using T = PassMOM; };
template <> struct PassOf<PASS_MLE> { using T = PassMLE; };
template <> struct PassOf<PASS_SANDWICH> { using T = PassSandwich; };

template <PassKind K>
static typename PassOf<K>::T::Params make_params(const PassParamsAny& a);
template <> PassIRLS::Params make_params<PASS_IRLS>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.k}; }
template <> PassMOM::Params make_params<PASS_MOM>(const PassParamsAny& a) { return {a.beta, a.beta_d}; }
template <> PassMLE::Params make_params<PASS_MLE>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.log_theta}; }
template <> PassSandwich::Params make_params<PASS_SANDWICH>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.theta}; }

template <PassKind K, int P, int GT>
static cudaError_t run(const PassLaunch& L) {
    using Pass = typename PassOf<K>::T;
    constexpr int PP = P <= 1 ? 1 : (P <= 2 ? 2 : (P <= 4 ? 4 : 8));
    if (L.xs_pad != PP) return cudaErrorInvalidValue;
    dim3 grid(L.nseg, L.ntiles);
    auto prm = make_params<K>(L.prm);
    if (L.occ_out) {
        const void* f;
        if constexpr (K == PASS_IRLS)
            f = L.val_u16 ? (const void*)reg_pass_kernel<P, PP, GT, kRegNT, Pass, uint16_t>
                          : (const void*)reg_pass_kernel<P, PP, GT, kRegNT, Pass, float>;
        else
            f = L.val_u16 ? (const void*)reg_pass_kernel_b1<P, PP, GT, kRegNT, Pass, uint16_t>
                          : (const void*)reg_pass_kernel_b1<P, PP, GT, kRegNT, Pass, float>;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(L.occ_out, f, kRegNT, 0);
    }
    if constexpr (!Pass::F64) {
        if (L.use_tma) {
            constexpr size_t smem = 2 * TmaChunk<PP>::STAGE_FLOATS * sizeof(float);
            if (L.val_u16) {
                auto k = tma_pass_kernel<P, PP, GT, kRegNT, Pass, uint16_t>;
                cudaError_t e = raise_dyn_smem(k, smem);
                if (e != cudaSuccess) return e;
                k<<<grid, kRegNT, smem, L.stream>>>(L.geo, prm);
            } else {
                auto k = tma_pass_kernel<P, PP, GT, kRegNT, Pass, float>;
                cudaError_t e = raise_dyn_smem(k, smem);
                if (e != cudaSuccess) return e;
                k<<<grid, kRegNT, smem, L.stream>>>(L.geo, prm);
            }
            return cudaGetLastError();
        }
    }
    if constexpr (K == PASS_IRLS) {
        if (L.val_u16)
            reg_pass_kernel<P, PP, GT, kRegNT, Pass, uint16_t><<<grid, kRegNT, 0, L.stream>>>(L.geo, prm);
        else
            reg_pass_kernel<P, PP, GT, kRegNT, Pass, float><<<grid, kRegNT, 0, L.stream>>>(L.geo, prm);
    } else {
        if (L.val_u16)
            reg_pass_kernel_b1<P, PP, GT, kRegNT, Pass, uint16_t><<<grid, kRegNT, 0, L.stream>>>(L.geo, prm);
        else
            reg_pass_kernel_b1<P, PP, GT, kRegNT, Pass, float><<<grid, kRegNT, 0, L.stream>>>(L.geo, prm);
    }
    return cudaGetLastError();
}

template <PassKind K, int P>
static cudaError_t run_gt(const PassLaunch& L) {
    if constexpr (K == PASS_IRLS) {
        switch (L.GT) {
            case 1: return run<K, P, 1>(L);
            case 2: return run<K, P, 2>(L);
            case 4: if constexpr (P <= 6) return run<K, P, 4>(L); break;
            case 8: if constexpr (P <= 4) return run<K, P, 8>(L); break;
        }
        return cudaErrorInvalidValue;
    } else if constexpr (K == PASS_MLE) {
        constexpr int G = P <= 2 ? 4 : (P <= 4 ? 2 : 1);
        if (L.GT == G) return run<K, P, G>(L);
        if constexpr (G != 1) {
            if (L.GT == 1) return run<K, P, 1>(L);
        }
        return cudaErrorInvalidValue;
    } else {
        constexpr int G = (K == PASS_MOM) ? 8
                        : (K == PASS_MLE) ? (P <= 2 ? 4 : (P <= 4 ? 2 : 1))
                        : (P <= 2 ? 8 : (P <= 4 ? 4 : (P <= 6 ? 2 : 1)));
        if (L.GT != G) return cudaErrorInvalidValue;
        return run<K, P, G>(L);
    }
}

template <PassKind K>
static cudaError_t run_p(const PassLaunch& L) {
    switch (L.P) {
        case 1: return run_gt<K, 1>(L);
        case 2: return run_gt<K, 2>(L);
        case 3: return run_gt<K, 3>(L);
        case 4: return run_gt<K, 4>(L);
        case 5: return run_gt<K, 5>(L);
        case 6: return run_gt<K, 6>(L);
        case 7: return run_gt<K, 7>(L);
        case 8: return run_gt<K, 8>(L);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_reg_pass(const PassLaunch& L) {
    switch (L.kind) {
        case PASS_IRLS: return run_p<PASS_IRLS>(L);
        case PASS_MOM: return run_p<PASS_MOM>(L);
        case PASS_MLE: return run_p<PASS_MLE>(L);
        case PASS_SANDWICH: return run_p<PASS_SANDWICH>(L);
    }
    return cudaErrorInvalidValue;
}

}  // namespace devil
