// Per-gene finalize kernels: reduce the per-segment partial sums of a pass
// in FP64 and apply the reference's per-gene step.  One warp per gene.
#include <type_traits>

#include "internal.h"
#include "warp_la.cuh"

namespace devil {

static inline unsigned nblk(int64_t m, int t) { return (unsigned)((m + t - 1) / t); }

// sums[a] = sum over segments of part[seg][slot][a]  (lanes split a)
template <class T>
DEV void reduce_partials(const T* part, int nseg, int slot_stride, int slot, int stride, int count,
                         double* sums, int lane) {
#pragma unroll 4
    for (int a = lane; a < count; a += 32) {
        double s = 0.0;
        for (int seg = 0; seg < nseg; ++seg)
            s += (double)part[((int64_t)seg * slot_stride + slot) * stride + a];
        sums[a] = s;
    }
}

// warps per finalize block given the shared bytes one warp needs
static int fin_warps(size_t per_warp) {
    int w = (int)((96 * 1024) / (per_warp > 0 ? per_warp : 1));
    return w < 1 ? 1 : (w > 4 ? 4 : w);
}

DEV void unpack_sym(int P, const double* packed, double* M) {
    for (int j = 0; j < P; ++j)
        for (int i = 0; i <= j; ++i) {
            double v = packed[tri_index(i, j)];
            M[j * P + i] = v;
            M[i * P + j] = v;
        }
}

// ------------------------------------------------------------------
// IRLS step (src/beta.cpp:38-46): delta = H^-1 score, beta += delta,
// converged when max|delta| < eps; NaN in delta[0] stops the gene.
// ------------------------------------------------------------------
template <class TW>
__global__ void irls_finalize_kernel(const TW* partW, int nseg, int slot_stride, int P,
                                     const int32_t* act, const int32_t* n_act, int32_t* act_next,
                                     int32_t* n_next, double* beta, float* beta_f, int32_t* iters,
                                     int32_t* status, int max_iter, double eps, const float* kf) {
    extern __shared__ double fsh[];
    const int NE = P * (P + 1) / 2, NA = NE + P, LD = wla_ld(P);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = NA + P * LD + P;  // sums, H, then perm and step (P ints each)
    double* sums = fsh + warp * per;
    double* H = sums + NA;
    int* perm = reinterpret_cast<int*>(H + P * LD);
    int* step = perm + P;
    const int slot = blockIdx.x * (blockDim.x >> 5) + warp;
    const int nact = *n_act;
    if (slot >= nact) return;
    const int g = act[slot];
    reduce_partials(partW, nseg, slot_stride, slot, NA, NA, sums, lane);
    __syncwarp();
    // the pass accumulates H / k^2 and -score / k (see PassIRLS)
    const double k = (double)kf[g];
    warp_unpack_sym(P, sums, k * k, 0.0, H, LD);
    const double s_own = lane < P ? -k * sums[NE + lane] : 0.0;
    warp_lu(H, LD, P, perm, step);
    const double x_own = warp_lu_solve(H, LD, P, perm, step, s_own);
    double b = 0.0;
    if (lane < P) {
        b = beta[(int64_t)g * P + lane] + x_own;
        beta[(int64_t)g * P + lane] = b;
        beta_f[(int64_t)g * P + lane] = (float)b;
    }
    // max |x| (NaN entries never compare greater) and x_0
    double mx = lane < P ? fabs(x_own) : 0.0;
    mx = (mx == mx) ? mx : 0.0;
    mx = warp_max(mx);
    const double x0 = __shfl_sync(0xffffffffu, x_own, 0);
    if (lane != 0) return;
    const int it = iters[g] + 1;
    iters[g] = it;
    const bool isnan0 = !(x0 == x0);
    const bool conv = mx < eps;
    if (isnan0) {
        status[g] = 2;  // DEVIL_GENE_NAN
    } else if (conv) {
        status[g] = 0;
    } else if (it >= max_iter) {
        status[g] = 1;
    } else {
        int pos = atomicAdd(n_next, 1);
        act_next[pos] = g;
    }
}

cudaError_t launch_irls_finalize(const void* partW, bool wide, int nseg, int slot_stride, int P,
                                 const int32_t* act, const int32_t* n_act, int max_slots,
                                 int32_t* act_next, int32_t* n_next, double* beta, float* beta_f,
                                 int32_t* iters, int32_t* status, int max_iter, double eps,
                                 const float* k, cudaStream_t st) {
    if (max_slots <= 0) return cudaSuccess;
    const int NA = P * (P + 1) / 2 + P;
    const size_t per = (size_t)(NA + P * wla_ld(P) + P) * sizeof(double);
    const int w = fin_warps(per);
    const size_t smem = per * w;
    auto go = [&](auto* pw) -> cudaError_t {
        using TW = std::remove_const_t<std::remove_pointer_t<decltype(pw)>>;
        if (smem > 48 * 1024) {
            cudaError_t e = raise_dyn_smem(irls_finalize_kernel<TW>, smem);
            if (e != cudaSuccess) return e;
        }
        irls_finalize_kernel<TW><<<nblk(max_slots, w), 32 * w, smem, st>>>(
            pw, nseg, slot_stride, P, act, n_act, act_next, n_next, beta, beta_f, iters, status,
            max_iter, eps, k);
        return cudaGetLastError();
    };
    // the register engine leaves FP32 partial sums, the generic engine FP64
    return wide ? go(static_cast<const double*>(partW)) : go(static_cast<const float*>(partW));
}

// ------------------------------------------------------------------
// IRLS step of the design-group engine's slice-major pass, warp per gene,
// with the assembly folded in: the group sums of the gene's per-slice sums
// (a segmented warp scan over the slices), H = k^2 sum over (group, pair)
// lists, score = -k sum over (group, entry) lists -- the sums of
// grp_assemble_kernel + irls_finalize_kernel, without the round trip of the
// p x p partial sums through global memory -- then the LU, the solve and the
// update of irls_finalize_kernel.
// ------------------------------------------------------------------
// Newton step of the SPD system H x = s when the exclusive columns D
// (geo.colD, m = P - nA of them) form a diagonal block of H:
//   S = H_AA - H_AD diag(H_DD)^-1 H_DA        (Schur complement, nA x nA)
//   S x_A = s_A - H_AD diag(H_DD)^-1 s_D,      x_D = diag(H_DD)^-1 (s_D - H_DA x_A)
// Lane t < m handles exclusive column colD[t]; the sums over t are warp
// sums in lane order.  Exact in exact arithmetic, like the LU of H (the
// arrowhead H of a one-hot design costs O(p) instead of O(p^3)).  Returns
// the step of column `lane` (lanes < P).
// HA: the rows of the dense columns ([nA][P]), Hd: the diagonal ([P])
DEV double schur_step(const GrpGeom& geo, const double* HA, const double* Hd, int P, double* Sm, int* perm,
                      int* step, double s_own, int lane) {
    constexpr unsigned FULL = 0xffffffffu;
    const int k = geo.nA, m = P - k;
    const int LDk = wla_ld(k);
    const int c = lane < m ? __ldg(geo.colD + lane) : 0;
    const double sc = __shfl_sync(FULL, s_own, c);
    double r = 0.0, hA[8];
    if (lane < m) r = 1.0 / Hd[c];
#pragma unroll
    for (int a = 0; a < 8; ++a) hA[a] = (a < k && lane < m) ? HA[a * P + c] : 0.0;
    double rhs_own = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        if (a >= k) break;
        const int ca = __ldg(geo.colA + a);
        const double ta = warp_sum(lane < m ? hA[a] * sc * r : 0.0);
        (void)ca;
        const double sa = __shfl_sync(FULL, s_own, ca);
        if (lane == a) rhs_own = sa - ta;
#pragma unroll
        for (int b = 0; b <= a; ++b) {
            const double tab = warp_sum(hA[a] * hA[b] * r);
            if (lane == 0) {
                const double v = HA[a * P + __ldg(geo.colA + b)] - tab;
                Sm[a * LDk + b] = v;
                Sm[b * LDk + a] = v;
            }
        }
    }
    __syncwarp();
    warp_lu(Sm, LDk, k, perm, step);
    const double xa = warp_lu_solve(Sm, LDk, k, perm, step, rhs_own);  // lanes < k
    double dot = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        if (a >= k) break;
        dot += hA[a] * __shfl_sync(FULL, xa, a);
    }
    const double xd = (sc - dot) * r;  // lanes < m
    const int pc = lane < P ? __ldg(geo.colpos + lane) : 0;
    const double fromA = __shfl_sync(FULL, xa, pc >= 0 ? pc : 0);
    const double fromD = __shfl_sync(FULL, xd, pc < 0 ? -1 - pc : 0);
    return pc >= 0 ? fromA : fromD;
}

constexpr int kSchurScratch = 8 * wla_ld(8);  // doubles: the Schur complement of at most 8 dense columns

__global__ void grp_irls_finalize_kernel(GrpGeom geo, int32_t* act_next, int32_t* n_next,
                                         double* beta, float* beta_f, int32_t* iters,
                                         int32_t* status, int max_iter, double eps,
                                         const float* kf, int8_t* keep) {
    extern __shared__ double fsh[];
    const int P = geo.P, U = geo.U, C = geo.C, S = geo.S, LD = wla_ld(P);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // group sums, then H (P x LD) for the LU step, or the compact store of
    // the Schur step (rows of the dense columns, the diagonal) and its
    // scratch; then perm and step (P ints each)
    const int k_a = geo.nA;
    const int per = k_a > 0 ? 2 * U + k_a * P + P + kSchurScratch + P : 2 * U + P * LD + P;
    double* gs = fsh + warp * per;
    double* H = gs + 2 * U;
    double* Sm = H + (k_a > 0 ? k_a * P + P : P * LD);
    int* perm = reinterpret_cast<int*>(k_a > 0 ? Sm + kSchurScratch : H + P * LD);
    int* step = perm + P;
    const int slot = blockIdx.x * (blockDim.x >> 5) + warp;
    if (slot >= *geo.n_act) return;
    const int g = geo.act[slot];
    const double* gsum = geo.gsum + (int64_t)slot * S * 2;
    // group sums: lanes over slices (one coalesced load each), then a
    // segmented warp scan over each run of slices of one group (a group's
    // slices are contiguous, keyed u * C + c); the run's last lane adds it in
    for (int i = lane; i < 2 * U; i += 32) gs[i] = 0.0;
    __syncwarp();
    for (int b = 0; b < S; b += 32) {
        const int sl = b + lane;
        const bool ok = sl < S;
        double v0 = ok ? gsum[sl * 2] : 0.0, v1 = ok ? gsum[sl * 2 + 1] : 0.0;
        const int q = ok ? __ldg(geo.sl_key + sl) / C : -1 - lane;  // past S: runs of their own
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double t0 = __shfl_up_sync(0xffffffffu, v0, o), t1 = __shfl_up_sync(0xffffffffu, v1, o);
            const int qo = __shfl_up_sync(0xffffffffu, q, o);
            if (lane >= o && qo == q) {
                v0 += t0;
                v1 += t1;
            }
        }
        const int qn = __shfl_down_sync(0xffffffffu, q, 1);
        if (ok && (lane == 31 || qn != q)) {
            gs[2 * q] += v0;
            gs[2 * q + 1] += v1;
        }
        __syncwarp();
    }
    // the pass accumulates H / k^2 and -score / k (see PassIRLS)
    const double k = (double)kf[g];
    const double k2 = k * k;
    const int NE = P * (P + 1) / 2;
    const int nout = k_a > 0 ? geo.n_need : NE;
    for (int o = lane; o < nout; o += 32) {
        const int a = k_a > 0 ? __ldg(geo.need_q + o) : o;
        // four partial sums: the intercept's lists run over every group
        const int q0 = __ldg(geo.qptr + a), q1 = __ldg(geo.qptr + a + 1);
        double s4[4] = {0.0, 0.0, 0.0, 0.0};
        int e = q0;
        for (; e + 4 <= q1; e += 4) {
#pragma unroll
            for (int r = 0; r < 4; ++r) s4[r] += gs[__ldg(geo.qu + e + r) * 2] * __ldg(geo.qv + e + r);
        }
        for (; e < q1; ++e) s4[0] += gs[__ldg(geo.qu + e) * 2] * __ldg(geo.qv + e);
        const double s = (s4[0] + s4[1]) + (s4[2] + s4[3]);
        const double v = s * k2;
        if (k_a > 0) {
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                const int d = __ldg(geo.need_d + 3 * o + t);
                if (d >= 0) H[d] = v;
            }
        } else {
            // packed upper-triangle index a = j (j + 1) / 2 + i, i <= j
            int j = (int)((sqrtf(8.f * (float)a + 1.f) - 1.f) * 0.5f);
            while (j * (j + 1) / 2 > a) --j;
            while ((j + 1) * (j + 2) / 2 <= a) ++j;
            const int i = a - j * (j + 1) / 2;
            H[i * LD + j] = v;
            H[j * LD + i] = v;
        }
    }
    double s_own = 0.0;
    if (lane < P) {
        const int v0 = __ldg(geo.vptr + lane), v1 = __ldg(geo.vptr + lane + 1);
        double s4[4] = {0.0, 0.0, 0.0, 0.0};
        int e = v0;
        for (; e + 4 <= v1; e += 4) {
#pragma unroll
            for (int r = 0; r < 4; ++r) s4[r] += gs[__ldg(geo.vu + e + r) * 2 + 1] * __ldg(geo.vv + e + r);
        }
        for (; e < v1; ++e) s4[0] += gs[__ldg(geo.vu + e) * 2 + 1] * __ldg(geo.vv + e);
        s_own = -k * ((s4[0] + s4[1]) + (s4[2] + s4[3]));
    }
    __syncwarp();
    double x_own;
    if (geo.nA > 0) {
        x_own = schur_step(geo, H, H + k_a * P, P, Sm, perm, step, s_own, lane);
    } else {
        warp_lu(H, LD, P, perm, step);
        x_own = warp_lu_solve(H, LD, P, perm, step, s_own);
    }
    double b_own = 0.0;
    if (lane < P) {
        b_own = beta[(int64_t)g * P + lane] + x_own;
        beta[(int64_t)g * P + lane] = b_own;
        beta_f[(int64_t)g * P + lane] = (float)b_own;
    }
    double mx = lane < P ? fabs(x_own) : 0.0;
    mx = (mx == mx) ? mx : 0.0;  // NaN entries never compare greater
    mx = warp_max(mx);
    const double x0 = __shfl_sync(0xffffffffu, x_own, 0);
    const int it = iters[g] + 1;
    // (the same decision on every lane)
    const bool more = (x0 == x0) && !(mx < eps) && it < max_iter;
    if (more && geo.rowexp) {
        // the next pass's exp(x_u . beta) of this gene (rows of the design
        // in shared memory order, as grp_rowexp_kernel sums them); H is free
        __syncwarp();
        if (lane < P) H[lane] = b_own;
        __syncwarp();
        for (int uu = lane; uu < U; uu += 32) {
            double a = 0.0;
            for (int e = __ldg(geo.rptr + uu); e < __ldg(geo.rptr + uu + 1); ++e)
                a += __ldg(geo.rval + e) * H[__ldg(geo.rcol + e)];
            geo.rowexp[(int64_t)g * U + uu] = exp(a);
        }
    }
    if (lane != 0) return;
    iters[g] = it;
    if (!(x0 == x0)) {
        status[g] = 2;  // DEVIL_GENE_NAN
    } else if (mx < eps) {
        status[g] = 0;
    } else if (it >= max_iter) {
        status[g] = 1;
    }
    if (keep) keep[g] = more ? 1 : 0;
    else if (more) act_next[atomicAdd(n_next, 1)] = g;
}

cudaError_t launch_grp_irls_finalize(const GrpGeom& geo, int max_slots, int32_t* act_next,
                                     int32_t* n_next, double* beta, float* beta_f, int32_t* iters,
                                     int32_t* status, int max_iter, double eps, const float* k,
                                     cudaStream_t st, int8_t* keep) {
    if (max_slots <= 0) return cudaSuccess;
    const int P = geo.P, na = geo.nA;
    const size_t per =
        (size_t)(na > 0 ? 2 * geo.U + na * P + P + kSchurScratch + P : 2 * geo.U + P * wla_ld(P) + P) *
        sizeof(double);
    const int w = fin_warps(per);
    const size_t smem = per * w;
    if (smem > 48 * 1024) {
        cudaError_t e = raise_dyn_smem(grp_irls_finalize_kernel, smem);
        if (e != cudaSuccess) return e;
    }
    grp_irls_finalize_kernel<<<nblk(max_slots, w), 32 * w, smem, st>>>(
        geo, act_next, n_next, beta, beta_f, iters, status, max_iter, eps, k, keep);
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// MOM (src/mom_overdispersion.cpp:47-53)
// ------------------------------------------------------------------
__global__ void mom_finalize_kernel(const double* partS, int nseg, int slot_stride,
                                    const int32_t* act, const int32_t* n_act, int64_t n, int P,
                                    double* theta) {
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= *n_act) return;
    int g = act[slot];
    double num = 0.0, den = 0.0;
    for (int seg = 0; seg < nseg; ++seg) {
        const double* p = partS + ((int64_t)seg * slot_stride + slot) * 2;
        num += p[0];
        den += p[1];
    }
    double corr = (double)n / (double)(n - P);
    double th = 0.0;
    if (den > 0.0) {
        th = corr * num / den;
        if (th < 0.0) th = 0.0;
    }
    theta[g] = th;
}
cudaError_t launch_mom_finalize(const double* partS, int nseg, int slot_stride,
                                const int32_t* act, const int32_t* n_act, int max_slots,
                                int64_t n, int P, double* theta, cudaStream_t st) {
    if (max_slots <= 0) return cudaSuccess;
    mom_finalize_kernel<<<nblk(max_slots, 128), 128, 0, st>>>(partS, nseg, slot_stride, act, n_act,
                                                              n, P, theta);
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// MLE of log theta (R/overdispersion.R:25-115 with the score and its
// derivative of src/overdispersion.cpp:95-242), bracketed Newton.
// ------------------------------------------------------------------
constexpr double kCrFactor = 0.99;  // src/overdispersion.cpp:25

__global__ void mle_init_kernel(const double* stats, int64_t G, MleState s, int32_t* act,
                                int32_t* n_act) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G;
         g += (int64_t)gridDim.x * blockDim.x) {
        s.it[g] = 0;
        if (stats[g * 6 + 2] == 0.0) {  // all(y == 0) -> 0
            s.phase[g] = 2;
            s.theta[g] = 0.0;
            s.x[g] = -INFINITY;
        } else {
            s.phase[g] = 0;
            s.x[g] = log(1e-8);
            if (!s.keep) act[atomicAdd(n_act, 1)] = (int32_t)g;
        }
        if (s.keep) s.keep[g] = s.phase[g] == 0 ? 1 : 0;
    }
}
cudaError_t launch_mle_init(const double* stats, int64_t G, int64_t n, MleState s, int32_t* act,
                            int32_t* n_act, cudaStream_t st) {
    (void)n;
    if (G == 0) return cudaSuccess;
    mle_init_kernel<<<(unsigned)std::min<int64_t>(nblk(G, 256), 1024), 256, 0, st>>>(stats, G, s,
                                                                                     act, n_act);
    return cudaGetLastError();
}

// The Cox-Reid terms tr(B^-1 db), tr((B^-1 db)^2), tr(B^-1 d2b) (B = b + 1e-6 I)
// when the exclusive columns D (colD, m of them) make b, db and d2b diagonal
// on D x D.  With Q = B_AD, delta = diag(B_DD) and S = B_AA - Q delta^-1 Q^T
// (the Schur complement on the nA dense columns A):
//   B^-1 = Y + V S^-1 V^T,  Y = [0 0; 0 delta^-1],  V = [I; -delta^-1 Q^T],
// so for E = db (e = diag(E_DD)):
//   tr(B^-1 E)     = sum e/delta + tr(S^-1 G),            G = V^T E V
//   tr((B^-1 E)^2) = sum (e/delta)^2 + 2 tr(S^-1 K) + tr((S^-1 G)^2),
//                    K = sum_t w_t w_t^T / delta_t,  w_t = E_A,t - Q_t e_t / delta_t
// and likewise tr(B^-1 d2b).  Lane t < m holds column colD[t]; the sums over
// t are warp sums; the nA x nA algebra runs on lane 0.  O(p nA^2) per gene
// instead of the O(p^3) factorisation, inverse and product.
DEV void mle_cr_structured(const double* sums, int P, int NE, int k, const int32_t* colA,
                           const int32_t* colD, double* Wk, double& ddetb, double& trmm, double& trbd2) {
    const int lane = threadIdx.x & 31, m = P - k;
    auto pk = [&](int base, int i, int j) { return i <= j ? sums[base + tri_index(i, j)] : sums[base + tri_index(j, i)]; };
    const int c = lane < m ? __ldg(colD + lane) : 0;
    double rd = 0.0, e = 0.0, e2 = 0.0;
    double q[8], w1[8], w2[8];
    if (lane < m) {
        rd = 1.0 / (pk(0, c, c) + 1e-6);
        e = pk(NE, c, c);
        e2 = pk(2 * NE, c, c);
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        q[a] = w1[a] = w2[a] = 0.0;
        if (a < k && lane < m) {
            const int ca = __ldg(colA + a);
            q[a] = pk(0, ca, c);
            w1[a] = pk(NE, ca, c) - q[a] * e * rd;
            w2[a] = pk(2 * NE, ca, c) - q[a] * e2 * rd;
        }
    }
    const double se = warp_sum(e * rd), see = warp_sum(e * rd * e * rd), se2 = warp_sum(e2 * rd);
    // k x k blocks on lane 0: S, G, K, G2, then two scratch blocks
    const int kk = k * k;
    double* Sm = Wk;
    double* Gm = Wk + kk;
    double* Km = Wk + 2 * kk;
    double* G2 = Wk + 3 * kk;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        if (a >= k) break;
        const int ca = __ldg(colA + a);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            if (b >= k) break;
            const int cb = __ldg(colA + b);
            // V^T E V = E_AA - Q d^-1 E_DA - W1_D d^-1 Q^T with W1_D = E_AD - Q d^-1 diag(e)
            const double qq = warp_sum(q[a] * q[b] * rd);
            const double qe = warp_sum(q[a] * (w1[b] + q[b] * e * rd) * rd);
            const double wq = warp_sum(w1[a] * q[b] * rd);
            const double ww = warp_sum(w1[a] * w1[b] * rd);
            const double qe2 = warp_sum(q[a] * (w2[b] + q[b] * e2 * rd) * rd);
            const double w2q = warp_sum(w2[a] * q[b] * rd);
            if (lane == 0) {
                Sm[a * k + b] = pk(0, ca, cb) + (a == b ? 1e-6 : 0.0) - qq;
                Gm[a * k + b] = pk(NE, ca, cb) - qe - wq;
                Km[a * k + b] = ww;
                G2[a * k + b] = pk(2 * NE, ca, cb) - qe2 - w2q;
            }
        }
    }
    __syncwarp();
    if (lane != 0) return;
    // S^-1 by Gauss-Jordan with partial pivoting (S is SPD), into Si
    double* Si = Wk + 4 * kk;
    double* T = Wk + 5 * kk;
    for (int i = 0; i < kk; ++i) {
        T[i] = Sm[i];
        Si[i] = (i / k == i % k) ? 1.0 : 0.0;
    }
    for (int col = 0; col < k; ++col) {
        int piv = col;
        for (int r = col + 1; r < k; ++r)
            if (fabs(T[r * k + col]) > fabs(T[piv * k + col])) piv = r;
        if (piv != col)
            for (int j = 0; j < k; ++j) {
                double t0 = T[col * k + j];
                T[col * k + j] = T[piv * k + j];
                T[piv * k + j] = t0;
                t0 = Si[col * k + j];
                Si[col * k + j] = Si[piv * k + j];
                Si[piv * k + j] = t0;
            }
        const double inv = 1.0 / T[col * k + col];
        for (int j = 0; j < k; ++j) {
            T[col * k + j] *= inv;
            Si[col * k + j] *= inv;
        }
        for (int r = 0; r < k; ++r) {
            if (r == col) continue;
            const double f = T[r * k + col];
            for (int j = 0; j < k; ++j) {
                T[r * k + j] -= f * T[col * k + j];
                Si[r * k + j] -= f * Si[col * k + j];
            }
        }
    }
    // traces; T = S^-1 G
    double t1 = 0.0, tk = 0.0, t2 = 0.0;
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) {
            t1 += Si[a * k + b] * Gm[b * k + a];
            tk += Si[a * k + b] * Km[b * k + a];
            t2 += Si[a * k + b] * G2[b * k + a];
        }
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) {
            double v = 0.0;
            for (int j = 0; j < k; ++j) v += Si[a * k + j] * Gm[j * k + b];
            T[a * k + b] = v;
        }
    double tgg = 0.0;
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) tgg += T[a * k + b] * T[b * k + a];
    ddetb = se + t1;
    trmm = see + 2.0 * tk + tgg;
    trbd2 = se2 + t2;
}

template <class TW>
__global__ void mle_finalize_kernel(const TW* partW, const double* partS, int nseg,
                                    int slot_stride, int P, const double* stats, int64_t n,
                                    const int32_t* act, const int32_t* n_act, int32_t* act_next,
                                    int32_t* n_next, MleState st, int max_iter, int cox_reid,
                                    int nA, const int32_t* colA, const int32_t* colD) {
    extern __shared__ double fsh[];
    const int NE = P * (P + 1) / 2, NA = 3 * NE + 2;  // b, db, d2b, two FP32 scalars
    const int LD = wla_ld(P);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = NA + 6 + (nA > 0 ? 6 * nA * nA : 4 * P * LD) + P;
    double* sums = fsh + warp * per;
    double* ss = sums + NA;
    double* B = ss + 6;
    double* Bi = B + P * LD;
    double* D = Bi + P * LD;
    double* M = D + P * LD;
    int* perm = reinterpret_cast<int*>(M + P * LD);
    const int slot = blockIdx.x * (blockDim.x >> 5) + warp;
    if (slot >= *n_act) return;
    const int g = act[slot];
    reduce_partials(partW, nseg, slot_stride, slot, NA, NA, sums, lane);
    reduce_partials(partS, nseg, slot_stride, slot, 4, 4, ss + 2, lane);
    __syncwarp();
    // Cox-Reid terms (warp-parallel): B = b + 1e-6 I (inv_sympd), M = B^-1 db
    double cr_s = 0.0, cr_d = 0.0, cr_d2 = 0.0;
    if (cox_reid && nA > 0) {
        double ddetb = 0.0, trmm = 0.0, trbd2 = 0.0;
        mle_cr_structured(sums, P, NE, nA, colA, colD, B, ddetb, trmm, trbd2);
        const double d2detb = ddetb * ddetb - trmm + trbd2;
        cr_s = -0.5 * ddetb * kCrFactor;
        cr_d = (0.5 * ddetb * ddetb - 0.5 * d2detb) * kCrFactor;
        cr_d2 = -0.5 * ddetb * kCrFactor;
    } else if (cox_reid) {
        warp_unpack_sym(P, sums, 1.0, 1e-6, B, LD);
        warp_lu(B, LD, P, perm);
        warp_lu_inverse(B, LD, P, perm, Bi, LD);
        warp_unpack_sym(P, sums + NE, 1.0, 0.0, D, LD);  // db
        warp_matmul(P, Bi, D, M, LD);
        const double ddetb = warp_sum(lane < P ? M[lane * LD + lane] : 0.0);
        const double trmm = warp_trace_prod(P, M, M, LD);
        warp_unpack_sym(P, sums + 2 * NE, 1.0, 0.0, D, LD);  // d2b
        const double trbd2 = warp_trace_prod(P, Bi, D, LD);
        const double d2detb = ddetb * ddetb - trmm + trbd2;
        cr_s = -0.5 * ddetb * kCrFactor;
        cr_d = (0.5 * ddetb * ddetb - 0.5 * d2detb) * kCrFactor;
        cr_d2 = -0.5 * ddetb * kCrFactor;
    }
    if (lane != 0) return;
    // ss[0..5]: sum ll_term, sum mu x/(1+x)^2, sum y theta/(1+x), sum y/(1+x)^2,
    // digamma sum, trigamma sum
    ss[0] = sums[3 * NE + 0];
    ss[1] = sums[3 * NE + 1];

    const double x = st.x[g];
    const double theta = exp(x), a = 1.0 / theta;
    const double* gs = stats + (int64_t)g * 6;
    const double sum_y = gs[2], sum_prod_y = gs[3], max_y = gs[4];
    // score (src/overdispersion.cpp:139-177)
    const double corr = a > 1e5 ? sum_prod_y / (2.0 * a) : 0.0;
    double dig;
    if (max_y * 1e6 < a) {
        dig = sum_y - corr;
    } else {
        dig = ss[4] * a;
        if (dig > sum_y - corr) dig = sum_y - corr;
    }
    const double score = a * (ss[0] + ss[2]) - dig + cr_s * theta;
    // derivative (src/overdispersion.cpp:218-241)
    const double l1 = ss[0] + ss[2], l2 = ss[1] + ss[3];
    const double digd = ss[4], trig = a * a * ss[5];
    const double ll = -2.0 * a * (l1 - digd) + (l2 + trig);
    const double deriv = ll + cr_d * theta * theta + (l1 - digd) * a + cr_d2 * theta;

    int phase = st.phase[g];
    bool done = false;
    double xn = x;
    if (phase == 0) {
        if (score < 0.0) {
            st.theta[g] = 0.0;
            st.phase[g] = 2;
            if (st.keep) st.keep[g] = 0;
            return;
        }
        const double mean = gs[0], var = gs[1];
        double start = (var - mean) / (mean * mean);
        if (isnan(start) || start <= 0.0) start = 0.5;
        // Newton converges to the same root from any start inside the
        // bracket; the method-of-moments estimate at the fitted beta is
        // usually within a few steps of it (the reference's start ignores
        // size factors and covariates)
        if (st.start_hint) {
            double h = st.start_hint[g];
            if (h > 1e-8 && h < 1e16) start = h;
        }
        double lo = log(1e-8), hi = log(1e16);
        xn = log(start);
        if (xn < lo) xn = lo;
        if (xn > hi) xn = hi;
        st.lo[g] = lo;
        st.hi[g] = hi;
        st.dx[g] = hi - lo;
        st.dxold[g] = hi - lo;
        st.phase[g] = 1;
    } else {
        double lo = st.lo[g], hi = st.hi[g];
        double dx = st.dx[g], dxold = st.dxold[g];
        int it = st.it[g];
        if (score == 0.0) {
            done = true;
        } else {
            if (score > 0.0) lo = x; else hi = x;
            // Newton inside the bracket; bisect when the step leaves it or
            // fails to halve the step before last
            double cand = deriv < 0.0 ? x - score / deriv : NAN;
            if (!(cand > lo && cand < hi) || fabs(cand - x) > 0.5 * fabs(dxold)) {
                dxold = dx;
                dx = 0.5 * (hi - lo);
                cand = lo + dx;
            } else {
                dxold = dx;
                dx = fabs(cand - x);
            }
            xn = cand;
            ++it;
            // stop once a step is below 1e-7 in log theta: after a Newton
            // step that size the error is ~1e-14, after a bisection step
            // theta is within 1e-7 relative (the parity bar is 1e-4)
            if (dx < 1e-7 || hi - lo < 1e-7 || it >= max_iter) done = true;
        }
        st.lo[g] = lo;
        st.hi[g] = hi;
        st.dx[g] = dx;
        st.dxold[g] = dxold;
        st.it[g] = it;
    }
    st.x[g] = xn;
    if (done) {
        st.theta[g] = exp(xn);
        st.phase[g] = 2;
    } else if (!st.keep) {
        act_next[atomicAdd(n_next, 1)] = g;
    }
    if (st.keep) st.keep[g] = done ? 0 : 1;
}
cudaError_t launch_mle_finalize(const void* partW, bool wide, const double* partS, int nseg,
                                int slot_stride, int P, const double* stats, int64_t n,
                                const int32_t* act, const int32_t* n_act, int max_slots,
                                int32_t* act_next, int32_t* n_next, MleState s, int max_iter,
                                int cox_reid, volatile int32_t* mirror, cudaStream_t st, int nA,
                                const int32_t* colA, const int32_t* colD) {
    (void)mirror;
    if (max_slots <= 0) return cudaSuccess;
    const int NA = 3 * (P * (P + 1) / 2) + 2;
    const size_t per = (size_t)(NA + 6 + (nA > 0 ? 6 * nA * nA : 4 * P * wla_ld(P)) + P) * sizeof(double);
    const int w = fin_warps(per);
    const size_t smem = per * w;
    auto go = [&](auto* pw) -> cudaError_t {
        using TW = std::remove_const_t<std::remove_pointer_t<decltype(pw)>>;
        if (smem > 48 * 1024) {
            cudaError_t e = raise_dyn_smem(mle_finalize_kernel<TW>, smem);
            if (e != cudaSuccess) return e;
        }
        mle_finalize_kernel<TW><<<nblk(max_slots, w), 32 * w, smem, st>>>(
            pw, partS, nseg, slot_stride, P, stats, n, act, n_act, act_next, n_next, s, max_iter,
            cox_reid, nA, colA, colD);
        return cudaGetLastError();
    };
    return wide ? go(static_cast<const double*>(partW)) : go(static_cast<const float*>(partW));
}

// ------------------------------------------------------------------
// bread = (X' W X)^-1 (src/variance.cpp:22-47); clustered meat
// (src/variance.cpp:186-228): per-cluster score sums from the partials of
// cluster-aligned segments, meat = adj/n sum_b s_b s_b', adj = C/(C-1)
// (1 when C = 1); sandwich = bread meat bread n (R/main.R:482-492).
// ------------------------------------------------------------------
__global__ void sandwich_finalize_kernel(const double* partW, int nseg, int slot_stride, int P,
                                         const int32_t* seg_cluster, int n_clusters, int64_t n,
                                         const int32_t* act, const int32_t* n_act, double* bread,
                                         double* sandwich, double* meat_out) {
    extern __shared__ double fsh[];
    const int NE = P * (P + 1) / 2, NA = NE + P, LD = wla_ld(P);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = NA + 4 * P * LD + 2 * P;
    double* sums = fsh + warp * per;
    double* H = sums + NA;
    double* Bi = H + P * LD;
    double* Mt = Bi + P * LD;
    double* T = Mt + P * LD;
    double* cur = T + P * LD;
    int* perm = reinterpret_cast<int*>(cur + P);
    const int slot = blockIdx.x * (blockDim.x >> 5) + warp;
    if (slot >= *n_act) return;
    const int g = act[slot];
    reduce_partials(partW, nseg, slot_stride, slot, NA, NE, sums, lane);  // H part only
    for (int i = lane; i < P * LD; i += 32) Mt[i] = 0.0;
    __syncwarp();
    if (n_clusters > 0) {
        // lane i holds component i of the running cluster sum
        double acc = 0.0;
        for (int seg = 0; seg < nseg; ++seg) {
            if (lane < P) acc += partW[((int64_t)seg * slot_stride + slot) * NA + NE + lane];
            bool last = (seg == nseg - 1) || (seg_cluster[seg + 1] != seg_cluster[seg]);
            if (last) {
                if (lane < P) cur[lane] = acc;
                __syncwarp();
                for (int i = lane; i < P * P; i += 32) {
                    const int r = i / P, c = i - r * P;
                    Mt[r * LD + c] += cur[r] * cur[c];
                }
                __syncwarp();
                acc = 0.0;
            }
        }
    }
    warp_unpack_sym(P, sums, 1.0, 0.0, H, LD);
    warp_lu(H, LD, P, perm);
    warp_lu_inverse(H, LD, P, perm, Bi, LD);
    double* bo = bread + (int64_t)g * P * P;  // column-major
    for (int q = lane; q < P * P; q += 32) {
        const int c = q / P, r = q - c * P;
        bo[q] = Bi[r * LD + c];
    }
    if (n_clusters > 0) {
        const double adj = n_clusters > 1 ? (double)n_clusters / (n_clusters - 1.0) : 1.0;
        for (int i = lane; i < P * LD; i += 32) Mt[i] *= adj / (double)n;
        __syncwarp();
        if (meat_out)
            for (int q = lane; q < P * P; q += 32) {
                const int c = q / P, r = q - c * P;
                meat_out[(int64_t)g * P * P + q] = Mt[r * LD + c];
            }
        if (sandwich) {
            warp_matmul(P, Bi, Mt, T, LD);  // T = Bi Mt
            warp_matmul(P, T, Bi, H, LD);   // H = T Bi (H is free after the inverse)
            double* so = sandwich + (int64_t)g * P * P;
            for (int q = lane; q < P * P; q += 32) {
                const int c = q / P, r = q - c * P;
                so[q] = H[r * LD + c] * (double)n;
            }
        }
    }
}
cudaError_t launch_sandwich_finalize(const double* partW, int nseg, int slot_stride, int P,
                                     const int32_t* seg_cluster, int n_clusters, int64_t n,
                                     const int32_t* act, const int32_t* n_act, int max_slots,
                                     double* bread, double* sandwich, double* meat,
                                     cudaStream_t st) {
    if (max_slots <= 0) return cudaSuccess;
    const int NA = P * (P + 1) / 2 + P;
    const size_t per = (size_t)(NA + 4 * P * wla_ld(P) + 2 * P) * sizeof(double);
    const int w = fin_warps(per);
    const size_t smem = per * w;
    if (smem > 48 * 1024) {
        cudaError_t e = raise_dyn_smem(sandwich_finalize_kernel, smem);
        if (e != cudaSuccess) return e;
    }
    sandwich_finalize_kernel<<<nblk(max_slots, w), 32 * w, smem, st>>>(
        partW, nseg, slot_stride, P, seg_cluster, n_clusters, n, act, n_act, bread, sandwich, meat);
    return cudaGetLastError();
}

}  // namespace devil
