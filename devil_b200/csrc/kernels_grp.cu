// Design-group engine.
//
// Designs built from an intercept, a condition and one-hot cell-type /
// batch columns have few distinct rows: a cell enters every pass only
// through its design row x_u and its offset o_i (log size factor).  With
// the cells grouped by design row (and by cluster for the sandwich), one
// pass computes per (gene, group)
//   * the terms of zero counts summed over all cells of the group,
//       sum_i f(exp(a_u + o_i)),  a_u = x_u . beta,
//     as a Gauss rule for the group's offsets: bins of width 2 in the
//     offset, each with its cells as nodes (at most 10 cells) or a 10-point
//     Gauss rule; checked against exact sums before use;
//   * the corrections of the nonzero counts from a CSR copy in which every
//     gene's entries are ordered by "slice": the cells are renumbered so
//     that each (design row, cluster) group is a contiguous range, cut into
//     slices of at most kSliceCells cells; an entry is 4 bytes (the cell's
//     16-bit index within its slice and the 16-bit count), and exp(offset)
//     is stored in the new cell order, so one slice's values fit in shared
//     memory;
// and assembles the p x p terms from the group sums.  A pass then reads
// every nonzero once and costs O(nnz + groups x nodes) per gene, plus the
// assembly over the (group, output) pairs whose design entries are nonzero
// (for one-hot rows: a handful per group), instead of O(cells x p^2).  Partial sums land in the layout of the other engines
// (FP64, one segment, or one per cluster for the sandwich), so the
// finalize kernels are shared.
#include <cub/cub.cuh>

#include <type_traits>

#include "internal.h"

namespace devil {

static inline unsigned nblk(int64_t m, int t) { return (unsigned)((m + t - 1) / t); }

// ---------------------------------------------------------------------
// grouping of the design rows
// ---------------------------------------------------------------------
// 64-bit hash of the bit patterns of a row (column-major X): equal rows
// hash equally; equal hashes are confirmed bit for bit afterwards
__global__ void row_hash_kernel(const double* X, int64_t n, int P, uint64_t* h, int32_t* idx) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t v = 0x9E3779B97F4A7C15ull;
    for (int j = 0; j < P; ++j) {
        uint64_t b = (uint64_t)__double_as_longlong(X[i + (int64_t)j * n]);
        v ^= b + 0x9E3779B97F4A7C15ull + (v << 6) + (v >> 2);
        v *= 0xBF58476D1CE4E5B9ull;
        v ^= v >> 31;
    }
    h[i] = v;
    idx[i] = (int32_t)i;
}

// run heads of the sorted hashes; rows with equal hashes must be equal
__global__ void group_heads_kernel(const double* X, int64_t n, int P, const uint64_t* hs,
                                   const int32_t* is, int32_t* flag, int32_t* bad) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int head = (i == 0) || hs[i] != hs[i - 1];
    flag[i] = head;
    if (!head) {
        const int64_t a = is[i], b = is[i - 1];
        for (int j = 0; j < P; ++j)
            if (__double_as_longlong(X[a + (int64_t)j * n]) != __double_as_longlong(X[b + (int64_t)j * n]))
                *bad = 1;  // hash collision: the caller falls back to the per-cell engines
    }
}

// group of every cell (0-based run number) and the first cell of each group
__global__ void group_assign_kernel(const int32_t* is, const int32_t* incl, const int32_t* flag,
                                    int64_t n, int32_t* ucell, int32_t* head) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int u = incl[i] - 1;
    ucell[is[i]] = u;
    if (flag[i]) head[u] = is[i];
}

__global__ void group_rows_kernel(const double* X, int64_t n, int P, const int32_t* head, int U,
                                  double* xg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= U * P) return;
    const int u = i / P, j = i - u * P;
    xg[i] = X[head[u] + (int64_t)j * n];
}

// fine key u * C + cluster; clusters are contiguous blocks with 1-based
// exclusive ends (the cluster_ends of the fit)
__global__ void fine_keys_kernel(const int32_t* ucell, const int32_t* ends, int C, int64_t n,
                                 int32_t* fkey, int32_t* cell) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = 0, hi = C - 1;  // first cluster whose end exceeds i
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (ends[mid] > i) hi = mid; else lo = mid + 1;
    }
    fkey[i] = ucell[i] * C + (C > 1 ? lo : 0);
    cell[i] = (int32_t)i;
}

// gstart[k] = first position of key k in the sorted keys (k = 0..K)
__global__ void group_starts_kernel(const int32_t* ks, int64_t n, int K, int64_t* gstart) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > K) return;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (ks[mid] < k) lo = mid + 1; else hi = mid;
    }
    gstart[k] = lo;
}

__global__ void gather_keys_kernel(const int32_t* keys, const int32_t* cells, int64_t n,
                                   int32_t* out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = keys[cells[i]];
}

__global__ void exp_kernel(const double* x, int64_t n, double* y) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] = exp(x[i]);
}

// ---------------------------------------------------------------------
// Gauss rules of the groups' offset distributions
// ---------------------------------------------------------------------
constexpr int kRuleNT = 256;

// block-wide sum; every thread gets the same value (same association)
DEV double block_sum(double v, double* red) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double r = l < nw ? red[l] : 0.0;
    return warp_sum(r);
}
DEV double block_min(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double r = l < nw ? red[l] : INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmin(r, __shfl_xor_sync(0xffffffffu, r, o));
    return r;
}

// number of eigenvalues below x of the Jacobi matrix with diagonal al[0..m)
// and squared off-diagonal be[1..m) (Sturm sequence of the LDL^T pivots)
DEV int jacobi_count_below(const double* al, const double* be, int m, double x) {
    int c = 0;
    double d = 1.0;
    for (int i = 0; i < m; ++i) {
        d = (al[i] - x) - (i ? be[i] / d : 0.0);
        if (d == 0.0) d = -1e-300;
        c += d < 0.0;
    }
    return c;
}

// Gauss rule of one bin of sorted offsets s[perm[c0..c1)] (more than
// kBinNodes cells, a spread above 1e-13) with m <= kBinNodes nodes, written
// to os/ow.  In t = (s - c)/h the monic orthogonal polynomials of the bin's
// measure are run over its cells (discretised Stieltjes procedure, stable
// at this degree), the nodes are the eigenvalues of the Jacobi matrix
// (bisection on Sturm counts), the weights the Christoffel numbers scaled
// to the bin's cell count.  The recurrence stops early when pi_{k+1}
// vanishes on the support (at most k+1 distinct offsets: the rule is then
// exact).  Returns m (same value in every thread).
DEV int bin_rule(const int32_t* perm, const double* off, int64_t c0, int64_t c1, double* tt,
                 double* p0, double* p1, double* red, double* al, double* be, double* nk,
                 double* wsum, double* os, double* ow) {
    const int t = threadIdx.x, nt = blockDim.x;
    const double cnt = (double)(c1 - c0);
    const double bmin = off[perm[c0]], bmax = off[perm[c1 - 1]];
    const double c = 0.5 * (bmax + bmin), h = 0.5 * (bmax - bmin);
    double st = 0.0;
    for (int64_t i = c0 + t; i < c1; i += nt) {
        const double x = (off[perm[i]] - c) / h;
        tt[i] = x;
        p0[i] = 1.0;
        p1[i] = 0.0;
        st += x;
    }
    st = block_sum(st, red);
    if (t == 0) {
        al[0] = st / cnt;
        be[0] = 0.0;
        nk[0] = cnt;
    }
    __syncthreads();
    int m = kBinNodes;
    for (int k = 0; k + 1 < kBinNodes; ++k) {
        const double a = al[k], bb = be[k];
        double sN = 0.0, sT = 0.0, sS = 0.0;
        for (int64_t i = c0 + t; i < c1; i += nt) {
            const double x = tt[i], pk = p0[i], pm = p1[i];
            const double pn = (x - a) * pk - bb * pm;
            const double sc = fabs(x - a) * fabs(pk) + bb * fabs(pm);
            p1[i] = pk;
            p0[i] = pn;
            sN += pn * pn;
            sT += x * pn * pn;
            sS += sc * sc;
        }
        sN = block_sum(sN, red);
        sT = block_sum(sT, red);
        sS = block_sum(sS, red);
        if (!(sN > 1e-26 * sS)) {  // pi_{k+1} is rounding noise on the support
            m = k + 1;
            break;
        }
        if (t == 0) {
            al[k + 1] = sT / sN;
            be[k + 1] = sN / nk[k];
            nk[k + 1] = sN;
        }
        __syncthreads();
    }
    __syncthreads();
    double xj = 0.0, wj = 0.0;
    if (t < m) {
        // eigenvalue t (ascending); all lie in [-1, 1]
        double lo = -1.0 - 1e-9, hi = 1.0 + 1e-9;
        for (int it = 0; it < 200; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (mid <= lo || mid >= hi) break;
            if (jacobi_count_below(al, be, m, mid) > t) hi = mid; else lo = mid;
        }
        xj = 0.5 * (lo + hi);
        // Christoffel number: 1 / sum_k pi_k(x)^2 / (N_k / N_0)
        double pm = 0.0, pk = 1.0, q = 1.0;
        for (int k = 0; k + 1 < m; ++k) {
            const double pn = (xj - al[k]) * pk - be[k] * pm;
            pm = pk;
            pk = pn;
            q += pn * pn * (nk[0] / nk[k + 1]);
        }
        wj = cnt / q;
        wsum[t] = wj;
    }
    __syncthreads();
    if (t < 32) {
        double v = t < m ? wsum[t] : 0.0;
        v = warp_sum(v);
        if (t < m) {
            os[t] = c + h * xj;
            ow[t] = wj * (cnt / v);  // weights sum to the bin's cell count
        }
    }
    __syncthreads();
    return m;
}

// first position in [lo, hi) of the sorted offsets s[perm[.]] with s >= v
DEV int64_t lower_bound_off(const int32_t* perm, const double* off, int64_t lo, int64_t hi, double v) {
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (off[perm[mid]] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Block per rule.  Rule b < U: coarse group b, cells permC[gsC[b]..gsC[b+1])
// sorted by offset; rule U + k: fine group k (row, cluster), cells
// permF[gsF[k]..gsF[k+1]).  The group's offsets are cut into bins of width
// kBinWidth; a bin of at most kBinNodes cells contributes its cells as
// nodes (weight 1), a bin of one offset (to 1e-13) one node at its mean,
// any other bin a kBinNodes-point Gauss rule (bin_rule).  With bins of
// width 2 the dense terms of the passes, analytic within pi of the real
// s axis, are integrated to ~1e-15.  The rule is checked on
// sum_i 1/(1 + exp(s_i - z)) for z at both ends and the middle of the
// group's range; rerr[b] is the worst relative error and a value above
// 1e-11 (or more than kMaxBins bins) sets *bad.
__global__ void __launch_bounds__(kRuleNT) group_rules_kernel(
    const int32_t* permC, const int64_t* gsC, const int32_t* permF, const int64_t* gsF, int U,
    const double* off, int64_t n, double* scr, double* rs, double* rw, int32_t* rm, double* rerr,
    int32_t* bad) {
    __shared__ double red[32];
    __shared__ double al[kBinNodes + 1], be[kBinNodes + 1], nk[kBinNodes + 1];
    __shared__ double wsum[32];
    __shared__ int64_t rng[2];
    const int b = blockIdx.x, t = threadIdx.x, nt = blockDim.x;
    const bool coarse = b < U;
    const int32_t* perm = coarse ? permC : permF;
    const int64_t b0 = coarse ? gsC[b] : gsF[b - U];
    const int64_t b1 = coarse ? gsC[b + 1] : gsF[b - U + 1];
    const int64_t base = coarse ? 0 : n;  // scratch of coarse and fine rules
    double* tt = scr + base;
    double* p0 = scr + 2 * n + base;
    double* p1 = scr + 4 * n + base;
    double* os = rs + (int64_t)b * kRuleCap;
    double* ow = rw + (int64_t)b * kRuleCap;
    if (b1 <= b0) {
        if (t == 0) {
            rm[b] = 0;
            rerr[b] = 0.0;
        }
        return;
    }
    const double smin = off[perm[b0]], smax = off[perm[b1 - 1]];
    const double span = (smax - smin) / kBinWidth;
    if (!(span < (double)kMaxBins)) {  // offsets too spread (or not finite)
        if (t == 0) {
            rm[b] = 0;
            rerr[b] = INFINITY;
            atomicExch(bad, 1);
        }
        return;
    }
    const int nb = (int)span + 1;
    int nodes = 0;
    for (int j = 0; j < nb; ++j) {
        if (t == 0) {
            rng[0] = j == 0 ? b0 : lower_bound_off(perm, off, b0, b1, smin + j * kBinWidth);
            rng[1] = j == nb - 1 ? b1 : lower_bound_off(perm, off, b0, b1, smin + (j + 1) * kBinWidth);
        }
        __syncthreads();
        const int64_t c0 = rng[0], c1 = rng[1];
        __syncthreads();
        const int64_t cnt = c1 - c0;
        if (cnt <= 0) continue;
        if (cnt <= kBinNodes) {
            if (t < cnt) {
                os[nodes + t] = off[perm[c0 + t]];
                ow[nodes + t] = 1.0;
            }
            nodes += (int)cnt;
            continue;
        }
        const double bmin = off[perm[c0]], bmax = off[perm[c1 - 1]];
        if (!(bmax - bmin > 1e-13 * fmax(1.0, fabs(bmax)))) {
            double sm = 0.0;
            for (int64_t i = c0 + t; i < c1; i += nt) sm += off[perm[i]];
            sm = block_sum(sm, red);
            if (t == 0) {
                os[nodes] = sm / (double)cnt;
                ow[nodes] = (double)cnt;
            }
            nodes += 1;
            continue;
        }
        nodes += bin_rule(perm, off, c0, c1, tt, p0, p1, red, al, be, nk, wsum, os + nodes,
                          ow + nodes);
    }
    if (t == 0) rm[b] = nodes;
    __syncthreads();
    // check the rule against exact sums of three logistic test functions
    const double mid = 0.5 * (smin + smax);
    double worst = 0.0;
    for (int z = 0; z < 3; ++z) {
        const double zc = z == 0 ? smin : (z == 1 ? mid : smax);
        double ex = 0.0, ap = 0.0;
        for (int64_t i = b0 + t; i < b1; i += nt) ex += 1.0 / (1.0 + exp(off[perm[i]] - zc));
        for (int i = t; i < nodes; i += nt) ap += ow[i] / (1.0 + exp(os[i] - zc));
        ex = block_sum(ex, red);
        ap = block_sum(ap, red);
        const double e = fabs(ap - ex) / ex;
        worst = e > worst ? e : (e == e ? worst : e);  // NaN sticks
    }
    if (t == 0) {
        rerr[b] = worst;
        if (!(worst <= 1e-11)) atomicExch(bad, 1);
    }
}

// ---------------------------------------------------------------------
// CSR copy ordered by key within each gene (stable), with per-gene key
// offsets gptr[g][k] (absolute; gptr[g][K] = row end).  Each row is cut
// into segments of S entries so that long rows spread over many warps:
//   1. count the keys of every segment (warp per segment),
//   2. per gene, turn the counts into the first output position of every
//      (segment, key) in key-major, segment-minor order (block per gene),
//   3. scatter every segment's entries from those cursors, in order
//      (warp per segment; ranks among equal keys from __match_any_sync).
// ---------------------------------------------------------------------
__global__ void seg_count_kernel(const int64_t* rowptr, int64_t G, int S, int64_t* nseg) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= G) return;
    const int64_t len = rowptr[g + 1] - rowptr[g];
    nseg[g] = (len + S - 1) / S;
}

// gene of global segment s: last g with segbase[g] <= s (segbase has G+1 entries)
DEV int64_t seg_gene(const int64_t* segbase, int64_t G, int64_t s) {
    int64_t lo = 0, hi = G;  // invariant: segbase[lo] <= s < segbase[hi]
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (segbase[mid] <= s) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void seg_hist_kernel(const int64_t* rowptr, const int32_t* col, int64_t G,
                                const int64_t* segbase, int S, const int32_t* ckey, int K,
                                int32_t* hist) {
    extern __shared__ int32_t cnt_all[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t s = (int64_t)blockIdx.x * (blockDim.x >> 5) + w;
    if (s >= segbase[G]) return;
    int32_t* cnt = cnt_all + (int64_t)w * K;
    for (int k = lane; k < K; k += 32) cnt[k] = 0;
    __syncwarp();
    const int64_t g = seg_gene(segbase, G, s);
    const int64_t r0 = rowptr[g] + (s - segbase[g]) * S;
    const int64_t r1 = min(r0 + S, rowptr[g + 1]);
    constexpr int U = 4;  // loads in flight per lane
    for (int64_t base = r0 + lane; base < r1; base += 32 * U) {
        int c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) c[u] = base + 32 * u < r1 ? __ldg(col + base + 32 * u) : -1;
        int k[U];
#pragma unroll
        for (int u = 0; u < U; ++u) k[u] = c[u] >= 0 ? __ldg(ckey + c[u]) : -1;
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k[u] >= 0) atomicAdd(&cnt[k[u]], 1);
    }
    __syncwarp();
    int32_t* h = hist + s * K;
    for (int k = lane; k < K; k += 32) h[k] = cnt[k];
}

constexpr int kOffNT = 256;
__global__ void __launch_bounds__(kOffNT) seg_offsets_kernel(const int64_t* rowptr, int64_t G,
                                                             const int64_t* segbase, int K,
                                                             int32_t* hist, int64_t* gptr) {
    using Scan = cub::BlockScan<int64_t, kOffNT>;
    __shared__ typename Scan::TempStorage tmp;
    const int64_t g = blockIdx.x;
    const int t = threadIdx.x;
    const int64_t s0 = segbase[g], s1 = segbase[g + 1];
    const int64_t r0 = rowptr[g];
    // thread t owns keys [t*per, (t+1)*per)
    const int per = (K + kOffNT - 1) / kOffNT;
    const int k0 = min(K, t * per), k1 = min(K, k0 + per);
    int64_t local = 0;
    for (int k = k0; k < k1; ++k)
        for (int64_t s = s0; s < s1; ++s) local += hist[s * K + k];
    int64_t excl;
    Scan(tmp).ExclusiveSum(local, excl);
    int64_t run = excl;  // offset of key k0 relative to the row start
    for (int k = k0; k < k1; ++k) {
        gptr[g * (K + 1) + k] = r0 + run;
        for (int64_t s = s0; s < s1; ++s) {
            const int32_t c = hist[s * K + k];
            hist[s * K + k] = (int32_t)run;
            run += c;
        }
    }
    if (t == 0) gptr[g * (K + 1) + K] = rowptr[g + 1];
}

template <class VT>
__global__ void seg_scatter_kernel(const int64_t* rowptr, const int32_t* col, const VT* val,
                                   int64_t G, const int64_t* segbase, int S, const int32_t* cloc, int K,
                                   const int32_t* hist, typename GrpEnt<VT>::T* gent) {
    extern __shared__ int32_t cur_all[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t s = (int64_t)blockIdx.x * (blockDim.x >> 5) + w;
    if (s >= segbase[G]) return;
    int32_t* cur = cur_all + (int64_t)w * K;
    for (int k = lane; k < K; k += 32) cur[k] = hist[s * K + k];
    __syncwarp();
    const int64_t g = seg_gene(segbase, G, s);
    const int64_t rs = rowptr[g];
    const int64_t r0 = rs + (s - segbase[g]) * S;
    const int64_t r1 = min(r0 + S, rowptr[g + 1]);
    const unsigned lt = (1u << lane) - 1u;
    // U rounds of 32 entries: every load and key lookup of the rounds is
    // issued first, then the rounds are placed in order (the same positions
    // as one round at a time)
    constexpr int U = 8;
    for (int64_t base = r0; base < r1; base += 32 * U) {
        int c[U], k[U], lc[U];
        VT v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t e = base + 32 * u + lane;
            c[u] = e < r1 ? __ldg(col + e) : -1;
            v[u] = e < r1 ? val[e] : VT(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            // (cloc packs the slice and the index in it)
            const uint32_t kl = c[u] >= 0 ? (uint32_t)__ldg(cloc + c[u]) : 0xffffffffu;
            k[u] = c[u] >= 0 ? (int)(kl >> 16) : -1;
            lc[u] = (int)(kl & 0xffffu);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool valid = c[u] >= 0;
            const unsigned peers = __match_any_sync(0xffffffffu, k[u]);
            const int rank = __popc(peers & lt);
            const int pos = valid ? cur[k[u]] + rank : 0;
            __syncwarp();
            if (valid) {
                gent[rs + pos] = GrpEnt<VT>::pack(lc[u], v[u]);
                if (lane == __ffs(peers) - 1) cur[k[u]] += __popc(peers);
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------
// the pass
// ---------------------------------------------------------------------
// accumulator for one lane: every term is scaled by q (the node weight for
// zero-count terms, 1 for the nonzeros)
template <int NWV, int NS>
struct GrpAcc {
    double w[NWV > 0 ? NWV : 1];
    double s[NS > 0 ? NS : 1];
    double q;
    DEV void zero() {
#pragma unroll
        for (int i = 0; i < NWV; ++i) w[i] = 0.0;
#pragma unroll
        for (int i = 0; i < NS; ++i) s[i] = 0.0;
        q = 1.0;
    }
    template <int W>
    DEV void outer(double v) { w[W] += q * v; }
    template <int V, int NW>
    DEV void vec(double v) { w[NW + V] += q * v; }
    template <int K>
    DEV void scal(double v) { s[K] += q * v; }
    template <int K, int NW, int NV>
    DEV void fscal(double v) { w[NW + NV + K] += q * v; }
};

constexpr int kGrpUnr = 8;          // entries per lane per batch of the nonzero loop
constexpr int kGrpChunk = 2048;     // nonzeros per work unit (at least)
constexpr int kGrpUnitsMax = 128;   // chunks beyond one per slice, per gene

// x_u . beta over the nonzero entries of design row u (warp-wide sum)
DEV double row_dot(const GrpGeom& geo, int u, const double* bet, int lane) {
    double a = 0.0;
    const int r1 = __ldg(geo.rptr + u + 1);
    for (int e = __ldg(geo.rptr + u) + lane; e < r1; e += 32) a += __ldg(geo.rval + e) * bet[__ldg(geo.rcol + e)];
    return warp_sum(a);
}

// The design-group pass, block per gene (MOM, MLE, bread/meat; the IRLS
// pass runs slice-major, grp_irls_slices_kernel).  Work units of a gene:
// one "rule unit" per group q (the zero-count terms of the group's cells
// from its Gauss rule), then the gene's nonzeros slice by slice in chunks of
// at least kGrpChunk entries.  Warps take units round robin; the group sums
// are then formed in unit order (deterministic) and assembled.
template <class Pass, class VT>
__global__ void __launch_bounds__(256) grp_pass_kernel(GrpGeom geo, typename Pass::Params prm) {
    using Ent = GrpEnt<VT>;
    using ET = typename Ent::T;
    constexpr int NW = Pass::NW, NV = Pass::NV, NF = Pass::NF;
    constexpr int NWV = NW + NV + NF, NS = Pass::NS, NQ = NWV + NS;
    if (geo.reset_next && blockIdx.x == 0 && threadIdx.x == 0) *geo.reset_next = 0;
    const int slot = blockIdx.x;
    if (slot >= *geo.n_act) return;
    const int g = __ldg(geo.act + slot);
    const int P = geo.P, U = geo.U, C = geo.C, S = geo.S;
    const int NGq = geo.fine ? U * C : U;
    extern __shared__ double gsm[];
    double* bet = gsm;                                   // [P]
    double* gs = bet + P;                                // [NGq][NQ] group sums
    double* up = gs + NGq * NQ;                          // [NGq + S + kGrpUnitsMax][NQ] unit sums
    int* sstart = reinterpret_cast<int*>(up + (NGq + S + kGrpUnitsMax) * NQ);  // [S + 1]
    const int t = threadIdx.x, nt = blockDim.x;
    for (int i = t; i < P; i += nt) bet[i] = __ldg(prm.beta_d + (int64_t)g * P + i);
    typename Pass::Gene gpar = Pass::load(prm, g);
    if constexpr (Pass::TABLES) {
        __shared__ double psitab[2 * kPsiTab];
        __shared__ double psiscr[kPsiTab];
        __shared__ double psia[1];
        if (t == 0) psia[0] = gpar.a;
        __syncthreads();
        build_psi_tables(1, psia, psitab, psiscr);
        gpar.tab.d1 = psitab;
        gpar.tab.d2 = psitab + kPsiTab;
        gpar.tab.pa = digamma_d(gpar.a);
        gpar.tab.ta = trigamma_d(gpar.a);
    }
    const int warp = t >> 5, lane = t & 31, nw = nt >> 5;
    const ET* __restrict__ gent = static_cast<const ET*>(geo.gent);
    const int64_t* gp = geo.gptr + (int64_t)g * (S + 1);
    // chunk size grows with the gene's nonzeros so that there are at most
    // S + kGrpUnitsMax nonzero units
    const int64_t CH = max((int64_t)kGrpChunk, (gp[S] - gp[0] + kGrpUnitsMax - 1) / kGrpUnitsMax);
    if (warp == 0) {
        int run = 0;
        for (int base = 0; base < S; base += 32) {
            const int sl = base + lane;
            int c = 0;
            if (sl < S) {
                const int64_t len = __ldg(gp + sl + 1) - __ldg(gp + sl);
                c = (int)((len + CH - 1) / CH);
            }
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (sl < S) sstart[sl] = run + incl - c;
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) sstart[S] = run;
    }
    __syncthreads();
    const int nunits = NGq + sstart[S];
    for (int un = warp; un < nunits; un += nw) {
        GrpAcc<NWV, NS> acc;
        acc.zero();
        if (un < NGq) {
            // zero-count terms of every cell of group q: its rule
            const int q = un;
            const int u = geo.fine ? q / C : q;
            const int ri = (geo.fine && C > 1) ? U + q : u;  // C == 1: fine == coarse
            const double A = exp(row_dot(geo, u, bet, lane));
            const int m = __ldg(geo.rm + ri);
            for (int j = lane; j < m; j += 32) {
                acc.q = __ldg(geo.rw + (int64_t)ri * kRuleCap + j);
                const double mu = A * __ldg(geo.res + (int64_t)ri * kRuleCap + j);
                Pass::template dense<double>(gpar, mu, acc);
            }
        } else {
            // a chunk of the nonzeros of slice sl
            const int cu = un - NGq;
            int sl = 0;  // last slice with sstart[sl] <= cu
            {
                int lo = 0, hi = S;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (sstart[mid] <= cu) lo = mid; else hi = mid;
                }
                sl = lo;
            }
            const int jc = cu - sstart[sl];
            const int u = __ldg(geo.sl_key + sl) / C;
            const double A = exp(row_dot(geo, u, bet, lane));
            const double* __restrict__ Es = geo.E + __ldg(geo.sl_start + sl);
            const int64_t e0 = __ldg(gp + sl) + jc * CH;
            const int64_t e1 = min(e0 + CH, __ldg(gp + sl + 1));
            // batches of kGrpUnr entries per lane, software-pipelined: the
            // next batch's entries are in flight while this batch gathers
            // exp(offset) and accumulates
            int64_t e = e0 + lane;
            constexpr int U8 = kGrpUnr;
            if (e + 32 * (U8 - 1) < e1) {
                ET c[U8];
#pragma unroll
                for (int j = 0; j < U8; ++j) c[j] = gent[e + 32 * j];
                for (;;) {
                    double ev[U8];
#pragma unroll
                    for (int j = 0; j < U8; ++j) ev[j] = __ldg(Es + Ent::loc(c[j]));
                    const int64_t en = e + 32 * U8;
                    const bool more = en + 32 * (U8 - 1) < e1;
                    ET cn[U8];
                    if (more) {
#pragma unroll
                        for (int j = 0; j < U8; ++j) cn[j] = gent[en + 32 * j];
                    }
#pragma unroll
                    for (int j = 0; j < U8; ++j) Pass::template sparse<double>(gpar, A * ev[j], Ent::y(c[j]), acc);
                    e = en;
                    if (!more) break;
#pragma unroll
                    for (int j = 0; j < U8; ++j) c[j] = cn[j];
                }
            }
            for (; e < e1; e += 32) {
                const ET c = gent[e];
                Pass::template sparse<double>(gpar, A * __ldg(Es + Ent::loc(c)), Ent::y(c), acc);
            }
        }
#pragma unroll
        for (int i = 0; i < NWV; ++i) {
            const double v = warp_sum(acc.w[i]);
            if (lane == 0) up[un * NQ + i] = v;
        }
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            const double v = warp_sum(acc.s[i]);
            if (lane == 0) up[un * NQ + NWV + i] = v;
        }
    }
    __syncthreads();
    // group sums in unit order: the rule unit, then the chunks of the
    // group's slices (slices are ordered by key u * C + c)
    for (int i = t; i < NGq * NQ; i += nt) {
        const int q = i / NQ, c = i - q * NQ;
        double v = up[q * NQ + c];
        const int k0 = geo.fine ? q : q * C, k1 = geo.fine ? q + 1 : q * C + C;
        const int s0 = __ldg(geo.kslice + k0), s1 = __ldg(geo.kslice + k1);
        for (int un = sstart[s0]; un < sstart[s1]; ++un) v += up[(NGq + un) * NQ + c];
        gs[i] = v;
    }
    __syncthreads();
    // assemble the partial sums of the pass: one segment, or one per cluster
    const int NE = P * (P + 1) / 2;
    const int NA = NW * NE + NV * P + NF;
    const int nout = geo.fine ? C : 1;
    const int per = NA + NS;
    for (int o = t; o < nout * per; o += nt) {
        const int seg = o / per, a = o - seg * per;
        double s = 0.0;
        if (a < NW * NE) {
            // the groups whose design entries i and j are both nonzero
            const int w = a / NE, qq = a - w * NE;
            for (int e = __ldg(geo.qptr + qq); e < __ldg(geo.qptr + qq + 1); ++e) {
                const int u = __ldg(geo.qu + e);
                const int q = geo.fine ? u * C + seg : u;
                s += gs[q * NQ + w] * __ldg(geo.qv + e);
            }
        } else if (a < NW * NE + NV * P) {
            const int r = a - NW * NE;
            const int v = r / P, i = r - v * P;
            for (int e = __ldg(geo.vptr + i); e < __ldg(geo.vptr + i + 1); ++e) {
                const int u = __ldg(geo.vu + e);
                const int q = geo.fine ? u * C + seg : u;
                s += gs[q * NQ + NW + v] * __ldg(geo.vv + e);
            }
        } else {
            const int f = a - NW * NE - NV * P;  // fscal (a < NA) or an FP64 scalar
            const int col = a < NA ? NW + NV + f : NWV + (a - NA);
            for (int u = 0; u < U; ++u) {
                const int q = geo.fine ? u * C + seg : u;
                s += gs[q * NQ + col];
            }
        }
        if (a < NA)
            geo.partW[((int64_t)seg * geo.slot_stride + slot) * NA + a] = s;
        else
            geo.partS[((int64_t)seg * geo.slot_stride + slot) * NS + (a - NA)] = s;
    }
}

// ---------------------------------------------------------------------
// IRLS and MLE passes, slice-major.  Block (slice s, share of the active
// genes): the slice's exp(offset) values are staged in shared memory once,
// then each warp takes the block's genes in turn: A = exp(x_u . beta)
// (computed per gene and group beforehand), the rule terms of group u when
// s is the group's first slice, and the gene's entries of the slice as
// 16-byte streaming loads (UNR in flight per lane), mu = A E[cell] with E
// from shared memory.  The active genes are listed in decreasing order of
// entries; those with fewer than kLightEntries (MLE: kLightEntriesMle) per
// slice on average (the tail of the list) take eight lanes each, four to a
// warp, so that the
// per-(gene, slice) bookkeeping (hand-out, ranges, sums, stores) is shared
// by four genes.  The per-(gene, slice) sums go to geo.gsum;
// grp_assemble_kernel / the IRLS step form the p x p terms per gene.
// ---------------------------------------------------------------------
constexpr int kSlNT = 1024;  // one block per SM: 32 warps, 64 registers each, the 128 KB slice stage
static_assert(kSliceCells % kSlNT == 0, "a slice is staged in whole rounds of the block");

// 16-byte loads in flight per lane: as many as 64 registers hold without
// spilling (the MLE's accumulators take more registers; beta_0's per-warp
// queue is sized for three)
template <class Pass>
constexpr int sl_unr() { return Pass::TABLES ? 2 : (std::is_same<Pass, PassInitZ>::value ? 3 : 4); }

// beta_0's pass: per warp, a queue of the entries with counts above 1 (one
// round adds at most 32 x 3 x 4 entries to fewer than 32 left over)
constexpr int kInitQ = 416;

template <class Pass>
constexpr size_t sl_smem_bytes() {
    return (size_t)kSliceCells * sizeof(double) + (Pass::TABLES ? (size_t)(kSlNT / 32) * kGrpTab * sizeof(double) : 0) +
           (size_t)2 * kRuleCap * sizeof(double) +
           (std::is_same<Pass, PassInitZ>::value ? (size_t)(kSlNT / 32) * kInitQ * sizeof(uint32_t) : 0);
}

// streaming 16-byte load that does not allocate in L1 (each entry is read
// once per pass)
DEV uint4 ld_stream(const uint4* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// one gene of a slice-major block: its list slot, index, exp(x_u . beta)
// and the range of its entries in the slice
struct SlItem {
    int j, g;
    double A;
    int64_t e0, e1;
};

template <class Pass, class VT>
__global__ void __launch_bounds__(kSlNT, 1) grp_slices_kernel(GrpGeom geo, typename Pass::Params prm,
                                                              int tile) {
    using Ent = GrpEnt<VT>;
    using ET = typename Ent::T;
    using Acc = GrpAcc<Pass::NW + Pass::NV + Pass::NF, Pass::NS>;
    constexpr int NWV = Pass::NW + Pass::NV + Pass::NF, NS = Pass::NS, NQ = NWV + NS;
    constexpr int EPL = sizeof(uint4) / sizeof(ET);  // entries per 16-byte piece
    constexpr int UNR = sl_unr<Pass>();
    constexpr int RW = 32 * UNR;                      // 16-byte pieces per round
    if (geo.reset_next && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *geo.reset_next = 0;
    (void)tile;
    const int nact = *geo.n_act;
    // genes [0, nheavy) of the list take a warp each, the rest eight lanes each
    const int nheavy = geo.n_heavy ? min(nact, *geo.n_heavy) : nact;
    // block y takes the slots y, y + T, y + 2T, ... (T = gridDim.y) of each
    // part: with the active genes listed in decreasing order of entries,
    // every block gets a like share of the work and hands its largest genes
    // out first, so the block's last warps finish together
    const int T = gridDim.y, y = blockIdx.y;
    if (y >= nact) return;
    const int s = blockIdx.x, S = geo.S, U = geo.U;
    extern __shared__ double Es[];  // [kSliceCells] exp(offset) of the slice's cells
    const int c0 = __ldg(geo.sl_start + s), nc = __ldg(geo.sl_start + s + 1) - c0;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31, nw = blockDim.x >> 5;
    // per warp: the psi tables of its current gene (passes with TABLES)
    double* wtab = Es + kSliceCells + warp * kGrpTab;
    // beta_0's pass stages log1p(1 / exp(offset)) instead: its term for a
    // count of 1 (two thirds of the nonzeros of sparse single-cell counts),
    // the same expression as PassInitZ::sparse
    constexpr bool kInitZ = std::is_same<Pass, PassInitZ>::value;
    {
        // every thread's kSliceCells / kSlNT loads in flight at once (a loop
        // of dependent L2 round trips would hold the block for microseconds)
        constexpr int K = kSliceCells / kSlNT;
        double e[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = t + k * kSlNT;
            e[k] = i < nc ? __ldg(geo.E + c0 + i) : 1.0;
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = t + k * kSlNT;
            if (i < nc) Es[i] = kInitZ ? log1p(1.0 / e[k]) : e[k];
        }
    }
    const int u = __ldg(geo.sl_key + s) / geo.C;
    const bool first = s == __ldg(geo.kslice + u * geo.C);  // the group's rule goes here
    constexpr bool kRule = !std::is_same<Pass, PassInitZ>::value;  // zero counts contribute
    const int m = (kRule && first) ? __ldg(geo.rm + u) : 0;
    // the group's rule (node weights, exp(node offsets)) in shared memory:
    // every gene of the block evaluates it
    double* rule = Es + kSliceCells + (Pass::TABLES ? nw * kGrpTab : 0);
    for (int j = t; j < m; j += blockDim.x) {
        rule[j] = __ldg(geo.rw + (int64_t)u * kRuleCap + j);
        rule[kRuleCap + j] = __ldg(geo.res + (int64_t)u * kRuleCap + j);
    }
    const uint4* __restrict__ v4 = static_cast<const uint4*>(geo.gent);
    // the block's genes are handed out one at a time (a shared counter), so
    // warps that drew short genes take more of them
    __shared__ int next_k, next_l;
    if (t == 0) {
        next_k = 0;
        next_l = 0;
    }
    __syncthreads();
    auto take = [&]() -> SlItem {
        int k = 0;
        if (lane == 0) k = atomicAdd(&next_k, 1);
        SlItem it{y + __shfl_sync(0xffffffffu, k, 0) * T, 0, 0.0, 0, 0};
        if (it.j >= nheavy) it.j = nact;  // past the heavy part
        if (it.j < nact) {
            it.g = __ldg(geo.act + it.j);
            it.A = __ldg(geo.rowexp + (int64_t)it.g * U + u);
            it.e0 = __ldg(geo.gptr + (int64_t)it.g * (S + 1) + s);
            it.e1 = __ldg(geo.gptr + (int64_t)it.g * (S + 1) + s + 1);
        }
        return it;
    };
    // a heavy gene's parameters, psi tables and rule terms (lanes over the
    // rule's nodes); the MLE's weight sums are final after the rule and
    // stored at once (the nonzeros add only FP64 scalars), freeing their
    // registers for the entries
    auto gene_start = [&](const SlItem& it, typename Pass::Gene& gpar, Acc& acc, double*& o) {
        gpar = Pass::load(prm, it.g);
        if constexpr (Pass::TABLES) {
            // the gene's psi tables (grp_psi_tables_kernel) into the warp's slot
            const double* src = geo.psitab + (int64_t)it.j * kGrpTab;
            for (int i = lane; i < kGrpTab; i += 32) wtab[i] = __ldg(src + i);
            __syncwarp();
            gpar.tab.d1 = wtab;
            gpar.tab.d2 = wtab + kPsiTab;
            gpar.tab.pa = wtab[2 * kPsiTab];
            gpar.tab.ta = wtab[2 * kPsiTab + 1];
        }
        acc.zero();
        for (int j = lane; j < m; j += 32) {
            acc.q = rule[j];
            Pass::template dense<double>(gpar, it.A * rule[kRuleCap + j], acc);
        }
        acc.q = 1.0;
        o = geo.gsum + ((int64_t)it.j * S + s) * NQ;
        if constexpr (NS > 0) {
#pragma unroll
            for (int i = 0; i < NWV; ++i) {
                const double v = warp_sum(acc.w[i]);
                if (lane == 0) o[i] = v;
            }
        }
    };
    auto gene_end = [&](Acc& acc, double* o) {
        if constexpr (NS == 0) {
#pragma unroll
            for (int i = 0; i < NWV; ++i) {
                const double v = warp_sum(acc.w[i]);
                if (lane == 0) o[i] = v;
            }
        }
#pragma unroll
        for (int i = 0; i < NS; ++i) {
            const double v = warp_sum(acc.s[i]);
            if (lane == 0) o[NWV + i] = v;
        }
    };
    // one entry: the pass's nonzero term (beta_0: the staged term for y = 1,
    // else log1p(y / exp(offset)) with exp(offset) from L2)
    auto entry = [&](const ET c, const typename Pass::Gene& gpar, double A, Acc& acc) {
        if constexpr (kInitZ) {
            const float y = Ent::y(c);
            const int loc = Ent::loc(c);
            acc.s[0] += y == 1.f ? Es[loc] : log1p((double)y / __ldg(geo.E + c0 + loc));
        } else if constexpr (std::is_same<VT, uint16_t>::value) {
            // (a 16-bit count converts to FP64 exactly, in one step)
            Pass::template sparse<double>(gpar, A * Es[Ent::loc(c)], (double)(c >> 16), acc);
        } else {
            Pass::template sparse<double>(gpar, A * Es[Ent::loc(c)], Ent::y(c), acc);
        }
    };
    // the entries of one 16-byte piece inside the gene's range; positions
    // relative to the first entry of the gene's first piece: the piece
    // starts at ea, the range is [lo, hi)
    auto piece = [&](const uint4& v, int ea, int lo, int hi, const typename Pass::Gene& gpar, double A,
                     Acc& acc) {
        const ET* c = reinterpret_cast<const ET*>(&v);
        if (ea >= lo && ea + EPL <= hi) {  // a whole piece inside the range
#pragma unroll
            for (int rr = 0; rr < EPL; ++rr) entry(c[rr], gpar, A, acc);
        } else {
#pragma unroll
            for (int rr = 0; rr < EPL; ++rr)
                if (ea + rr >= lo && ea + rr < hi) entry(c[rr], gpar, A, acc);
        }
    };
    {
        // entries loaded to registers, UNR pieces per lane in flight; the
        // next gene's range is loaded while this one runs
        SlItem cur = take();
        if constexpr (kInitZ && std::is_same<VT, uint16_t>::value) {
            // beta_0 on 16-bit counts: a count of 1 takes the staged term; the
            // others are queued (warp ballots, in entry order) and evaluated
            // 32 at a time, every lane on a log1p, instead of a divergent
            // log1p path in nearly every entry position
            static_assert(RW * EPL <= kInitQ - 32, "queue holds a round and a partial batch");
            uint32_t* qbuf = reinterpret_cast<uint32_t*>(rule + 2 * kRuleCap) + warp * kInitQ;
            const unsigned lt = (1u << lane) - 1u;
            while (cur.j < nact) {
                const SlItem nx = take();
                typename Pass::Gene gpar;
                Acc acc;
                double* o;
                gene_start(cur, gpar, acc, o);
                const int64_t b0 = cur.e0 / EPL;
                const int nb = (int)((cur.e1 + EPL - 1) / EPL - b0);
                const int lo = (int)(cur.e0 - b0 * EPL), hi = (int)(cur.e1 - b0 * EPL);
                int qn = 0;  // queued entries (warp-uniform)
                auto drain = [&](bool all) {
                    __syncwarp();
                    while (qn >= 32 || (all && qn > 0)) {
                        const int k = qn - 32 + lane;  // the newest 32, or all that are left
                        if (k >= 0) {
                            const uint32_t c = qbuf[k];
                            acc.s[0] += log1p((double)(c >> 16) / __ldg(geo.E + c0 + (int)(c & 0xffffu)));
                        }
                        qn = qn > 32 ? qn - 32 : 0;
                    }
                    __syncwarp();
                };
                for (int b = 0; b < nb; b += RW) {
                    const int base = b + lane;
                    uint4 v[UNR];
#pragma unroll
                    for (int q = 0; q < UNR; ++q)
                        v[q] = base + 32 * q < nb ? ld_stream(v4 + b0 + base + 32 * q) : make_uint4(0, 0, 0, 0);
#pragma unroll
                    for (int q = 0; q < UNR; ++q) {
                        const uint32_t* c = reinterpret_cast<const uint32_t*>(&v[q]);
                        const int ea = (base + 32 * q) * EPL;
                        const bool inb = base + 32 * q < nb;
#pragma unroll
                        for (int rr = 0; rr < EPL; ++rr) {
                            const bool valid = inb && ea + rr >= lo && ea + rr < hi;
                            const uint32_t y = c[rr] >> 16;
                            if (valid && y == 1u) acc.s[0] += Es[c[rr] & 0xffffu];
                            const bool slow = valid && y != 1u;
                            const unsigned bal = __ballot_sync(0xffffffffu, slow);
                            if (slow) qbuf[qn + __popc(bal & lt)] = c[rr];
                            qn += __popc(bal);
                        }
                    }
                    drain(false);
                }
                drain(true);
                gene_end(acc, o);
                cur = nx;
            }
        }
        while (cur.j < nact) {
            const SlItem nx = take();
            typename Pass::Gene gpar;
            Acc acc;
            double* o;
            gene_start(cur, gpar, acc, o);
            const int64_t b0 = cur.e0 / EPL;
            const int nb = (int)((cur.e1 + EPL - 1) / EPL - b0);
            const int lo = (int)(cur.e0 - b0 * EPL), hi = (int)(cur.e1 - b0 * EPL);
            for (int base = lane; base < nb; base += RW) {
                uint4 v[UNR];
#pragma unroll
                for (int q = 0; q < UNR; ++q)
                    if (base + 32 * q < nb) v[q] = ld_stream(v4 + b0 + base + 32 * q);
#pragma unroll
                for (int q = 0; q < UNR; ++q)
                    if (base + 32 * q < nb) piece(v[q], (base + 32 * q) * EPL, lo, hi, gpar, cur.A, acc);
            }
            gene_end(acc, o);
            cur = nx;
            if constexpr (Pass::TABLES) __syncwarp();  // the table slot is rewritten next
        }
    }
    {
        // the light genes: four per warp, eight lanes each (the per-gene
        // bookkeeping is shared by four genes), loads straight to registers;
        // their psi tables (passes with TABLES) are read from L2
        constexpr int LW = 8, LUNR = Pass::TABLES ? 1 : UNR, LRW = LW * LUNR;
        const int sub = lane / LW, sl = lane % LW;
        const int nlight = nact - nheavy;
        // a batch of four: each eight lanes' gene (j = -1: none); `any`: the
        // batch has one (warp-uniform).  The next batch's loads are in flight
        // while this one runs.
        auto ltake = [&](bool& any) -> SlItem {
            int k0 = 0;
            if (lane == 0) k0 = atomicAdd(&next_l, 32 / LW);
            k0 = __shfl_sync(0xffffffffu, k0, 0);
            any = y + k0 * T < nlight;
            const int jl = y + (k0 + sub) * T;
            SlItem it{jl < nlight ? nheavy + jl : -1, 0, 0.0, 0, 0};
            if (it.j >= 0) {
                it.g = __ldg(geo.act + it.j);
                it.A = __ldg(geo.rowexp + (int64_t)it.g * U + u);
                it.e0 = __ldg(geo.gptr + (int64_t)it.g * (S + 1) + s);
                it.e1 = __ldg(geo.gptr + (int64_t)it.g * (S + 1) + s + 1);
            }
            return it;
        };
        bool any = false;
        SlItem cur = ltake(any);
        while (any) {
            bool any_nx = false;
            const SlItem nx = ltake(any_nx);
            const bool valid = cur.j >= 0;
            const int j = cur.j;
            Acc acc;
            acc.zero();
            if (valid) {
                const int g = cur.g;
                const double A = cur.A;
                const int64_t e0 = cur.e0, e1 = cur.e1;
                typename Pass::Gene gpar = Pass::load(prm, g);
                if constexpr (Pass::TABLES) {
                    const double* src = geo.psitab + (int64_t)j * kGrpTab;
                    gpar.tab.d1 = src;
                    gpar.tab.d2 = src + kPsiTab;
                    gpar.tab.pa = __ldg(src + 2 * kPsiTab);
                    gpar.tab.ta = __ldg(src + 2 * kPsiTab + 1);
                }
                for (int jr = sl; jr < m; jr += LW) {
                    acc.q = rule[jr];
                    Pass::template dense<double>(gpar, A * rule[kRuleCap + jr], acc);
                }
                acc.q = 1.0;
                const int64_t b0 = e0 / EPL;
                const int nb = (int)((e1 + EPL - 1) / EPL - b0);
                const int lo = (int)(e0 - b0 * EPL), hi = (int)(e1 - b0 * EPL);
                for (int base = sl; base < nb; base += LRW) {
                    uint4 v[LUNR];
#pragma unroll
                    for (int q = 0; q < LUNR; ++q)
                        if (base + LW * q < nb) v[q] = ld_stream(v4 + b0 + base + LW * q);
#pragma unroll
                    for (int q = 0; q < LUNR; ++q)
                        if (base + LW * q < nb) piece(v[q], (base + LW * q) * EPL, lo, hi, gpar, A, acc);
                }
            }
            // sums over each gene's eight lanes
#pragma unroll
            for (int i = 0; i < NWV; ++i) {
#pragma unroll
                for (int o = LW / 2; o > 0; o >>= 1) acc.w[i] += __shfl_xor_sync(0xffffffffu, acc.w[i], o);
            }
#pragma unroll
            for (int i = 0; i < NS; ++i) {
#pragma unroll
                for (int o = LW / 2; o > 0; o >>= 1) acc.s[i] += __shfl_xor_sync(0xffffffffu, acc.s[i], o);
            }
            if (valid && sl == 0) {
                double* o = geo.gsum + ((int64_t)j * S + s) * NQ;
#pragma unroll
                for (int i = 0; i < NWV; ++i) o[i] = acc.w[i];
#pragma unroll
                for (int i = 0; i < NS; ++i) o[NWV + i] = acc.s[i];
            }
            cur = nx;
            any = any_nx;
        }
    }
}

// psi(v + a) - psi(a) and psi1(v + a) - psi1(a) (v < kPsiTab), psi(a),
// psi1(a) for every active gene of an MLE evaluation (a = 1/theta), built
// as the block-per-gene pass builds them; the slice-major pass copies a
// gene's tables into shared memory once per (gene, slice)
__global__ void __launch_bounds__(32) grp_psi_tables_kernel(const int32_t* act, const int32_t* n_act,
                                                            const double* log_theta, double* tab) {
    __shared__ double a[1];
    __shared__ double t[2 * kPsiTab];
    __shared__ double scr[kPsiTab];
    const int slot = blockIdx.x;
    if (slot >= *n_act) return;
    const double th = exp(log_theta[__ldg(act + slot)]);
    if (threadIdx.x == 0) a[0] = 1.0 / th;
    __syncthreads();
    build_psi_tables(1, a, t, scr);
    double* o = tab + (int64_t)slot * kGrpTab;
    for (int i = threadIdx.x; i < 2 * kPsiTab; i += 32) o[i] = t[i];
    if (threadIdx.x == 0) {
        o[2 * kPsiTab] = digamma_d(a[0]);
        o[2 * kPsiTab + 1] = trigamma_d(a[0]);
    }
}

// exp(x_u . beta) for every (active gene, design group): the factor the
// slice-major pass multiplies each cell's exp(offset) by, stored by gene
// ([G][U]; the IRLS step refreshes a gene's row after its update)
__global__ void grp_rowexp_kernel(GrpGeom geo, const double* beta_d, int64_t max_slots) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int U = geo.U, P = geo.P;
    const int64_t slot = i / U;
    if (slot >= *geo.n_act || slot >= max_slots) return;
    const int u = (int)(i - slot * U);
    const int64_t g = __ldg(geo.act + slot);
    const double* b = beta_d + g * P;
    double a = 0.0;
    for (int e = __ldg(geo.rptr + u); e < __ldg(geo.rptr + u + 1); ++e)
        a += __ldg(geo.rval + e) * __ldg(b + __ldg(geo.rcol + e));
    geo.rowexp[g * U + u] = exp(a);
}

// Per active gene: group sums over the gene's slices (in slice order) and
// the assembly of the pass's partial sums (one segment).
template <class Pass>
__global__ void __launch_bounds__(256) grp_assemble_kernel(GrpGeom geo) {
    constexpr int NW = Pass::NW, NV = Pass::NV, NF = Pass::NF;
    constexpr int NWV = NW + NV + NF, NS = Pass::NS, NQ = NWV + NS;
    const int slot = blockIdx.x;
    if (slot >= *geo.n_act) return;
    const int P = geo.P, U = geo.U, C = geo.C, S = geo.S;
    extern __shared__ double gs[];  // [U][NQ]
    const int t = threadIdx.x, nt = blockDim.x;
    const double* gsum = geo.gsum + (int64_t)slot * S * NQ;
    for (int i = t; i < U * NQ; i += nt) {
        const int q = i / NQ, c = i - q * NQ;
        double v = 0.0;
        for (int sl = __ldg(geo.kslice + q * C); sl < __ldg(geo.kslice + q * C + C); ++sl)
            v += gsum[sl * NQ + c];
        gs[i] = v;
    }
    __syncthreads();
    const int NE = P * (P + 1) / 2;
    const int NA = NW * NE + NV * P + NF;
    for (int a = t; a < NA + NS; a += nt) {
        double s = 0.0;
        if (a < NW * NE) {
            const int w = a / NE, qq = a - w * NE;
            for (int e = __ldg(geo.qptr + qq); e < __ldg(geo.qptr + qq + 1); ++e)
                s += gs[__ldg(geo.qu + e) * NQ + w] * __ldg(geo.qv + e);
        } else if (a < NW * NE + NV * P) {
            const int r = a - NW * NE;
            const int v = r / P, i = r - v * P;
            for (int e = __ldg(geo.vptr + i); e < __ldg(geo.vptr + i + 1); ++e)
                s += gs[__ldg(geo.vu + e) * NQ + NW + v] * __ldg(geo.vv + e);
        } else {
            const int f = a - NW * NE - NV * P;
            const int col = a < NA ? NW + NV + f : NWV + (a - NA);
            for (int u = 0; u < U; ++u) s += gs[u * NQ + col];
        }
        if (a < NA)
            geo.partW[(int64_t)slot * NA + a] = s;
        else
            geo.partS[(int64_t)slot * NS + (a - NA)] = s;
    }
}

// the sort keys of the work order of the slice-major passes: the gene's
// entries (the sort is descending) and its index
__global__ void gene_entries_kernel(const int64_t* rowptr, int64_t G, int32_t* key, int32_t* idx) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = rowptr[g + 1] - rowptr[g];
        key[g] = (int32_t)(e < INT32_MAX ? e : INT32_MAX);
        idx[g] = (int32_t)g;
    }
}
cudaError_t launch_gene_entries(const int64_t* rowptr, int64_t G, int32_t* key, int32_t* idx,
                                cudaStream_t st) {
    if (G <= 0) return cudaSuccess;
    gene_entries_kernel<<<(unsigned)std::min<int64_t>(nblk(G, 256), 1024), 256, 0, st>>>(rowptr, G, key, idx);
    return cudaGetLastError();
}

int grp_slices_tile(int64_t hint, int S, int sm_count, int waves) {
    // one resident block per SM (1,024 threads at 64 registers, the 128 KB
    // slice stage); about `waves` waves (3 unless tuned), the tile count
    // chosen so the last wave is nearly full, tiles of 16..1024 genes
    const int64_t cap = (int64_t)sm_count;
    int64_t tiles = std::max<int64_t>(1, ((int64_t)std::max(1, waves) * cap + S - 1) / S);
    double best_eff = 0.0;
    int64_t best = tiles;
    for (int64_t tc = tiles; tc <= 2 * tiles; ++tc) {
        const double waves = (double)tc * S / (double)cap;
        const double eff = waves / std::ceil(waves);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = tc;
        }
        if (eff >= 0.95) break;
    }
    const int64_t tile = (hint + best - 1) / best;
    return (int)std::max<int64_t>(16, std::min<int64_t>(1024, tile));
}

template <class Pass>
static cudaError_t slices_run(const GrpGeom& geo, typename Pass::Params prm, int val_u16,
                              int max_slots, int tile, bool assemble, bool rowexp_fresh, cudaStream_t st) {
    constexpr int NQ = Pass::NW + Pass::NV + Pass::NF + Pass::NS;
    const size_t smem = sl_smem_bytes<Pass>();
    if constexpr (Pass::TABLES)
        grp_psi_tables_kernel<<<(unsigned)max_slots, 32, 0, st>>>(geo.act, geo.n_act, prm.log_theta,
                                                                 geo.psitab);
    if (!rowexp_fresh) {
        const int64_t nrow = (int64_t)max_slots * geo.U;
        grp_rowexp_kernel<<<nblk(nrow, 256), 256, 0, st>>>(geo, prm.beta_d, max_slots);
    }
    dim3 grid((unsigned)geo.S, (unsigned)((max_slots + tile - 1) / tile));
    auto go = [&](auto kern) -> cudaError_t {
        cudaError_t e = raise_dyn_smem(kern, smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, kSlNT, smem, st>>>(geo, prm, tile);
        return cudaGetLastError();
    };
    cudaError_t e = val_u16 ? go(grp_slices_kernel<Pass, uint16_t>) : go(grp_slices_kernel<Pass, float>);
    if (e != cudaSuccess || !assemble) return e;
    grp_assemble_kernel<Pass><<<(unsigned)max_slots, 256, (size_t)geo.U * NQ * sizeof(double), st>>>(geo);
    return cudaGetLastError();
}

int grp_slices_nq(PassKind k) { return pass_nw(k) + pass_nv(k) + pass_nf(k) + pass_ns(k); }

cudaError_t launch_grp_slices(PassKind kind, const GrpGeom& geo, const PassParamsAny& pa,
                              int val_u16, int max_slots, int tile, bool assemble, cudaStream_t st,
                              bool rowexp_fresh) {
    if (max_slots <= 0) return cudaSuccess;
    if (kind == PASS_IRLS)
        return slices_run<PassIRLS>(geo, PassIRLS::Params{pa.beta, pa.beta_d, pa.k}, val_u16,
                                    max_slots, tile, assemble, rowexp_fresh, st);
    if (kind == PASS_MLE)
        return slices_run<PassMLE>(geo, PassMLE::Params{pa.beta, pa.beta_d, pa.log_theta}, val_u16,
                                   max_slots, tile, assemble, rowexp_fresh, st);
    if (kind == PASS_MOM)
        return slices_run<PassMOM>(geo, PassMOM::Params{pa.beta, pa.beta_d}, val_u16, max_slots, tile,
                                   assemble, rowexp_fresh, st);
    if (kind == PASS_SANDWICH)
        return slices_run<PassSandwich>(geo, PassSandwich::Params{pa.beta, pa.beta_d, pa.theta}, val_u16,
                                        max_slots, tile, assemble, rowexp_fresh, st);
    return cudaErrorInvalidValue;
}

// init_beta (R/beta.R:12-24) on a grouped design: X' z with
// z = log1p(y / exp(offset)) (zero where y = 0) is sum_u x_u z_u where z_u
// sums the group's nonzeros, so the nonzeros are read once
// (grp_slices_kernel<PassInitZ>, per-(gene, slice) sums) and then, per gene,
// z_u = the sum over the group's slices, r = X' z = sum_u x_u z_u and
// beta_0 = (X'X)^-1 r.
__global__ void grp_init_finish_kernel(GrpGeom geo, const double* ginv, int64_t G, double* beta,
                                       float* beta_f) {
    __shared__ double zu[kMaxGroups];
    __shared__ double r[32];
    const int64_t g = blockIdx.x;
    if (g >= G) return;
    const int t = threadIdx.x, nt = blockDim.x;
    const int U = geo.U, C = geo.C, P = geo.P, S = geo.S;
    const double* gs = geo.gsum + g * S;
    for (int u = t; u < U; u += nt) {
        double z = 0.0;
        for (int sl = __ldg(geo.kslice + u * C); sl < __ldg(geo.kslice + u * C + C); ++sl) z += gs[sl];
        zu[u] = z;
    }
    __syncthreads();
    if (t < P) {
        double v = 0.0;
        for (int u = 0; u < U; ++u) v += geo.xg[u * P + t] * zu[u];
        r[t] = v;
    }
    __syncthreads();
    if (t < P) {
        double b = 0.0;
        for (int j = 0; j < P; ++j) b += ginv[j * P + t] * r[j];
        beta[g * P + t] = b;
        beta_f[g * P + t] = (float)b;
    }
}

cudaError_t launch_grp_init_beta(const GrpGeom& geo, int val_u16, const double* zero_beta,
                                 const double* ginv, int64_t G, int tile, double* beta,
                                 float* beta_f, cudaStream_t st) {
    if (G <= 0) return cudaSuccess;
    PassInitZ::Params prm{nullptr, zero_beta};
    const size_t smem = sl_smem_bytes<PassInitZ>();
    // (beta_0's pass reads no exp(x_u . beta): no row factors)
    dim3 grid((unsigned)geo.S, (unsigned)((G + tile - 1) / tile));
    auto go = [&](auto kern) -> cudaError_t {
        cudaError_t e = raise_dyn_smem(kern, smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, kSlNT, smem, st>>>(geo, prm, tile);
        return cudaGetLastError();
    };
    cudaError_t e = val_u16 ? go(grp_slices_kernel<PassInitZ, uint16_t>) : go(grp_slices_kernel<PassInitZ, float>);
    if (e != cudaSuccess) return e;
    grp_init_finish_kernel<<<(unsigned)G, 64, 0, st>>>(geo, ginv, G, beta, beta_f);
    return cudaGetLastError();
}

template <class Pass>
static typename Pass::Params grp_params(const PassParamsAny& a);
template <> PassIRLS::Params grp_params<PassIRLS>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.k}; }
template <> PassMOM::Params grp_params<PassMOM>(const PassParamsAny& a) { return {a.beta, a.beta_d}; }
template <> PassMLE::Params grp_params<PassMLE>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.log_theta}; }
template <> PassSandwich::Params grp_params<PassSandwich>(const PassParamsAny& a) { return {a.beta, a.beta_d, a.theta}; }

size_t grp_smem_bytes(PassKind k, int P, int NGq, int S) {
    const int nq = pass_nw(k) + pass_nv(k) + pass_nf(k) + pass_ns(k);
    return ((size_t)P + (size_t)NGq * nq + (size_t)(NGq + S + kGrpUnitsMax) * nq) * sizeof(double) +
           (size_t)(S + 1) * sizeof(int);
}

template <class Pass>
static cudaError_t grp_run(const GrpGeom& geo, const PassParamsAny& pa, PassKind kind, int val_u16,
                           int max_slots, cudaStream_t st) {
    const int NGq = geo.fine ? geo.U * geo.C : geo.U;
    const size_t smem = grp_smem_bytes(kind, geo.P, NGq, geo.S);
    auto prm = grp_params<Pass>(pa);
    auto go = [&](auto kern) -> cudaError_t {
        // static shared memory (psi tables) counts against the 48 KB default
        cudaError_t e = raise_dyn_smem(kern, smem);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)max_slots, 256, smem, st>>>(geo, prm);
        return cudaGetLastError();
    };
    return val_u16 ? go(grp_pass_kernel<Pass, uint16_t>) : go(grp_pass_kernel<Pass, float>);
}

cudaError_t launch_grp_pass(PassKind kind, const GrpGeom& geo, const PassParamsAny& prm, int val_u16,
                            int max_slots, cudaStream_t st) {
    if (max_slots <= 0) return cudaSuccess;
    switch (kind) {
        case PASS_IRLS: return grp_run<PassIRLS>(geo, prm, kind, val_u16, max_slots, st);
        case PASS_MOM: return grp_run<PassMOM>(geo, prm, kind, val_u16, max_slots, st);
        case PASS_MLE: return grp_run<PassMLE>(geo, prm, kind, val_u16, max_slots, st);
        case PASS_SANDWICH: return grp_run<PassSandwich>(geo, prm, kind, val_u16, max_slots, st);
    }
    return cudaErrorInvalidValue;
}

// cells in slice order: for position i of the key-sorted cells (pnew[i] is
// the original cell), its slice (the last with sl_start <= i), its index in
// the slice, and exp(offset) in slice order
__global__ void slice_cells_kernel(const int32_t* pnew, const int32_t* sl_start, int S, int64_t n,
                                   const double* off, int32_t* cslice, int32_t* cloc, double* E) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = 0, hi = S;  // sl_start[lo] <= i < sl_start[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (sl_start[mid] <= i) lo = mid; else hi = mid;
    }
    const int c = pnew[i];
    cslice[c] = lo;
    // slice (high 16 bits: fewer than kMaxSlices < 2^16) and index in the
    // slice (low 16 bits: fewer than kSliceCells), one gather for the copy
    cloc[c] = (int32_t)(((uint32_t)lo << 16) | (uint32_t)(i - sl_start[lo]));
    E[i] = exp(off[c]);
}

cudaError_t launch_slice_cells(const int32_t* pnew, const int32_t* sl_start, int S, int64_t n,
                               const double* off, int32_t* cslice, int32_t* cloc, double* E,
                               cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    slice_cells_kernel<<<nblk(n, 256), 256, 0, st>>>(pnew, sl_start, S, n, off, cslice, cloc, E);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------
// launchers of the grouping steps
// ---------------------------------------------------------------------
cudaError_t launch_row_hash(const double* X, int64_t n, int P, uint64_t* h, int32_t* idx,
                            cudaStream_t st) {
    row_hash_kernel<<<nblk(n, 256), 256, 0, st>>>(X, n, P, h, idx);
    return cudaGetLastError();
}
cudaError_t launch_group_heads(const double* X, int64_t n, int P, const uint64_t* hs,
                               const int32_t* is, int32_t* flag, int32_t* bad, cudaStream_t st) {
    group_heads_kernel<<<nblk(n, 256), 256, 0, st>>>(X, n, P, hs, is, flag, bad);
    return cudaGetLastError();
}
cudaError_t launch_group_assign(const int32_t* is, const int32_t* incl, const int32_t* flag,
                                int64_t n, int32_t* ucell, int32_t* head, cudaStream_t st) {
    group_assign_kernel<<<nblk(n, 256), 256, 0, st>>>(is, incl, flag, n, ucell, head);
    return cudaGetLastError();
}
cudaError_t launch_group_rows(const double* X, int64_t n, int P, const int32_t* head, int U,
                              double* xg, cudaStream_t st) {
    group_rows_kernel<<<nblk((int64_t)U * P, 256), 256, 0, st>>>(X, n, P, head, U, xg);
    return cudaGetLastError();
}
cudaError_t launch_fine_keys(const int32_t* ucell, const int32_t* ends, int C, int64_t n,
                             int32_t* fkey, int32_t* cell, cudaStream_t st) {
    fine_keys_kernel<<<nblk(n, 256), 256, 0, st>>>(ucell, ends, C, n, fkey, cell);
    return cudaGetLastError();
}
cudaError_t launch_group_starts(const int32_t* ks, int64_t n, int K, int64_t* gstart,
                                cudaStream_t st) {
    group_starts_kernel<<<nblk(K + 1, 256), 256, 0, st>>>(ks, n, K, gstart);
    return cudaGetLastError();
}
cudaError_t launch_gather_keys(const int32_t* keys, const int32_t* cells, int64_t n, int32_t* out,
                               cudaStream_t st) {
    gather_keys_kernel<<<nblk(n, 256), 256, 0, st>>>(keys, cells, n, out);
    return cudaGetLastError();
}
cudaError_t launch_exp(const double* x, int64_t n, double* y, cudaStream_t st) {
    exp_kernel<<<nblk(n, 256), 256, 0, st>>>(x, n, y);
    return cudaGetLastError();
}
cudaError_t launch_group_rules(const int32_t* permC, const int64_t* gsC, const int32_t* permF,
                               const int64_t* gsF, int U, int nrules, const double* off, int64_t n,
                               double* scr, double* rs, double* rw, int32_t* rm, double* rerr,
                               int32_t* bad, cudaStream_t st) {
    group_rules_kernel<<<(unsigned)nrules, kRuleNT, 0, st>>>(permC, gsC, permF, gsF, U, off, n, scr,
                                                             rs, rw, rm, rerr, bad);
    return cudaGetLastError();
}
int group_csr_segment(int64_t nnz, int64_t G, int K) {
    int S = 2048;  // entries per segment; the count table stays below 2^27 entries
    while (((nnz / S) + G) * (int64_t)K > ((int64_t)1 << 27) && S < (1 << 24)) S *= 2;
    return S;
}

cudaError_t launch_group_segments(const int64_t* rowptr, int64_t G, int S, int64_t* segcnt,
                                  int64_t* segbase, void* scan_tmp, size_t* scan_bytes,
                                  cudaStream_t st) {
    if (!scan_tmp)  // size query
        return cub::DeviceScan::ExclusiveSum(nullptr, *scan_bytes, segcnt, segbase, (int)(G + 1));
    cudaError_t e = cudaMemsetAsync(segcnt + G, 0, sizeof(int64_t), st);
    if (e != cudaSuccess) return e;
    if (G > 0) seg_count_kernel<<<nblk(G, 256), 256, 0, st>>>(rowptr, G, S, segcnt);
    return cub::DeviceScan::ExclusiveSum(scan_tmp, *scan_bytes, segcnt, segbase, (int)(G + 1), st);
}

cudaError_t launch_group_csr(const int64_t* rowptr, const int32_t* col, const void* val, int val_u16,
                             int64_t G, const int64_t* segbase, int S, const int32_t* ckey,
                             const int32_t* cloc, int K, int32_t* hist, int64_t nsegs,
                             int64_t* gptr, void* gent, cudaStream_t st) {
    if (G <= 0) return cudaSuccess;
    int wpb = 12288 / K;  // 48 KB of per-warp key tables per block
    wpb = wpb < 1 ? 1 : (wpb > 8 ? 8 : wpb);
    const size_t smem = (size_t)wpb * K * sizeof(int32_t);
    const unsigned grid = (unsigned)((nsegs + wpb - 1) / wpb);
    if (grid > 0) seg_hist_kernel<<<grid, 32 * wpb, smem, st>>>(rowptr, col, G, segbase, S, ckey, K, hist);
    seg_offsets_kernel<<<(unsigned)G, kOffNT, 0, st>>>(rowptr, G, segbase, K, hist, gptr);
    if (grid > 0) {
        if (val_u16)
            seg_scatter_kernel<uint16_t><<<grid, 32 * wpb, smem, st>>>(
                rowptr, col, static_cast<const uint16_t*>(val), G, segbase, S, cloc, K, hist,
                static_cast<GrpEnt<uint16_t>::T*>(gent));
        else
            seg_scatter_kernel<float><<<grid, 32 * wpb, smem, st>>>(
                rowptr, col, static_cast<const float*>(val), G, segbase, S, cloc, K, hist,
                static_cast<GrpEnt<float>::T*>(gent));
    }
    return cudaGetLastError();
}

}  // namespace devil
