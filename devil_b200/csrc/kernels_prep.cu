// Preparation kernels: count-matrix conversion, design staging, per-gene
// statistics, size factors (R/size_factors.R), theta_0
// (R/overdispersion.R:129-135), beta_0 (R/beta.R:13-20, R/main.R:404-406)
// and the CSR offsets of every cell segment.
#include "internal.h"

#include <type_traits>

namespace devil {

static inline unsigned nblk(int64_t m, int t) { return (unsigned)((m + t - 1) / t); }

// ------------------------------------------------------------------
// dense -> CSR (gene-major)
// ------------------------------------------------------------------
__global__ void dense_count_kernel(const void* Y, int is_f64, int cell_major, int64_t G, int64_t n,
                                   int64_t* rowcnt) {
    int64_t g = blockIdx.x;
    if (g >= G) return;
    int64_t cnt = 0;
    for (int64_t c = threadIdx.x; c < n; c += blockDim.x) {
        int64_t idx = cell_major ? c * G + g : g * n + c;
        double v = is_f64 ? ((const double*)Y)[idx] : (double)((const float*)Y)[idx];
        cnt += (v != 0.0);
    }
    cnt = warp_sum(cnt);
    __shared__ int64_t red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        rowcnt[g] = s;
    }
}

// one warp per gene walks its row in order and compacts the nonzeros
__global__ void dense_fill_kernel(const void* Y, int is_f64, int cell_major, int64_t G, int64_t n,
                                  const int64_t* rowptr, int32_t* col, float* val) {
    int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (g >= G) return;
    int64_t pos = rowptr[g];
    for (int64_t c0 = 0; c0 < n; c0 += 32) {
        int64_t c = c0 + lane;
        double v = 0.0;
        if (c < n) {
            int64_t idx = cell_major ? c * G + g : g * n + c;
            v = is_f64 ? ((const double*)Y)[idx] : (double)((const float*)Y)[idx];
        }
        unsigned m = __ballot_sync(0xffffffffu, v != 0.0);
        if (v != 0.0) {
            int r = __popc(m & ((1u << lane) - 1u));
            col[pos + r] = (int32_t)c;
            val[pos + r] = (float)v;
        }
        pos += __popc(m);
    }
}

cudaError_t launch_dense_count(const void* Y, int is_f64, int cell_major, int64_t G, int64_t n,
                               int64_t* rowcnt, cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    dense_count_kernel<<<(unsigned)G, 256, 0, st>>>(Y, is_f64, cell_major, G, n, rowcnt);
    return cudaGetLastError();
}
cudaError_t launch_dense_fill(const void* Y, int is_f64, int cell_major, int64_t G, int64_t n,
                              const int64_t* rowptr, int32_t* col, float* val, cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    dense_fill_kernel<<<nblk(G, 8), 256, 0, st>>>(Y, is_f64, cell_major, G, n, rowptr, col, val);
    return cudaGetLastError();
}

__global__ void f64_to_f32_kernel(const double* in, float* out, int64_t m) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}
cudaError_t launch_csr_f64_to_f32(const double* in, float* out, int64_t nnz, cudaStream_t st) {
    if (nnz == 0) return cudaSuccess;
    f64_to_f32_kernel<<<(unsigned)std::min<int64_t>(nblk(nnz, 256), 148 * 16), 256, 0, st>>>(in, out, nnz);
    return cudaGetLastError();
}
cudaError_t launch_double_to_float(const double* in, float* out, int64_t m, cudaStream_t st) {
    return launch_csr_f64_to_f32(in, out, m, st);
}

// CSC (cell-major) -> sortable (gene, cell) keys
// out-of-range gene indices or column pointers set bad[0] and produce key 0
__global__ void csc_keys_kernel(const int64_t* colptr, const int32_t* rowidx, int64_t n, int64_t G,
                                int64_t nnz, int64_t* keys, int32_t* bad) {
    int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (c >= n) return;
    const int64_t e0 = colptr[c], e1 = colptr[c + 1];
    if (e0 < 0 || e1 < e0 || e1 > nnz) {
        if (lane == 0) atomicOr(bad, 1);
        return;
    }
    for (int64_t e = e0 + lane; e < e1; e += 32) {
        int32_t g = rowidx[e];
        if (g < 0 || g >= G) {
            atomicOr(bad, 1);
            keys[e] = 0;
        } else {
            keys[e] = (int64_t)g * n + c;
        }
    }
}
cudaError_t launch_csc_keys(const int64_t* colptr, const int32_t* rowidx, int64_t n, int64_t G,
                            int64_t nnz, int64_t* keys, int32_t* bad, cudaStream_t st) {
    if (n == 0 || nnz == 0) return cudaSuccess;
    csc_keys_kernel<<<nblk(n, 8), 256, 0, st>>>(colptr, rowidx, n, G, nnz, keys, bad);
    return cudaGetLastError();
}
__global__ void keys_to_csr_kernel(const int64_t* keys, int64_t nnz, int64_t n, int32_t* col,
                                   unsigned long long* rowcnt) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t k = keys[i];
        int64_t g = k / n;
        col[i] = (int32_t)(k - g * n);
        atomicAdd(rowcnt + g, 1ull);
    }
}
cudaError_t launch_keys_to_csr(const int64_t* keys, int64_t nnz, int64_t n, int64_t G,
                               int32_t* col, int64_t* rowcnt, cudaStream_t st) {
    (void)G;
    if (nnz == 0) return cudaSuccess;
    keys_to_csr_kernel<<<(unsigned)std::min<int64_t>(nblk(nnz, 256), 148 * 16), 256, 0, st>>>(
        keys, nnz, n, col, reinterpret_cast<unsigned long long*>(rowcnt));
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// design matrix: column-major doubles -> row-major padded floats
// ------------------------------------------------------------------
__global__ void x_rowmajor_kernel(const double* Xcm, int64_t n, int P, int xs, float* Xrm) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * xs;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t c = i / xs;
        int j = (int)(i - c * xs);
        Xrm[i] = j < P ? (float)Xcm[(int64_t)j * n + c] : 0.f;
    }
}
cudaError_t launch_x_rowmajor(const double* Xcm, int64_t n, int P, int xs, float* Xrm,
                              cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    x_rowmajor_kernel<<<(unsigned)std::min<int64_t>(nblk(n * xs, 256), 148 * 16), 256, 0, st>>>(
        Xcm, n, P, xs, Xrm);
    return cudaGetLastError();
}

__global__ void x_rowmajor_d_kernel(const double* Xcm, int64_t n, int P, int xs, double* Xrm) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * xs;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t c = i / xs;
        int j = (int)(i - c * xs);
        Xrm[i] = j < P ? Xcm[(int64_t)j * n + c] : 0.0;
    }
}
cudaError_t launch_x_rowmajor_d(const double* Xcm, int64_t n, int P, int xs, double* Xrm,
                                cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    x_rowmajor_d_kernel<<<(unsigned)std::min<int64_t>(nblk(n * xs, 256), 148 * 16), 256, 0, st>>>(
        Xcm, n, P, xs, Xrm);
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// per-gene statistics, two passes over each row (warp per gene):
// stats[g*6 + 0..5] = mean, sample variance (n-1), sum y,
//                     sum (y-1) y, max y, nnz
// ------------------------------------------------------------------
template <class VT>
__global__ void gene_stats_kernel(const int64_t* rowptr, const VT* val, int64_t G, int64_t n,
                                  double* stats, const int32_t* order) {
    int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (g >= G) return;
    if (order) g = order[g];
    const int64_t e0 = rowptr[g], e1 = rowptr[g + 1];
    // Counts that are whole numbers (always for uint16; checked for float):
    // one pass with exact integer sums of y and y^2 (below 2^64 for any int32
    // cell count and counts below 2^16) and the variance from the exact
    // numerator n sum y^2 - (sum y)^2 in 128 bits, so a uint16 and a float
    // copy of the same counts give the same statistics.  Other float counts:
    // a second pass over the squared deviations in FP64.
    unsigned long long s1 = 0, s2 = 0;
    double s = 0.0, mx = 0.0;
    bool whole = true;
    constexpr int U = 4;  // loads in flight per lane
    for (int64_t base = e0 + lane; base < e1; base += 32 * U) {
        VT raw[U];
#pragma unroll
        for (int u = 0; u < U; ++u) raw[u] = base + 32 * u < e1 ? __ldg(val + base + 32 * u) : VT(0);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const double y = (double)raw[u];
            s += y;
            mx = fmax(mx, y);
            if constexpr (std::is_same<VT, uint16_t>::value) {
                const unsigned long long v = (unsigned long long)raw[u];
                s1 += v;
                s2 += v * v;
            } else {
                const bool w = y >= 0.0 && y < 65536.0 && y == floor(y);
                whole = whole && w;
                if (w) {
                    const unsigned long long v = (unsigned long long)y;
                    s1 += v;
                    s2 += v * v;
                }
            }
        }
    }
    whole = __all_sync(0xffffffffu, whole);
    double* o = stats + g * 6;
    if (whole) {
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) {
            s1 += __shfl_xor_sync(0xffffffffu, s1, sh);
            s2 += __shfl_xor_sync(0xffffffffu, s2, sh);
        }
        mx = warp_max(mx);
        if (lane == 0) {
            const __int128 num = (__int128)n * (__int128)s2 - (__int128)s1 * (__int128)s1;
            o[0] = (double)s1 / (double)n;
            o[1] = (double)num / ((double)n * (double)(n - 1));
            o[2] = (double)s1;
            o[3] = (double)(s2 - s1);
            o[4] = mx;
            o[5] = (double)(e1 - e0);
        }
        return;
    }
    double sp = 0.0;
    for (int64_t e = e0 + lane; e < e1; e += 32) {
        const double y = (double)val[e];
        sp += (y - 1.0) * y;
    }
    s = warp_sum(s);
    sp = warp_sum(sp);
    mx = warp_max(mx);
    const double mean = s / (double)n;
    double ss = 0.0;
    for (int64_t e = e0 + lane; e < e1; e += 32) {
        const double d = (double)val[e] - mean;
        ss += d * d;
    }
    ss = warp_sum(ss);
    if (lane == 0) {
        ss += (double)(n - (e1 - e0)) * mean * mean;
        o[0] = mean;
        o[1] = ss / (double)(n - 1);
        o[2] = s;
        o[3] = sp;
        o[4] = mx;
        o[5] = (double)(e1 - e0);
    }
}
// The same statistics for uint16 counts whose array starts on a 16-byte
// boundary: warp per gene, the row read as 16-byte pieces of eight counts
// (four pieces in flight per lane), pieces that straddle the row's ends
// masked, the last piece of the array (which may end past nnz) read count
// by count.  Exact integer sums, as above.
__global__ void gene_stats_u16v_kernel(const int64_t* rowptr, const uint16_t* val, int64_t G, int64_t n,
                                       double* stats, const int32_t* order) {
    int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (g >= G) return;
    if (order) g = order[g];
    const int64_t e0 = rowptr[g], e1 = rowptr[g + 1], nnz = rowptr[G];
    const int64_t p0 = e0 >> 3, p1 = (e1 + 7) >> 3, pfull = nnz >> 3;
    const uint4* v4 = reinterpret_cast<const uint4*>(val);
    unsigned long long s1 = 0, s2 = 0;
    unsigned mx = 0;
    constexpr int U = 4;
    for (int64_t base = p0 + lane; base < p1; base += 32 * U) {
        uint4 pc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t pp = base + 32 * u;
            pc[u] = make_uint4(0, 0, 0, 0);
            if (pp < p1) {
                if (pp < pfull) {
                    pc[u] = __ldg(v4 + pp);
                } else {
                    uint16_t h[8];
#pragma unroll
                    for (int r = 0; r < 8; ++r) h[r] = pp * 8 + r < nnz ? val[pp * 8 + r] : (uint16_t)0;
                    pc[u] = make_uint4(h[0] | (unsigned)h[1] << 16, h[2] | (unsigned)h[3] << 16,
                                       h[4] | (unsigned)h[5] << 16, h[6] | (unsigned)h[7] << 16);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t pp = base + 32 * u;
            if (pp >= p1) continue;
            const int64_t ea = pp * 8;
            const unsigned w[4] = {pc[u].x, pc[u].y, pc[u].z, pc[u].w};
            const bool whole = ea >= e0 && ea + 8 <= e1;
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const unsigned y = (w[r >> 1] >> (16 * (r & 1))) & 0xffffu;
                if (whole || (ea + r >= e0 && ea + r < e1)) {
                    s1 += y;
                    s2 += (unsigned long long)(y * y);
                    mx = max(mx, y);
                }
            }
        }
    }
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, sh);
        s2 += __shfl_xor_sync(0xffffffffu, s2, sh);
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, sh));
    }
    if (lane == 0) {
        double* o = stats + g * 6;
        const __int128 num = (__int128)n * (__int128)s2 - (__int128)s1 * (__int128)s1;
        o[0] = (double)s1 / (double)n;
        o[1] = (double)num / ((double)n * (double)(n - 1));
        o[2] = (double)s1;
        o[3] = (double)(s2 - s1);
        o[4] = (double)mx;
        o[5] = (double)(e1 - e0);
    }
}

cudaError_t launch_gene_stats(const int64_t* rowptr, const void* val, int val_u16, int64_t G,
                              int64_t n, double* stats, cudaStream_t st, const int32_t* order) {
    if (G == 0) return cudaSuccess;
    if (val_u16 && (reinterpret_cast<uintptr_t>(val) & 15) == 0)
        gene_stats_u16v_kernel<<<nblk(G, 8), 256, 0, st>>>(rowptr, (const uint16_t*)val, G, n, stats, order);
    else if (val_u16)
        gene_stats_kernel<uint16_t><<<nblk(G, 8), 256, 0, st>>>(rowptr, (const uint16_t*)val, G, n, stats, order);
    else
        gene_stats_kernel<float><<<nblk(G, 8), 256, 0, st>>>(rowptr, (const float*)val, G, n, stats, order);
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// column statistics for size factors (atomics; integer-valued sums are
// exact in FP64 whatever the order)
// ------------------------------------------------------------------
template <class VT>
__global__ void colstats_kernel(const int32_t* col, const VT* val, int64_t nnz, double* colsum,
                                double* collog, int32_t* colcnt, int32_t* colmin_bits) {
    if (!collog) {
        // normed_sum: column sums only; four entries' loads in flight per thread
        constexpr int U = 4;
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e0 < nnz; e0 += stride * U) {
            int c[U];
            float v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t e = e0 + stride * u;
                c[u] = e < nnz ? __ldg(col + e) : -1;
                v[u] = e < nnz ? (float)val[e] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (c[u] >= 0) atomicAdd(colsum + c[u], (double)v[u]);
        }
        return;
    }
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        int c = col[e];
        float v = (float)val[e];
        atomicAdd(colsum + c, (double)v);
        if (collog) {
            atomicAdd(collog + c, log1p((double)v));
            atomicAdd(colcnt + c, 1);
            float l = (float)log1p((double)v);
            // log1p of counts is >= 0; int ordering of non-negative floats
            // matches float ordering
            atomicMin(colmin_bits + c, __float_as_int(fmaxf(l, 0.f)));
        }
    }
}
// normed_sum column sums of 16-bit counts as 32-bit integer atomics (a
// column sum is at most G x 65535, below 2^32 for G <= 65537), four entries'
// loads in flight per thread; colsum_from_u32_kernel turns them into FP64
// (the same exact integers the FP64 atomics give)
__global__ void colsum_u32_kernel(const int32_t* col, const uint16_t* val, int64_t nnz, uint32_t* colsum) {
    constexpr int U = 4;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e0 < nnz; e0 += stride * U) {
        int c[U];
        uint32_t v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t e = e0 + stride * u;
            c[u] = e < nnz ? __ldg(col + e) : -1;
            v[u] = e < nnz ? (uint32_t)__ldg(val + e) : 0u;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (c[u] >= 0 && v[u]) atomicAdd(colsum + c[u], v[u]);
    }
}
__global__ void colsum_from_u32_kernel(const uint32_t* in, int64_t n, double* out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

cudaError_t launch_colstats(const int64_t* rowptr, const int32_t* col, const void* val,
                            int val_u16, int64_t G, int64_t nnz, double* colsum,
                            double* collog, int32_t* colcnt, int32_t* colmin_bits,
                            cudaStream_t st, uint32_t* colsum_u32, int64_t n) {
    (void)rowptr;
    if (nnz == 0) return cudaSuccess;
    unsigned b = (unsigned)std::min<int64_t>(nblk(nnz, 256), 148 * 32);
    if (colsum_u32 && val_u16 && !collog && G <= 65537) {
        colsum_u32_kernel<<<b, 256, 0, st>>>(col, (const uint16_t*)val, nnz, colsum_u32);
        colsum_from_u32_kernel<<<(unsigned)std::min<int64_t>(nblk(n, 256), 1024), 256, 0, st>>>(colsum_u32, n,
                                                                                               colsum);
        return cudaGetLastError();
    }
    if (val_u16)
        colstats_kernel<uint16_t><<<b, 256, 0, st>>>(col, (const uint16_t*)val, nnz, colsum, collog, colcnt, colmin_bits);
    else
        colstats_kernel<float><<<b, 256, 0, st>>>(col, (const float*)val, nnz, colsum, collog, colcnt, colmin_bits);
    return cudaGetLastError();
}

// size factors from the column statistics; one block.
// method 1 = normed_sum (R/size_factors.R:75-88), 2 = psinorm (:100-117).
__global__ void sf_finalize_kernel(int method, int64_t G, int64_t n, const double* colsum,
                                   const double* collog, const int32_t* colcnt,
                                   const int32_t* colmin_bits, double offset, double* sf,
                                   double* off, float* off_f, int32_t* err) {
    __shared__ double red[32];
    __shared__ double red2[32];
    __shared__ double gm_s;
    double acc = 0.0, cntv = 0.0;
    int zero = 0;
    for (int64_t c = threadIdx.x; c < n; c += blockDim.x) {
        double v;
        if (G <= 1) {
            v = 1.0;
        } else if (method == 1) {
            v = colsum[c];
            if (v == 0.0) zero = 1;
        } else {
            double m = colcnt[c] < G ? 0.0 : (double)__int_as_float(colmin_bits[c]);
            v = collog[c] / (double)G - m;
        }
        sf[c] = v;
        double l = log(v);
        if (!isnan(l)) { acc += l; cntv += 1.0; }
    }
    zero = __syncthreads_or(zero);
    acc = warp_sum(acc);
    cntv = warp_sum(cntv);
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = acc; red2[threadIdx.x >> 5] = cntv; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0, k = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { s += red[w]; k += red2[w]; }
        gm_s = (G <= 1) ? 1.0 : exp(s / k);
        if (err) *err = (method == 1 && zero && G > 1) ? 1 : 0;
    }
    __syncthreads();
    const double gm = gm_s;
    for (int64_t c = threadIdx.x; c < n; c += blockDim.x) {
        double v = (G <= 1) ? 1.0 : sf[c] / gm;
        sf[c] = v;
        double o = offset + log(v);
        off[c] = o;
        off_f[c] = (float)o;
    }
}
cudaError_t launch_sf_finalize(int method, int64_t G, int64_t n, const double* colsum,
                               const double* collog, const int32_t* colcnt,
                               const int32_t* colmin_bits, double offset, double* sf,
                               double* off, float* off_f, int32_t* err, cudaStream_t st) {
    sf_finalize_kernel<<<1, 1024, 0, st>>>(method, G, n, colsum, collog, colcnt, colmin_bits,
                                           offset, sf, off, off_f, err);
    return cudaGetLastError();
}

// offsets from given (or unit) size factors: compute_offset_vector
// (R/size_factors.R:172-184)
__global__ void sf_given_kernel(const double* sf_in, int64_t n, double offset, int use_sf,
                                double* sf, double* off, float* off_f) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        double s = use_sf ? sf_in[c] : 1.0;
        sf[c] = s;
        double o = use_sf ? offset + log(s) : offset;
        off[c] = o;
        off_f[c] = (float)o;
    }
}
cudaError_t launch_sf_given(const double* sf_in, int64_t n, double offset, int use_sf, double* sf,
                            double* off, float* off_f, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    sf_given_kernel<<<(unsigned)std::min<int64_t>(nblk(n, 256), 1024), 256, 0, st>>>(
        sf_in, n, offset, use_sf, sf, off, off_f);
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// theta_0 = (var - mean / mean(exp(off))) / mean^2, NaN or < 0 -> 0.01
// (R/overdispersion.R:129-135); k = 1/theta_0 as the float beta_fit keeps
// (src/beta.cpp:25-28: theta_0 arrives as float, 1.0/k stored as float).
// ------------------------------------------------------------------
__global__ void theta0_kernel(const double* stats, const double* off, int64_t G, int64_t n,
                              int has_init, double init_value, double* theta0, float* k) {
    __shared__ double red[32];
    __shared__ double moi_s;
    double acc = 0.0;
    for (int64_t c = threadIdx.x; c < n; c += blockDim.x) acc += exp(off[c]);
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        moi_s = 1.0 / (s / (double)n);
    }
    __syncthreads();
    const double moi = moi_s;
    for (int64_t g = threadIdx.x; g < G; g += blockDim.x) {
        double th;
        if (has_init) {
            th = init_value;
        } else {
            double mean = stats[g * 6 + 0], var = stats[g * 6 + 1];
            double d = (var - moi * mean) / (mean * mean);
            th = (isnan(d) || d < 0.0) ? 0.01 : d;
        }
        theta0[g] = th;
        float kf = (float)th;
        k[g] = (float)(1.0 / (double)kf);
    }
}
cudaError_t launch_theta0(const double* stats, const double* off, int64_t G, int64_t n,
                          int has_init, double init_value, double* theta0, float* k,
                          cudaStream_t st) {
    theta0_kernel<<<1, 1024, 0, st>>>(stats, off, G, n, has_init, init_value, theta0, k);
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// (X'X)^-1 in FP64 (one block): the least-squares solve of init_beta
// ------------------------------------------------------------------
// partial X'X over the cells of one block (kXtxCells cells, staged in
// shared memory 256 at a time, row stride P+1); thread t owns packed
// pairs t, t + 256, ...
constexpr int kXtxCells = 8192;
constexpr int kXtxStage = 256;
__global__ void __launch_bounds__(256) xtx_partial_kernel(const double* Xcm, int64_t n, int P,
                                                          double* part) {
    extern __shared__ double xs[];  // [kXtxStage][P + 1]
    const int NP = P * (P + 1) / 2;
    const int RS = P + 1;
    const int64_t c0 = (int64_t)blockIdx.x * kXtxCells;
    const int64_t c1 = c0 + kXtxCells < n ? c0 + kXtxCells : n;
    double acc[3] = {0.0, 0.0, 0.0};  // NP <= 528 = 256 * 3 (rounded up)
    int pi[3], pj[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int q = threadIdx.x + k * 256;
        int j = 0;
        while ((j + 1) * (j + 2) / 2 <= q) ++j;
        pi[k] = q < NP ? q - j * (j + 1) / 2 : 0;
        pj[k] = q < NP ? j : 0;
    }
    for (int64_t cb = c0; cb < c1; cb += kXtxStage) {
        const int nc = (int)(c1 - cb < kXtxStage ? c1 - cb : kXtxStage);
        __syncthreads();
        for (int i = threadIdx.x; i < nc * P; i += blockDim.x) {
            const int col = i / nc, c = i - col * nc;  // coalesced along cells
            xs[c * RS + col] = Xcm[(int64_t)col * n + cb + c];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (threadIdx.x + k * 256 >= NP) break;
            double s = 0.0;
            for (int c = 0; c < nc; ++c) s = fma(xs[c * RS + pi[k]], xs[c * RS + pj[k]], s);
            acc[k] += s;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int q = threadIdx.x + k * 256;
        if (q < NP) part[(int64_t)blockIdx.x * NP + q] = acc[k];
    }
}

// sum the partials in block order (deterministic), then invert with LU;
// rank check on the pivots relative to the largest diagonal
__global__ void xtx_finish_kernel(const double* part, int nb, int P, double* ginv, int32_t* err) {
    extern __shared__ double sh[];
    double* Gm = sh;         // P*P
    double* W = sh + P * P;  // P*P
    int* piv = reinterpret_cast<int*>(W + P * P);
    const int NP = P * (P + 1) / 2;
    for (int q = threadIdx.x; q < NP; q += blockDim.x) {
        int j = 0;
        while ((j + 1) * (j + 2) / 2 <= q) ++j;
        const int i = q - j * (j + 1) / 2;
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += part[(int64_t)b * NP + q];
        Gm[j * P + i] = s;
        Gm[i * P + j] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double dmax = 0.0;
        for (int i = 0; i < P; ++i) dmax = fmax(dmax, fabs(Gm[i * P + i]));
        bool ok = lu_factor(P, Gm, piv);
        for (int i = 0; i < P; ++i)
            if (!(fabs(Gm[i * P + i]) > 1e-12 * dmax)) ok = false;
        if (ok) lu_inverse(P, Gm, piv, W);
        for (int i = 0; i < P * P; ++i) ginv[i] = ok ? W[i] : NAN;
        *err = ok ? 0 : 1;
    }
}

int xtx_blocks(int64_t n) { return (int)((n + kXtxCells - 1) / kXtxCells); }

// (X'X)^-1 in FP64 for the least-squares solve of init_beta: partial
// sums over cell blocks on every SM, then one block sums and inverts
cudaError_t launch_xtx_inverse(const double* Xcm, int64_t n, int P, double* part, double* ginv,
                               int32_t* err, cudaStream_t st) {
    const int nb = xtx_blocks(n);
    const size_t sm1 = (size_t)kXtxStage * (P + 1) * sizeof(double);
    cudaError_t e = raise_dyn_smem(xtx_partial_kernel, sm1);
    if (e != cudaSuccess) return e;
    xtx_partial_kernel<<<nb, 256, sm1, st>>>(Xcm, n, P, part);
    const size_t sm2 = (size_t)2 * P * P * 8 + (size_t)P * 4 + 16;
    xtx_finish_kernel<<<1, 256, sm2, st>>>(part, nb, P, ginv, err);
    return cudaGetLastError();
}

// beta_0 (warp per gene).  QR least squares of log1p(y / exp(off)) on X:
// the solution equals (X'X)^-1 X' z; z is zero wherever y is zero, so
// X' z is a sum over the nonzero entries of the row.  Rough init:
// beta_0 = (log1p(mean y), 0, ..., 0).
template <class VT, int PMAX>
__global__ void init_beta_kernel(const int64_t* rowptr, const int32_t* col, const VT* val,
                                 const double* Xrm, int xs, const double* inv_sf,
                                 const double* ginv, const double* stats, int64_t G, int64_t n,
                                 int P, int rough, double* beta, float* beta_f) {
    int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (g >= G) return;
    if (rough) {
        if (lane < P) {
            double b = lane == 0 ? log1p(stats[g * 6 + 0]) : 0.0;
            beta[g * P + lane] = b;
            beta_f[g * P + lane] = (float)b;
        }
        return;
    }
    double r[PMAX];
#pragma unroll
    for (int i = 0; i < PMAX; ++i) r[i] = 0.0;
    for (int64_t e = rowptr[g] + lane; e < rowptr[g + 1]; e += 32) {
        int c = col[e];
        double z = log1p((double)val[e] * inv_sf[c]);
        const double* xr = Xrm + (int64_t)c * xs;
#pragma unroll
        for (int i = 0; i < PMAX; ++i)
            if (i < P) r[i] += xr[i] * z;
    }
#pragma unroll
    for (int i = 0; i < PMAX; ++i)
        if (i < P) r[i] = warp_sum(r[i]);
    if (lane < P) {
        double b = 0.0;
#pragma unroll
        for (int j = 0; j < PMAX; ++j)
            if (j < P) b += ginv[j * P + lane] * r[j];
        beta[g * P + lane] = b;
        beta_f[g * P + lane] = (float)b;
    }
}
__global__ void inv_exp_kernel(const double* off, int64_t n, double* out) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x)
        out[c] = exp(-off[c]);
}
// z = log1p(y / exp(off)) as in R/beta.R:18; y * exp(-off) differs from
// y / exp(off) by at most an ulp of the quotient
cudaError_t launch_init_beta(const int64_t* rowptr, const int32_t* col, const void* val,
                             int val_u16, const double* Xrm, int xs, const double* off,
                             double* inv_sf, const double* ginv, const double* stats, int64_t G,
                             int64_t n, int P, int rough, double* beta, float* beta_f,
                             cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    if (!rough) {
        inv_exp_kernel<<<(unsigned)std::min<int64_t>(nblk(n, 256), 1024), 256, 0, st>>>(off, n, inv_sf);
    }
    const unsigned b = nblk(G, 8);
#define DEVIL_INIT(PM)                                                                          \
    if (val_u16)                                                                                 \
        init_beta_kernel<uint16_t, PM><<<b, 256, 0, st>>>(rowptr, col, (const uint16_t*)val, Xrm, \
                                                            xs, inv_sf, ginv, stats, G, n, P,     \
                                                            rough, beta, beta_f);                \
    else                                                                                         \
        init_beta_kernel<float, PM><<<b, 256, 0, st>>>(rowptr, col, (const float*)val, Xrm, xs,   \
                                                         inv_sf, ginv, stats, G, n, P, rough,     \
                                                         beta, beta_f);
    if (P <= 4) {
        DEVIL_INIT(4)
    } else if (P <= 8) {
        DEVIL_INIT(8)
    } else if (P <= 16) {
        DEVIL_INIT(16)
    } else {
        DEVIL_INIT(32)
    }
#undef DEVIL_INIT
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// segptr[g][b] = first CSR entry of row g with col >= bound[b]
// (warp per gene, lanes search boundaries in parallel)
// ------------------------------------------------------------------
__global__ void segptr_kernel(const int64_t* rowptr, const int32_t* col, int64_t G,
                              const int32_t* bound, int nbound, int64_t* segptr) {
    int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (g >= G) return;
    const int64_t e0 = rowptr[g], e1 = rowptr[g + 1];
    for (int b = lane; b < nbound; b += 32) {
        int32_t key = bound[b];
        int64_t lo = e0, hi = e1;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (col[mid] < key) lo = mid + 1; else hi = mid;
        }
        segptr[g * nbound + b] = lo;
    }
}
cudaError_t launch_segptr(const int64_t* rowptr, const int32_t* col, int64_t G,
                          const int32_t* bound, int nbound, int64_t* segptr, cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    segptr_kernel<<<nblk(G, 8), 256, 0, st>>>(rowptr, col, G, bound, nbound, segptr);
    return cudaGetLastError();
}

// CSR sanity (warp per gene): rowptr non-decreasing, cell indices in
// [0, n) and strictly increasing within each row.  bad[0] != 0 on failure.
__global__ void validate_csr_kernel(const int64_t* rowptr, const int32_t* col, int64_t G, int64_t n,
                                    int64_t nnz, int32_t* bad, const int32_t* order) {
    int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (g >= G) return;
    if (order) g = order[g];
    const int64_t e0 = rowptr[g], e1 = rowptr[g + 1];
    int b = 0;
    if (e0 < 0 || e1 < e0 || e1 > nnz) {
        b = 1;
    } else {
        for (int64_t e = e0 + lane; e < e1; e += 32) {
            int c = col[e];
            if (c < 0 || c >= n) b = 1;
            if (e > e0 && col[e - 1] >= c) b = 1;
        }
    }
    b = __any_sync(0xffffffffu, b);
    if (lane == 0 && b) atomicOr(bad, 1);
    if (g == G - 1 && lane == 0 && e1 != nnz) atomicOr(bad, 1);
}
// The same checks for a cell-index array that starts on a 16-byte boundary:
// the row read as 16-byte pieces of four indices (four in flight per lane),
// each index compared with the one before it in the row (the previous
// piece's last index comes from the lane before, or from the previous
// round's last lane); the array's last piece, which may end past nnz, is
// read index by index.
__global__ void validate_csr_v_kernel(const int64_t* rowptr, const int32_t* col, int64_t G, int64_t n,
                                      int64_t nnz, int32_t* bad, const int32_t* order) {
    int64_t g = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (g >= G) return;
    if (order) g = order[g];
    const int64_t e0 = rowptr[g], e1 = rowptr[g + 1];
    int b = 0;
    if (e0 < 0 || e1 < e0 || e1 > nnz) {
        b = 1;
    } else {
        const int64_t p0 = e0 >> 2, p1 = (e1 + 3) >> 2, pfull = nnz >> 2;
        const int4* c4 = reinterpret_cast<const int4*>(col);
        constexpr int U = 4;
        int carry = -1;  // the last index of the previous round (-1: none; indices are >= 0)
        for (int64_t base = p0; base < p1; base += 32 * U) {
            int4 pc[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t pp = base + 32 * u + lane;
                pc[u] = make_int4(-1, -1, -1, -1);
                if (pp < p1) {
                    if (pp < pfull) {
                        pc[u] = __ldg(c4 + pp);
                    } else {
                        int h[4];
#pragma unroll
                        for (int r = 0; r < 4; ++r) h[r] = pp * 4 + r < nnz ? col[pp * 4 + r] : -1;
                        pc[u] = make_int4(h[0], h[1], h[2], h[3]);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int64_t pp = base + 32 * u + lane;
                // the index before this piece: the previous lane's last, or
                // (lane 0) the last of round u - 1, or of the previous round
                int before = __shfl_up_sync(0xffffffffu, pc[u].w, 1);
                const int last_prev = u > 0 ? __shfl_sync(0xffffffffu, pc[u > 0 ? u - 1 : 0].w, 31) : carry;
                if (lane == 0) before = last_prev;
                if (pp < p1) {
                    const int c[4] = {pc[u].x, pc[u].y, pc[u].z, pc[u].w};
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const int64_t e = pp * 4 + r;
                        if (e >= e0 && e < e1) {
                            if (c[r] < 0 || c[r] >= n) b = 1;
                            const int prv = r == 0 ? before : c[r - 1];
                            if (e > e0 && prv >= c[r]) b = 1;
                        }
                    }
                }
            }
            carry = __shfl_sync(0xffffffffu, pc[U - 1].w, 31);
        }
    }
    b = __any_sync(0xffffffffu, b);
    if (lane == 0 && b) atomicOr(bad, 1);
    if (g == G - 1 && lane == 0 && e1 != nnz) atomicOr(bad, 1);
}
cudaError_t launch_validate_csr(const int64_t* rowptr, const int32_t* col, int64_t G, int64_t n,
                                int64_t nnz, int32_t* bad, cudaStream_t st, const int32_t* order) {
    if (G == 0) return cudaSuccess;
    if ((reinterpret_cast<uintptr_t>(col) & 15) == 0)
        validate_csr_v_kernel<<<nblk(G, 8), 256, 0, st>>>(rowptr, col, G, n, nnz, bad, order);
    else
        validate_csr_kernel<<<nblk(G, 8), 256, 0, st>>>(rowptr, col, G, n, nnz, bad, order);
    return cudaGetLastError();
}

// acc[0] += sum_g passes[g] * nnz_g, acc[1] += sum_g passes[g]
__global__ void pass_volume_kernel(const int64_t* rowptr, const int32_t* passes, int64_t G,
                                   long long* acc) {
    long long v = 0, w = 0;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G;
         g += (int64_t)gridDim.x * blockDim.x) {
        long long k = passes[g];
        v += k * (long long)(rowptr[g + 1] - rowptr[g]);
        w += k;
    }
    v = warp_sum(v);
    w = warp_sum(w);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(acc), (unsigned long long)v);
        atomicAdd(reinterpret_cast<unsigned long long*>(acc + 1), (unsigned long long)w);
    }
}
cudaError_t launch_pass_volume(const int64_t* rowptr, const int32_t* passes, int64_t G,
                               int64_t* acc, cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    pass_volume_kernel<<<(unsigned)std::min<int64_t>(nblk(G, 256), 256), 256, 0, st>>>(
        rowptr, passes, G, reinterpret_cast<long long*>(acc));
    return cudaGetLastError();
}
__global__ void fill_i32_kernel(int32_t* a, int32_t v, int64_t m) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}
cudaError_t launch_fill_i32(int32_t* a, int32_t v, int64_t m, cudaStream_t st) {
    if (m == 0) return cudaSuccess;
    fill_i32_kernel<<<(unsigned)std::min<int64_t>(nblk(m, 256), 1024), 256, 0, st>>>(a, v, m);
    return cudaGetLastError();
}
// MLE passes per gene: 0 for all-zero genes, else the far-left evaluation
// plus the Newton evaluations
__global__ void mle_passes_kernel(const int32_t* it, const int32_t* phase, const double* stats,
                                  int64_t G, int32_t* out) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G;
         g += (int64_t)gridDim.x * blockDim.x)
        out[g] = stats[g * 6 + 2] == 0.0 ? 0 : 1 + it[g];
}
cudaError_t launch_mle_passes(const int32_t* it, const int32_t* phase, const double* stats,
                              int64_t G, int32_t* out, cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    mle_passes_kernel<<<(unsigned)std::min<int64_t>(nblk(G, 256), 1024), 256, 0, st>>>(it, phase, stats, G, out);
    return cudaGetLastError();
}

__global__ void iota_kernel(int32_t* a, int64_t m) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        a[i] = (int32_t)i;
}
cudaError_t launch_iota(int32_t* a, int64_t m, cudaStream_t st) {
    if (m == 0) return cudaSuccess;
    iota_kernel<<<(unsigned)std::min<int64_t>(nblk(m, 256), 1024), 256, 0, st>>>(a, m);
    return cudaGetLastError();
}
// act_next = the genes of act[0, n) with keep[g] != 0, in their order in
// act; *n_next = their count.  Keeping the order keeps a list sorted by work
// sorted from one iteration to the next.  One block; per batch every thread
// loads kCompactR elements strided by the block size (coalesced, all loads
// in flight), the kept ones are placed by warp ballots and one scan of the
// (round, warp) totals.
constexpr int kCompactNT = 1024, kCompactR = 16;
__global__ void __launch_bounds__(kCompactNT) compact_kept_kernel(const int32_t* act, const int32_t* n_act,
                                                                  int64_t n_fixed, const int8_t* keep,
                                                                  int32_t* act_next, int32_t* n_next,
                                                                  const int32_t* wkey, int32_t thr,
                                                                  int32_t* n_heavy_next,
                                                                  volatile int32_t* mirror) {
    __shared__ int wtot[kCompactR][32];
    __shared__ int batch_total;
    const int64_t n = n_act ? (int64_t)*n_act : n_fixed;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned lt = (1u << lane) - 1u;
    int base = 0, heavy = 0;
    for (int64_t c0 = 0; c0 < n; c0 += (int64_t)kCompactNT * kCompactR) {
        int32_t g[kCompactR];
        unsigned bal[kCompactR];
#pragma unroll
        for (int r = 0; r < kCompactR; ++r) {
            const int64_t i = c0 + (int64_t)r * kCompactNT + t;
            g[r] = i < n ? act[i] : -1;
        }
#pragma unroll
        for (int r = 0; r < kCompactR; ++r) {
            const bool f = g[r] >= 0 && keep[g[r]] != 0;
            bal[r] = __ballot_sync(0xffffffffu, f);
            if (f && wkey) heavy += wkey[g[r]] >= thr;
            if (lane == 0) wtot[r][w] = __popc(bal[r]);
        }
        __syncthreads();
        if (w == 0) {
            // lane r: the exclusive offsets of round r's warps, after the
            // rounds before it
            int v = 0;
            if (lane < kCompactR)
                for (int q = 0; q < 32; ++q) v += wtot[lane][q];
            int incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int x = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += x;
            }
            if (lane < kCompactR) {
                int run = incl - v;
                for (int q = 0; q < 32; ++q) {
                    const int c = wtot[lane][q];
                    wtot[lane][q] = run;
                    run += c;
                }
            }
            if (lane == 31) batch_total = incl;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kCompactR; ++r)
            if (bal[r] >> lane & 1u) act_next[base + wtot[r][w] + __popc(bal[r] & lt)] = g[r];
        base += batch_total;
        __syncthreads();  // wtot and batch_total are rewritten by the next batch
    }
    if (t == 0) {
        *n_next = base;
        if (mirror) *mirror = base;  // the host's copy (pinned, mapped)
    }
    if (wkey) {
        heavy = __reduce_add_sync(0xffffffffu, heavy);
        if (lane == 0) wtot[0][w] = heavy;
        __syncthreads();
        if (t == 0) {
            int h = 0;
            for (int q = 0; q < kCompactNT / 32; ++q) h += wtot[0][q];
            *n_heavy_next = h;
        }
    }
}
cudaError_t launch_compact_kept(const int32_t* act, const int32_t* n_act, int64_t n_fixed, const int8_t* keep,
                                int32_t* act_next, int32_t* n_next, cudaStream_t st, const int32_t* wkey,
                                int32_t thr, int32_t* n_heavy_next, volatile int32_t* mirror) {
    compact_kept_kernel<<<1, kCompactNT, 0, st>>>(act, n_act, n_fixed, keep, act_next, n_next, wkey, thr,
                                                  n_heavy_next, mirror);
    return cudaGetLastError();
}
// *out = the number of leading entries of key (descending) that are >= thr
__global__ void count_at_least_kernel(const int32_t* key, int64_t n, int32_t thr, int32_t* out) {
    int64_t lo = 0, hi = n;  // key[0, lo) >= thr, key[hi, n) < thr
    while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (key[mid] >= thr) lo = mid + 1; else hi = mid;
    }
    *out = (int32_t)lo;
}
cudaError_t launch_count_at_least(const int32_t* key, int64_t n, int32_t thr, int32_t* out, cudaStream_t st) {
    count_at_least_kernel<<<1, 1, 0, st>>>(key, n, thr, out);
    return cudaGetLastError();
}
__global__ void set_i32_kernel(int32_t* a, int32_t v) { *a = v; }
cudaError_t launch_set_i32(int32_t* a, int32_t v, cudaStream_t st) {
    set_i32_kernel<<<1, 1, 0, st>>>(a, v);
    return cudaGetLastError();
}
__global__ void mirror_kernel(const int32_t* src, volatile int32_t* dst) { *dst = *src; }
cudaError_t launch_copy_i32_to_host_mapped(const int32_t* src, volatile int32_t* dst,
                                           cudaStream_t st) {
    mirror_kernel<<<1, 1, 0, st>>>(src, dst);
    return cudaGetLastError();
}

}  // namespace devil
