// overdispersion = "new" / "I": fit_overdispersion_cppp
// (src/new_overdispersion.cpp:195-481).
//
// The reference searches k = 1/kappa for a fixed point of
//   F(k) = H(+1/2) / H(-1/2),  H(p) = int_0^inf x^p exp(n (x log x - lgamma x) - C1(k) x) dx,
//   C1(k) = sum_i x_i.beta - (sum_i psi(k + y_i) - sum_i log1p(k w_i)) + sum_i (k + y_i) w_i / (1 + k w_i),
// with w_i = exp(-(x_i.beta + o_i)), H by Laplace-centred Gauss-Hermite
// quadrature, and a safeguarded Aitken iteration with secant, bracketing
// and Brent fallbacks.  One warp per gene runs that search: its control
// flow depends only on warp-reduced values, so every lane takes the same
// path; each evaluation of C1 is a warp-parallel FP64 pass over the gene's
// cells (zero-count terms for all cells, corrections for the nonzeros).
// A gene that reaches one of the reference's stop() conditions records an
// error code; the host then fails the call with the reference's message.
#include "internal.h"

namespace devil {

namespace {

constexpr int kNodWarps = 4;  // genes per block

struct NodGene {
    const NodArgs* a;
    int64_t g;
    int lane;
    double xbs;       // sum_i x_i . beta
    const double* b;  // beta of the gene (shared memory)
    int err;          // 1: C1 <= n, 2: mode search, 3: quadrature underflow
};

DEV double nod_g(double s, double t, double x) { return s * (x * log(x) - lgamma(x)) - t * x; }
DEV double nod_g1(double s, double t, double x) { return s * (log(x) + 1.0 - digamma_d(x)) - t; }
DEV double nod_g2(double s, double x) { return s * (1.0 / x - trigamma_d(x)); }

// find_mode (src/new_overdispersion.cpp:71-97); false on failure
DEV bool nod_mode(double p, double s, double t, int max_newton, double tol, double x0,
                  double& mu0, double& sigma0, double& hmu0) {
    double x = x0 > 1e-9 ? x0 : 1e-9;
    for (int i = 0; i < max_newton; ++i) {
        const double g1v = p / x + nod_g1(s, t, x);
        if (fabs(g1v) < tol) break;
        const double g2v = -p / (x * x) + nod_g2(s, x);
        double xn = x - g1v / g2v;
        if (!(xn > 0.0) || !isfinite(xn)) xn = 0.5 * x;
        if (fabs(xn - x) < tol * (1.0 + fabs(x))) {
            x = xn;
            break;
        }
        x = xn;
    }
    const double curv = -(-p / (x * x) + nod_g2(s, x));
    if (!(curv > 0.0) || !isfinite(curv)) return false;
    mu0 = x > 1e-12 ? x : 1e-12;
    sigma0 = sqrt(1.0 / curv);
    hmu0 = p * log(mu0) + nod_g(s, t, mu0);
    return true;
}

// log_integral_at (src/new_overdispersion.cpp:99-126); false on underflow
DEV bool nod_log_integral(double p, double s, double t, const NodArgs& a, double mu0,
                          double sigma0, double hmu0, double& out) {
    const double scale = sigma0 * 1.4142135623730951;
    double mx = -INFINITY;
    for (int i = 0; i < a.gh_m; ++i) {
        const double u = a.gx[i], xx = mu0 + scale * u;
        if (xx <= 0.0 || !isfinite(xx)) continue;
        const double lt = log(a.gw[i]) + (p * log(xx) + nod_g(s, t, xx)) - hmu0 + u * u;
        if (lt > mx) mx = lt;
    }
    double acc = 0.0;
    for (int i = 0; i < a.gh_m; ++i) {
        const double u = a.gx[i], xx = mu0 + scale * u;
        if (xx <= 0.0 || !isfinite(xx)) continue;
        acc += exp(log(a.gw[i]) + (p * log(xx) + nod_g(s, t, xx)) - hmu0 + u * u - mx);
    }
    if (!(acc > 0.0)) return false;
    out = hmu0 + log(scale) + mx + log(acc);
    return true;
}

template <class VT>
DEV double nod_F(NodGene& G, double kk) {
    if (G.err) return NAN;
    const NodArgs& a = *G.a;
    const int P = a.P;
    double sl = 0.0, sm = 0.0, sd = 0.0;
    for (int64_t c = G.lane; c < a.n; c += 32) {
        double eta = a.off[c];
        for (int i = 0; i < P; ++i) eta = fma(a.Xd[c * a.xs + i], G.b[i], eta);
        const double w = exp(-eta), kw = kk * w;
        sl += log1p(kw);
        sm += kk * w / (1.0 + kw);
    }
    const VT* val = static_cast<const VT*>(a.val);
    const double dk = digamma_d(kk);
    const int64_t e0 = a.rowptr[G.g], e1 = a.rowptr[G.g + 1];
    for (int64_t e = e0 + G.lane; e < e1; e += 32) {
        const int c = a.col[e];
        const double y = (double)load_val(val, e);
        double eta = a.off[c];
        for (int i = 0; i < P; ++i) eta = fma(a.Xd[(int64_t)c * a.xs + i], G.b[i], eta);
        const double w = exp(-eta);
        sd += digamma_d(kk + y) - dk;
        sm += y * w / (1.0 + kk * w);
    }
    sl = warp_sum(sl);
    sm = warp_sum(sm);
    sd = warp_sum(sd);
    const double sn = (double)a.n;
    const double C1 = G.xbs - ((sn * dk + sd) - sl) + sm;
    if (!(C1 > sn)) {
        G.err = 1;
        return NAN;
    }
    double m1, s1, h1, m2, s2, h2, lp, lm;
    double x01 = (0.5 + sn) / (C1 - sn);
    if (x01 < 1e-3) x01 = 1e-3;
    if (!nod_mode(0.5, sn, C1, a.max_newton, a.eps, x01, m1, s1, h1) ||
        !nod_mode(-0.5, sn, C1, a.max_newton, a.eps, m1, m2, s2, h2)) {
        G.err = 2;
        return NAN;
    }
    if (!nod_log_integral(0.5, sn, C1, a, m1, s1, h1, lp) ||
        !nod_log_integral(-0.5, sn, C1, a, m2, s2, h2, lm)) {
        G.err = 3;
        return NAN;
    }
    return exp(lp - lm);
}

template <class VT>
DEV double nod_f(NodGene& G, double kk) { return log(nod_F<VT>(G, kk)) - log(kk); }

DEV double nod_clamp(double k) { return k < 1e-4 ? 1e-4 : (k > 1e4 ? 1e4 : k); }

// the reference's Brent search (src/new_overdispersion.cpp:343-373)
template <class VT>
DEV double nod_brent(NodGene& G, double a, double b, double fa, double fb) {
    double c = a, fc = fa, d = b - a, e = d;
    const double tol = G.a->eps, epsm = 2.220446049250313e-16;
    for (int it = 0; it < 60; ++it) {
        if (fabs(fc) < fabs(fb)) {
            a = b; b = c; c = a;
            fa = fb; fb = fc; fc = fa;
        }
        const double tol1 = 2.0 * epsm * fabs(b) + 0.5 * tol;
        const double xm = 0.5 * (c - b);
        if (fabs(xm) <= tol1 || fb == 0.0) return b;
        if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
            const double s = fb / fa;
            double p, q;
            if (a == c) {
                p = 2.0 * xm * s;
                q = 1.0 - s;
            } else {
                const double r = fb / fc, t = fa / fc;
                p = s * (2.0 * xm * t * (t - r) - (b - a) * (r - 1.0));
                q = (t - 1.0) * (r - 1.0) * (s - 1.0);
            }
            if (p > 0) q = -q;
            p = fabs(p);
            const double m1 = 3.0 * xm * q - fabs(tol1 * q), m2 = fabs(e * q);
            if (2.0 * p < (m1 < m2 ? m1 : m2)) {
                e = d;
                d = p / q;
            } else {
                d = xm;
                e = d;
            }
        } else {
            d = xm;
            e = d;
        }
        a = b;
        fa = fb;
        b += (fabs(d) > tol1 ? d : (xm > 0 ? tol1 : -tol1));
        fb = nod_f<VT>(G, b);
        if ((fb > 0 && fc > 0) || (fb < 0 && fc < 0)) {
            c = a;
            fc = fa;
            e = d = b - a;
        }
    }
    return b;
}

template <class VT>
__global__ void __launch_bounds__(32 * kNodWarps) new_od_kernel(NodArgs a) {
    __shared__ double bsh[kNodWarps][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t g = (int64_t)blockIdx.x * kNodWarps + warp;
    if (g >= a.G) return;
    double* b = bsh[warp];
    if (lane < a.P) b[lane] = a.beta[g * a.P + lane];
    __syncwarp();
    NodGene G{&a, g, lane, 0.0, b, 0};
    for (int i = 0; i < a.P; ++i) G.xbs += a.xcolsum[i] * b[i];

    // moment start (src/new_overdispersion.cpp:225-254) from the raw counts
    const double ym = a.stats[g * 6 + 0], yv = a.stats[g * 6 + 1];
    double kap = (yv - ym) / (ym * ym);
    if (!isfinite(kap) || kap <= 0.0) kap = 0.01;
    double k = 1.0 / kap;
    if (!isfinite(k)) k = 1e-4;
    k = nod_clamp(k);
    const double kmin = 1e-4, jump = 10.0;
    int conv = 0, itk = 0, bad = 0;

    double k0 = nod_clamp(k), f0 = nod_f<VT>(G, k0);
    if (!isfinite(f0)) {
        if (lane == 0) {
            a.err[g] = G.err ? G.err : 4;
            a.theta[g] = NAN;
            a.iters[g] = 0;
        }
        return;
    }
    const double h = 1e-6 * k0 > 1e-8 ? 1e-6 * k0 : 1e-8;
    const double fp0 = (nod_f<VT>(G, k0 + h) - f0) / h;
    if (isfinite(fp0) && fabs(fp0) > 1e-10) {
        const double kn = nod_clamp(k0 - f0 / fp0), fn = nod_f<VT>(G, kn);
        if (isfinite(fn) && fabs(fn) < fabs(f0)) {
            k0 = kn;
            f0 = fn;
        }
    }
    double k1 = nod_F<VT>(G, k0);
    const double cap = jump * (k0 > 1.0 ? k0 : 1.0);
    if (k1 > cap) k1 = cap;
    k1 = nod_clamp(k1);
    double f1 = nod_f<VT>(G, k1);
    if (f0 * f1 < 0) {
        k = nod_brent<VT>(G, k0 < k1 ? k0 : k1, k0 < k1 ? k1 : k0, f0, f1);
        conv = 1;
    } else {
        for (itk = 0; itk < a.max_iter; ++itk) {
            const double aj = jump / (1.0 + 0.1 * itk);
            double k2 = nod_F<VT>(G, k1);
            const double c2 = aj * (k1 > 1.0 ? k1 : 1.0);
            if (k2 > c2) k2 = c2;
            k2 = nod_clamp(k2);
            const double f2 = nod_f<VT>(G, k2);
            const double d1 = k1 - k0, d2 = k2 - k1, den = d2 - d1;
            double ka = fabs(den) > 1e-14 ? k0 - d1 * d1 / den : k2;
            if (!(ka > 0) || !isfinite(ka)) ka = k2;
            const double c3 = aj * (k2 > 1.0 ? k2 : 1.0);
            if (ka > c3) ka = c3;
            ka = nod_clamp(ka);
            double kp = ka, fp = nod_f<VT>(G, kp);
            for (int bt = 0; (fabs(fp) >= fabs(f1) || !isfinite(fp)) && bt < 8; ++bt) {
                kp = 0.5 * (kp + k1);
                fp = nod_f<VT>(G, kp);
            }
            if (!(fabs(fp) < fabs(f1))) {
                ++bad;
                if (bad == 1 && fabs(f1 - f0) > 1e-14) {
                    const double ks = nod_clamp(k1 - f1 * (k1 - k0) / (f1 - f0));
                    const double fs = nod_f<VT>(G, ks);
                    if (isfinite(fs) && fabs(fs) < fabs(f1)) {
                        kp = ks;
                        fp = fs;
                        bad = 0;
                    }
                }
                if (bad >= 1 && f1 * f2 < 0) {
                    k = nod_brent<VT>(G, k1 < k2 ? k1 : k2, k1 < k2 ? k2 : k1, f1, f2);
                    conv = 1;
                    break;
                }
                if (bad >= 1) {
                    // find_bracket (src/new_overdispersion.cpp:324-339)
                    double lo = -1.0, hi = -1.0;
                    const double fc = nod_f<VT>(G, k1);
                    for (int ex = 1; ex <= 10; ++ex) {
                        const double fac = (double)(1 << ex);
                        const double l = k1 / fac > kmin ? k1 / fac : kmin;
                        const double u = k1 * fac < 1e4 ? k1 * fac : 1e4;
                        const double fl = nod_f<VT>(G, l);
                        if (fl * fc < 0) { lo = l; hi = k1; break; }
                        const double fu = nod_f<VT>(G, u);
                        if (fc * fu < 0) { lo = k1; hi = u; break; }
                        if (fl * fu < 0) { lo = l; hi = u; break; }
                    }
                    if (lo > 0) {
                        const double flo = nod_f<VT>(G, lo), fhi = nod_f<VT>(G, hi);
                        k = nod_brent<VT>(G, lo, hi, flo, fhi);
                        conv = 1;
                        break;
                    }
                }
                kp = k2;
                fp = f2;
            } else {
                bad = 0;
            }
            if (fabs(kp - k1) < a.eps * (1.0 + k1)) {
                k = kp;
                conv = 1;
                break;
            }
            k0 = k1; f0 = f1;
            k1 = kp; f1 = fp;
        }
        if (!conv) k = k1 > kmin ? k1 : kmin;
    }
    if (lane == 0) {
        a.err[g] = G.err;
        a.theta[g] = G.err ? NAN : 1.0 / k;
        a.iters[g] = itk + 1;
    }
}

__global__ void colsum_kernel(const double* Xcm, int64_t n, double* out) {
    __shared__ double red[32];
    const int j = blockIdx.x;
    double s = 0.0;
    for (int64_t c = threadIdx.x; c < n; c += blockDim.x) s += Xcm[(int64_t)j * n + c];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) out[j] = v;
    }
}

}  // namespace

cudaError_t launch_new_od(const NodArgs& a, const double* Xcm, double* xcolsum, cudaStream_t st) {
    if (a.G <= 0) return cudaSuccess;
    colsum_kernel<<<a.P, 256, 0, st>>>(Xcm, a.n, xcolsum);
    const unsigned grid = (unsigned)((a.G + kNodWarps - 1) / kNodWarps);
    if (a.val_u16)
        new_od_kernel<uint16_t><<<grid, 32 * kNodWarps, 0, st>>>(a);
    else
        new_od_kernel<float><<<grid, 32 * kNodWarps, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace devil
