// Overlap sign function as a Chebyshev polynomial (the fast form; FP32 or FP64).
//
// The reference approximates (h_W^2)^(-1/2) by a 25-pole Zolotarev rational
// function solved with a multi-shift CG (FERMIONS/OVERLAP/OPERATOR/OverlapU.cpp);
// here the same operator is a polynomial in X = h_W^2 / lambda_max:
//   (h_W^2)^(-1/2) ~ lambda_max^(-1/2) [c_0/2 + sum_{k=1..K} c_k T_k(t(X))],
//   t(X) = (2X - 1 - eps) / (1 - eps),
// the Chebyshev series of x^(-1/2) on [eps, 1].  Clenshaw's recurrence
//   b_k = 2 t(X) b_{k+1} - b_{k+2} + c_k phi,  y = t(X) b_1 - b_2 + c_0/2 phi
// needs one application of X per term, X b = -D(D b) / lambda_max with
// D = -i h_W.  Each term is two stencil launches: w = D b_{k+1}, then one
// kernel that applies D to w and forms b_k in its epilogue (reads w with its
// neighbours, b_{k+1}, b_{k+2}, phi; writes b_k).  The result
//   out = M [ -i g0 (1 + m/2) phi + (1 - m/2) D chi ],  chi = lambda_max^(-1/2) y
// is the reference's overlap evolution operator (OverlapU.cpp:188-202) with the
// Chebyshev approximation of the inverse square root; its error against the
// exact function is set by K and eps and is stated by the caller.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ovl_internal.h"
#include "ovl_stencil.cuh"

namespace ovl {

// Chebyshev coefficients of x^(-1/2) on [eps, 1] (first kind, c_0 counted
// with weight 1/2), by Chebyshev-Gauss quadrature on max(4K, 256) nodes.
void chebyshev_inverse_sqrt(int K, double eps, double *c) {
    const int M = std::max(4 * K, 256);
    std::vector<double> f(M), th(M);
    for (int j = 0; j < M; j++) {
        th[j] = M_PI * (j + 0.5) / M;
        const double x = 0.5 * (1.0 + eps) + 0.5 * (1.0 - eps) * std::cos(th[j]);
        f[j] = 1.0 / std::sqrt(x);
    }
    for (int k = 0; k <= K; k++) {
        double s = 0.0;
        for (int j = 0; j < M; j++) s += f[j] * std::cos(k * th[j]);
        c[k] = 2.0 * s / M;
    }
}

// The mode blocks of a CTA's row and the links its warps read.  TABLE (FP64):
// a CTA runs mblk mode blocks on its sites' links gathered once in shared
// memory (fill_link_table); otherwise one mode block with LK itself.  Every
// thread of the CTA calls body(links, site, mb) for each of its mode blocks.
template <typename T, bool TABLE, class LK, class Body>
__device__ __forceinline__ void cheb_blocks(const LK &lk, const Lattice &L, int n_mb, int mblk, Body &&body) {
    const int site = blockIdx.x * kSitesPerCta + threadIdx.y;
    if constexpr (TABLE) {
        static_assert(sizeof(T) == 8, "the link table holds FP64 matrices");
        __shared__ cmat2<double> tab[kSitesPerCta][6];
        const int site0 = blockIdx.x * kSitesPerCta;
        fill_link_table<kSitesPerCta>(lk, L, [&](int j) { return site0 + j < L.V ? site0 + j : -1; }, tab);
        if (site >= L.V) return;
        const LinksTable lt{tab[threadIdx.y], site};
        const int mb0 = blockIdx.y * mblk, mb1 = min(n_mb, mb0 + mblk);
        for (int mb = mb0; mb < mb1; mb++) body(lt, site, mb);
    } else {
        if (site >= L.V) return;
        body(lk, site, (int)blockIdx.y);
    }
}

// Launches K<TABLE> on the grid of n_mb mode blocks: in FP64 with mblk =
// link_blocks(...) mode blocks per CTA when that is more than one.
template <typename T, class Launch>
static void cheb_launch(const Lattice &L, int n_mb, Launch &&launch) {
    const int gx = (L.V + kSitesPerCta - 1) / kSitesPerCta;
    if constexpr (sizeof(T) == 8) {
        const int m = link_blocks(gx, n_mb, current_sm_count());
        if (m > 1) {
            launch(std::true_type{}, dim3(gx, (n_mb + m - 1) / m), m);
            return;
        }
    }
    launch(std::false_type{}, dim3(gx, n_mb), 1);
}

// w = D b (the first half of X = -D^2 / lambda_max), with the links of LK.
template <typename T, class LK, bool TABLE>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta)
    cheb_wilson_kernel(LK lk, const cpx<T> *__restrict__ b, cpx<T> *__restrict__ w, Lattice L, T amass, int n_mb,
                       int mblk) {
    const int lane = threadIdx.x;
    cheb_blocks<T, TABLE>(lk, L, n_mb, mblk, [&](const auto &links, int site, int mb) {
        Spinor<T> acc;
        wilson_site_lk(links, b, L, site, mb, lane, amass, acc);
        cpx<T> *o = w + field_index(L.V, mb, site, 0, lane);
#pragma unroll
        for (int c = 0; c < kColours; c++)
#pragma unroll
            for (int s = 0; s < kSpin; s++) st(o + (c * kSpin + s) * kModeBlock, finish_component(acc.c[c][s], s));
    });
}

// b_out = factor * (a * (-D w) + beta * b1) - b2 + ck * phi, per mode and site;
// -D w is the stencil applied to w (the second half of X = -D^2 / lambda_max).
template <typename T, class LK, bool TABLE>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta)
    clenshaw_kernel(LK lk, const cpx<T> *__restrict__ w, const cpx<T> *__restrict__ b1, const cpx<T> *__restrict__ b2,
                    const cpx<T> *__restrict__ phi, cpx<T> *__restrict__ bout, Lattice L, T amass, T a, T beta,
                    T factor, T ck, int n_mb, int mblk) {
    const int lane = threadIdx.x;
    cheb_blocks<T, TABLE>(lk, L, n_mb, mblk, [&](const auto &links, int site, int mb) {
        Spinor<T> acc;
        wilson_site_lk(links, w, L, site, mb, lane, amass, acc);
        const size_t base = field_index(L.V, mb, site, 0, lane);
#pragma unroll
        for (int c = 0; c < kColours; c++)
#pragma unroll
            for (int s = 0; s < kSpin; s++) {
                const size_t i = base + (c * kSpin + s) * kModeBlock;
                const cpx<T> dw = finish_component(acc.c[c][s], s);
                const cpx<T> v1 = ld(b1 + i), v2 = ld(b2 + i), f = ld(phi + i);
                const cpx<T> tx = mk<T>(-a * dw.re + beta * v1.re, -a * dw.im + beta * v1.im);
                st(bout + i, mk<T>(factor * tx.re - v2.re + ck * f.re, factor * tx.im - v2.im + ck * f.im));
            }
    });
}

// out = M [ -i g0 (1 + m/2) phi + (1 - m/2) dchi ];  dst = out or dst += dt out
template <typename T>
__global__ void overlap_finish_t_kernel(const cpx<T> *__restrict__ phi, const cpx<T> *__restrict__ dchi, cpx<T> *dst,
                                        size_t n, T mdw, T mf, T dt, int accumulate) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int spin = (int)((e / kModeBlock) % kComp) % kSpin;
        const cpx<T> f = ld(phi + e), d = ld(dchi + e);
        const T cp = (T)1 + (T)0.5 * mf, cm = (T)1 - (T)0.5 * mf;
        const cpx<T> g = spin < 2 ? mk<T>(cp * f.im, -cp * f.re) : mk<T>(-cp * f.im, cp * f.re);
        const cpx<T> o = mk<T>(mdw * (g.re + cm * d.re), mdw * (g.im + cm * d.im));
        if (accumulate) {
            const cpx<T> v = ld(dst + e);
            st(dst + e, mk<T>(v.re + dt * o.re, v.im + dt * o.im));
        } else {
            st(dst + e, o);
        }
    }
}

// w = D b over all modes: FP32 with hop variant 3 (and the FP32 link copy) in
// the packed-pair kernel's plain form, otherwise cheb_wilson_kernel.
template <typename T, class LK>
static void d_pass(const LK &lk, const HopConfig &hc, const cpx<T> *b, cpx<T> *w, const Lattice &L, int n_mb, T amass,
                   cudaStream_t stream) {
    if (sizeof(T) == 4 && hc.variant == kPackedVariant && hc.U32 != nullptr) {
        launch_wilson_tuned<float>(hc, b, w, L, 0, n_mb, (double)amass, 0.0, false, stream);
        return;
    }
    cheb_launch<T>(L, n_mb, [&](auto table, dim3 grid, int m) {
        cheb_wilson_kernel<T, LK, decltype(table)::value><<<grid, dim3(kModeBlock, kSitesPerCta), 0, stream>>>(
            lk, b, w, L, amass, n_mb, m);
    });
}

template <typename T, class LK>
static void cheb_run(const LK &lk, const HopConfig &hc, ChebyshevWork &w, const void *src, void *dst, const Lattice &L,
                     int n_mb, const double *coeff, int K, double eps, double lambda_max, double amass, double mdw,
                     double mf, double dt, bool accumulate, int sm_count, cudaStream_t stream, uint64_t *launches) {
    const size_t n = (size_t)n_mb * L.V * kComp * kModeBlock;
    dim3 block(kModeBlock, kSitesPerCta);
    const cpx<T> *phi = reinterpret_cast<const cpx<T> *>(src);
    cpx<T> *b[3] = {reinterpret_cast<cpx<T> *>(w.b0), reinterpret_cast<cpx<T> *>(w.b1), reinterpret_cast<cpx<T> *>(w.b2)};
    cpx<T> *tmp = reinterpret_cast<cpx<T> *>(w.w);
    const double scale = 1.0 / std::sqrt(lambda_max);
    // t(X) = a (-D^2) + beta with X = -D^2 / lambda_max
    const T a = (T)(2.0 / ((1.0 - eps) * lambda_max));
    const T beta = (T)(-(1.0 + eps) / (1.0 - eps));
    const T am = (T)amass;
    uint64_t nl = 0;
    // b_{K+1} = b_{K+2} = 0
    cudaMemsetAsync(b[1], 0, n * sizeof(cpx<T>), stream);
    cudaMemsetAsync(b[2], 0, n * sizeof(cpx<T>), stream);
    int i1 = 1, i2 = 2, io = 0;  // b_{k+1}, b_{k+2}, b_k
    for (int k = K; k >= 0; k--) {  // k = 0: y = t(X) b_1 - b_2 + c_0/2 phi (chi, scaled by lambda_max^-1/2)
        d_pass<T>(lk, hc, b[i1], tmp, L, n_mb, am, stream);
        const T factor = (T)(k > 0 ? 2 : 1), ck = (T)((k > 0 ? coeff[k] : 0.5 * coeff[0]) * scale);
        cheb_launch<T>(L, n_mb, [&](auto table, dim3 grid, int m) {
            clenshaw_kernel<T, LK, decltype(table)::value><<<grid, block, 0, stream>>>(
                lk, tmp, b[i1], b[i2], phi, b[io], L, am, a, beta, factor, ck, n_mb, m);
        });
        nl += 2;
        const int t = i2;
        i2 = i1;
        i1 = io;
        io = t;
    }
    // D chi (chi = b[i1]), then the overlap combination
    d_pass<T>(lk, hc, b[i1], tmp, L, n_mb, am, stream);
    size_t blocks = (n + 255) / 256, cap = (size_t)sm_count * 16;
    overlap_finish_t_kernel<T><<<(int)(blocks < cap ? blocks : cap), 256, 0, stream>>>(
        phi, tmp, reinterpret_cast<cpx<T> *>(dst), n, (T)mdw, (T)mf, (T)dt, accumulate ? 1 : 0);
    nl += 2;
    if (launches) *launches += nl;
}

template <typename T>
void chebyshev_apply(ChebyshevWork &w, const HopConfig &hc, const void *src, void *dst, const Lattice &L, int n_mb,
                     const double *coeff, int K, double eps, double lambda_max, double amass, double mdw, double mf,
                     double dt, bool accumulate, int sm_count, cudaStream_t stream, uint64_t *launches) {
    const int n01 = L.N0 * L.N1;
    auto go = [&](const auto &lk) {
        cheb_run<T>(lk, hc, w, src, dst, L, n_mb, coeff, K, eps, lambda_max, amass, mdw, mf, dt, accumulate, sm_count,
                    stream, launches);
    };
    if (sizeof(T) == 4 && hc.U32 != nullptr) {  // FP32 modes: the FP32 link copy
        const float4 *u = reinterpret_cast<const float4 *>(hc.U32);
        if (hc.u1_32) go(LinksF32<true>{u, reinterpret_cast<const float2 *>(hc.u1_32), n01});
        else go(LinksF32<false>{u, nullptr, n01});
    } else {
        if (hc.u1) go(LinksF64<true>{hc.U, reinterpret_cast<const double2 *>(hc.u1), n01});
        else go(LinksF64<false>{hc.U, nullptr, n01});
    }
}

template void chebyshev_apply<float>(ChebyshevWork &, const HopConfig &, const void *, void *, const Lattice &, int,
                                     const double *, int, double, double, double, double, double, double, bool, int,
                                     cudaStream_t, uint64_t *);
template void chebyshev_apply<double>(ChebyshevWork &, const HopConfig &, const void *, void *, const Lattice &, int,
                                      const double *, int, double, double, double, double, double, double, bool, int,
                                      cudaStream_t, uint64_t *);

}  // namespace ovl
