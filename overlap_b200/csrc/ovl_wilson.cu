// Wilson evolution operator D = -i h_W on blocks of modes, and the leapfrog
// half step built on it.
//
// Reference: WilsonEvoOperator::Compute (FERMIONS/WILSON/OPERATOR/WilsonOperator.cpp:30-114)
// and Dynamics::Fermions::SingleModeUpdate (FERMIONS/WILSON/Update.cpp:6-27):
//   (D phi)(x) = -(i/2) gamma_0 [ (6r + 2m - 2M) phi(x)
//                  - sum_mu (1 - G_mu) U_mu(x) phi(x+mu) + (1 + G_mu) U_mu(x-mu)^+ phi(x-mu) ]
// with G_mu = -i gamma_mu.  (1 -+ G_mu)/2 are rank-2 spin projectors, so each
// hop multiplies two colour vectors by the link instead of four
// (spin projection); the result is the reference's operator, evaluated in a
// different order.
//
// Launch shape: a warp owns 32 modes (one mode block) at one site, so every
// link load is warp-uniform and every field load is one contiguous 32-element
// run.  blockDim = (32, kSitesPerCta); grid.x walks sites fastest so that the
// CTAs resident at one time cover a compact window of one mode block and the
// six neighbour reads of a site come from L1/L2 rather than HBM.

#include "ovl_device.cuh"
#include "ovl_internal.h"

namespace ovl {

template <typename T> struct Spinor { cpx<T> c[kColours][kSpin]; };

template <typename T>
__device__ __forceinline__ void load_spinor(const cpx<T> *__restrict__ f, int V, int mb, int site, int lane, Spinor<T> &s) {
    const cpx<T> *p = f + field_index(V, mb, site, 0, lane);
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) s.c[c][a] = ld(p + (c * kSpin + a) * kModeBlock);
}

// acc -= (1 - G_mu) U phi(x+mu)   (forward)    or
// acc -= (1 + G_mu) U^+ phi(x-mu) (backward); the projected two-spinor h is
// multiplied by the link and the two lower spin components are rebuilt from it.
template <typename T, int MU, bool FWD>
__device__ __forceinline__ void hop(Spinor<T> &acc, const Spinor<T> &f, const cmat2<T> &M) {
    cpx<T> h0[kColours], h1[kColours];
#pragma unroll
    for (int c = 0; c < kColours; c++) {
        const cpx<T> *p = f.c[c];
        if (MU == 0) {
            h0[c] = FWD ? p[0] + times_i(p[3]) : p[0] - times_i(p[3]);
            h1[c] = FWD ? p[1] + times_i(p[2]) : p[1] - times_i(p[2]);
        } else if (MU == 1) {
            h0[c] = FWD ? p[0] + p[3] : p[0] - p[3];
            h1[c] = FWD ? p[1] - p[2] : p[1] + p[2];
        } else {
            h0[c] = FWD ? p[0] + times_i(p[2]) : p[0] - times_i(p[2]);
            h1[c] = FWD ? p[1] - times_i(p[3]) : p[1] + times_i(p[3]);
        }
    }
    cpx<T> k0[kColours], k1[kColours];
    if (FWD) {
        mul(M, h0[0], h0[1], k0[0], k0[1]);
        mul(M, h1[0], h1[1], k1[0], k1[1]);
    } else {
        mul_dag(M, h0[0], h0[1], k0[0], k0[1]);
        mul_dag(M, h1[0], h1[1], k1[0], k1[1]);
    }
#pragma unroll
    for (int c = 0; c < kColours; c++) {
        cpx<T> *a = acc.c[c];
        a[0] = a[0] - k0[c];
        a[1] = a[1] - k1[c];
        if (MU == 0) {
            // forward: spin 2 = -i h1, spin 3 = -i h0; backward: +i
            a[2] = FWD ? a[2] - times_mi(k1[c]) : a[2] - times_i(k1[c]);
            a[3] = FWD ? a[3] - times_mi(k0[c]) : a[3] - times_i(k0[c]);
        } else if (MU == 1) {
            // forward: spin 2 = -h1, spin 3 = +h0; backward: +h1, -h0
            a[2] = FWD ? a[2] + k1[c] : a[2] - k1[c];
            a[3] = FWD ? a[3] - k0[c] : a[3] + k0[c];
        } else {
            // forward: spin 2 = -i h0, spin 3 = +i h1; backward: +i h0, -i h1
            a[2] = FWD ? a[2] - times_mi(k0[c]) : a[2] - times_i(k0[c]);
            a[3] = FWD ? a[3] - times_i(k1[c]) : a[3] - times_mi(k1[c]);
        }
    }
}

// MODE: 0 = dst  = D src          (derivative buffer, plain form)
//       1 = dst += dt * D src     (fused leapfrog half step)
template <typename T, int MODE>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta)
    wilson_kernel(const double *__restrict__ links, const cpx<T> *__restrict__ src, cpx<T> *__restrict__ dst,
                  Lattice L, T amass, T dt) {
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSitesPerCta + threadIdx.y;
    const int mb = blockIdx.y;
    if (site >= L.V) return;
    int x, y, z;
    site_coords(L, site, x, y, z);
    const int V = L.V;

    Spinor<T> acc, f;
    load_spinor(src, V, mb, site, lane, f);
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) acc.c[c][a] = amass * f.c[c][a];

    const int xp = x + 1 == L.N0 ? site + 1 - L.N0 : site + 1;
    const int xm = x == 0 ? site - 1 + L.N0 : site - 1;
    const int n01 = L.N0 * L.N1;
    const int yp = y + 1 == L.N1 ? site + L.N0 - n01 : site + L.N0;
    const int ym = y == 0 ? site - L.N0 + n01 : site - L.N0;
    const int zp = z + 1 == L.N2 ? site + n01 - V : site + n01;
    const int zm = z == 0 ? site - n01 + V : site - n01;

    load_spinor(src, V, mb, xp, lane, f);
    hop<T, 0, true>(acc, f, link_matrix<T>(load_link(links, site, 0)));
    load_spinor(src, V, mb, xm, lane, f);
    hop<T, 0, false>(acc, f, link_matrix<T>(load_link(links, xm, 0)));
    load_spinor(src, V, mb, yp, lane, f);
    hop<T, 1, true>(acc, f, link_matrix<T>(load_link(links, site, 1)));
    load_spinor(src, V, mb, ym, lane, f);
    hop<T, 1, false>(acc, f, link_matrix<T>(load_link(links, ym, 1)));
    load_spinor(src, V, mb, zp, lane, f);
    hop<T, 2, true>(acc, f, link_matrix<T>(load_link(links, site, 2)));
    load_spinor(src, V, mb, zm, lane, f);
    hop<T, 2, false>(acc, f, link_matrix<T>(load_link(links, zm, 2)));

    // -i gamma_0 / 2: spins 0,1 times -i/2, spins 2,3 times +i/2
    cpx<T> *out = dst + field_index(V, mb, site, 0, lane);
    const T half = (T)0.5;
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) {
            cpx<T> d = a < 2 ? times_mi(acc.c[c][a]) : times_i(acc.c[c][a]);
            d = half * d;
            cpx<T> *o = out + (c * kSpin + a) * kModeBlock;
            if (MODE == 0) {
                st(o, d);
            } else {
                cpx<T> v = ld(o);
                st(o, v + dt * d);
            }
        }
}

// dst += dt * deriv over n complex numbers (plain form, second phase).
template <typename T>
__global__ void axpy_kernel(cpx<T> *__restrict__ dst, const cpx<T> *__restrict__ deriv, size_t n, T dt) {
    using V2 = typename vec2_of<T>::type;
    V2 *d = reinterpret_cast<V2 *>(dst);
    const V2 *s = reinterpret_cast<const V2 *>(deriv);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        V2 a = d[i], b = __ldg(s + i);
        a.x += dt * b.x;
        a.y += dt * b.y;
        d[i] = a;
    }
}

template <typename T>
void launch_wilson(const double *links, const void *src, void *dst, const Lattice &L, int mb_first, int n_mb,
                   double amass, double dt, bool accumulate, cudaStream_t stream) {
    if (n_mb <= 0) return;
    dim3 block(kModeBlock, kSitesPerCta);
    dim3 grid((L.V + kSitesPerCta - 1) / kSitesPerCta, n_mb);
    const size_t off = field_index(L.V, mb_first, 0, 0, 0);
    const cpx<T> *s = reinterpret_cast<const cpx<T> *>(src);
    cpx<T> *d = reinterpret_cast<cpx<T> *>(dst);
    if (accumulate)
        wilson_kernel<T, 1><<<grid, block, 0, stream>>>(links, s + off, d + off, L, (T)amass, (T)dt);
    else
        wilson_kernel<T, 0><<<grid, block, 0, stream>>>(links, s + off, d, L, (T)amass, (T)dt);
}

template <typename T>
void launch_axpy(void *dst, const void *deriv, size_t n_complex, double dt, int sm_count, cudaStream_t stream) {
    const int threads = 256;
    size_t want = (n_complex + threads - 1) / threads;
    size_t cap = (size_t)sm_count * 16;
    int blocks = (int)(want < cap ? want : cap);
    if (blocks < 1) blocks = 1;
    axpy_kernel<T><<<blocks, threads, 0, stream>>>(reinterpret_cast<cpx<T> *>(dst),
                                                   reinterpret_cast<const cpx<T> *>(deriv), n_complex, (T)dt);
}

template void launch_wilson<double>(const double *, const void *, void *, const Lattice &, int, int, double, double, bool, cudaStream_t);
template void launch_wilson<float>(const double *, const void *, void *, const Lattice &, int, int, double, double, bool, cudaStream_t);
template void launch_axpy<double>(void *, const void *, size_t, double, int, cudaStream_t);
template void launch_axpy<float>(void *, const void *, size_t, double, int, cudaStream_t);

}  // namespace ovl
