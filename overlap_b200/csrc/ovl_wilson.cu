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

#include "ovl_internal.h"
#include "ovl_stencil.cuh"

namespace ovl {

// MODE: 0 = dst  = D src          (derivative buffer, plain form)
//       1 = dst += dt * D src     (fused leapfrog half step)
template <typename T, int MODE>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta)
    wilson_kernel(const double *__restrict__ links, const double2 *__restrict__ u1, const cpx<T> *__restrict__ src,
                  cpx<T> *__restrict__ dst, Lattice L, T amass, T dt) {
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSitesPerCta + threadIdx.y;
    const int mb = blockIdx.y;
    if (site >= L.V) return;
    Spinor<T> acc;
    wilson_site(links, u1, src, L, site, mb, lane, amass, acc);
    cpx<T> *out = dst + field_index(L.V, mb, site, 0, lane);
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) {
            const cpx<T> d = finish_component(acc.c[c][a], a);
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
void launch_wilson(const double *links, const double *u1, const void *src, void *dst, const Lattice &L, int mb_first,
                   int n_mb, double amass, double dt, bool accumulate, cudaStream_t stream) {
    if (n_mb <= 0) return;
    dim3 block(kModeBlock, kSitesPerCta);
    dim3 grid((L.V + kSitesPerCta - 1) / kSitesPerCta, n_mb);
    const size_t off = field_index(L.V, mb_first, 0, 0, 0);
    const cpx<T> *s = reinterpret_cast<const cpx<T> *>(src);
    cpx<T> *d = reinterpret_cast<cpx<T> *>(dst);
    const double2 *ph = reinterpret_cast<const double2 *>(u1);
    if (accumulate)
        wilson_kernel<T, 1><<<grid, block, 0, stream>>>(links, ph, s + off, d + off, L, (T)amass, (T)dt);
    else
        wilson_kernel<T, 0><<<grid, block, 0, stream>>>(links, ph, s + off, d, L, (T)amass, (T)dt);
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

template void launch_wilson<double>(const double *, const double *, const void *, void *, const Lattice &, int, int, double,
                                    double, bool, cudaStream_t);
template void launch_wilson<float>(const double *, const double *, const void *, void *, const Lattice &, int, int, double,
                                   double, bool, cudaStream_t);
template void launch_axpy<double>(void *, const void *, size_t, double, int, cudaStream_t);
template void launch_axpy<float>(void *, const void *, size_t, double, int, cudaStream_t);

}  // namespace ovl
