// The Wilson stencil shared by the kernels that apply D = -i h_W
// (ovl_wilson.cu: leapfrog half steps; ovl_chebyshev.cu: Clenshaw recurrence).
// Reference: WilsonEvoOperator::Compute (FERMIONS/WILSON/OPERATOR/WilsonOperator.cpp:30-114):
//   (D phi)(x) = -(i/2) gamma_0 [ (6r + 2m - 2M) phi(x)
//                  - sum_mu (1 - G_mu) U_mu(x) phi(x+mu) + (1 + G_mu) U_mu(x-mu)^+ phi(x-mu) ]
// with G_mu = -i gamma_mu.  (1 -+ G_mu)/2 are rank-2 spin projectors, so each
// hop multiplies two colour vectors by the link instead of four (spin
// projection): the reference's operator, evaluated in a different order.
#pragma once

#include "ovl_device.cuh"

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

// (D phi)(site) for the 32 modes of block mb (one per lane), before the
// -i gamma_0 / 2 factor: amass phi(x) - sum of the six projected hops.
template <typename T>
__device__ __forceinline__ void wilson_site(const double *__restrict__ links, const double2 *__restrict__ u1,
                                            const cpx<T> *__restrict__ src, const Lattice &L, int site, int mb,
                                            int lane, T amass, Spinor<T> &acc) {
    int x, y, z;
    site_coords(L, site, x, y, z);
    const int V = L.V;
    Spinor<T> f;
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
    hop<T, 0, true>(acc, f, dressed_link<T>(links, u1, site, 0, n01));
    load_spinor(src, V, mb, xm, lane, f);
    hop<T, 0, false>(acc, f, dressed_link<T>(links, u1, xm, 0, n01));
    load_spinor(src, V, mb, yp, lane, f);
    hop<T, 1, true>(acc, f, dressed_link<T>(links, u1, site, 1, n01));
    load_spinor(src, V, mb, ym, lane, f);
    hop<T, 1, false>(acc, f, dressed_link<T>(links, u1, ym, 1, n01));
    load_spinor(src, V, mb, zp, lane, f);
    hop<T, 2, true>(acc, f, dressed_link<T>(links, u1, site, 2, n01));
    load_spinor(src, V, mb, zm, lane, f);
    hop<T, 2, false>(acc, f, dressed_link<T>(links, u1, zm, 2, n01));
}

// Component (c, a) of -i gamma_0 / 2 acc: spins 0,1 times -i/2, spins 2,3 times +i/2.
template <typename T> __device__ __forceinline__ cpx<T> finish_component(const cpx<T> &v, int a) {
    const cpx<T> d = a < 2 ? times_mi(v) : times_i(v);
    return (T)0.5 * d;
}

}  // namespace ovl
