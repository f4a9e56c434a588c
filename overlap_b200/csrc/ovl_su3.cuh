// Three colours: SU(3) link algebra and the Wilson stencil for 12-component
// modes.  No reference counterpart exists for the fermions (the reference's
// fermion code is written for two colours, FermionField.cpp:8-9,
// WilsonOperator.cpp:45-46); the operator is the two-colour one
// (ovl_stencil.cuh) with 3x3 links.
//   links: 9 complex numbers per link, U_ij at i + 3j (SUNc/SU3/GroupOperations.cpp:4-12),
//          link (site, mu) at 18 (mu + 3 site) doubles; an FP32 copy keeps the
//          same order in floats, each link padded to 20 floats (80 bytes);
//   E:     8 components per link (t^a = lambda^a / 2), E[a + 8 (mu + 3 site)];
//   modes: mode blocks [mb][site][colour * 4 + spin][32 lanes].
#pragma once

#include "ovl_device.cuh"

namespace ovl {

constexpr int kColours3 = 3;
constexpr int kComp3 = kColours3 * kSpin;
constexpr int kSites3 = 4;  // sites (warps) per CTA of the three-colour stencil kernels
// The FP32 link copy: each link's 18 floats (the FP64 order) padded to 80 bytes.
constexpr int kLink32Floats = 20;
constexpr int kLink32Vec4 = kLink32Floats / 4;

__host__ __device__ inline size_t field_index3(int V, int mb, int site, int comp, int lane) {
    return (((size_t)mb * V + site) * kComp3 + comp) * kModeBlock + lane;
}

template <typename T> struct cmat3 { cpx<T> m[3][3]; };
template <typename T> struct Spinor3 { cpx<T> c[kColours3][kSpin]; };

template <typename T> __device__ __forceinline__ cmat3<T> m3_unit() {
    cmat3<T> a;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) a.m[i][j] = mk<T>(i == j ? (T)1 : (T)0, (T)0);
    return a;
}

__device__ __forceinline__ cmat3<double> load_su3(const double *__restrict__ U, int site, int mu) {
    const double2 *p = reinterpret_cast<const double2 *>(U) + 9 * (size_t)(3 * site + mu);
    cmat3<double> a;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const double2 v = __ldg(p + i + 3 * j);
            a.m[i][j] = mk<double>(v.x, v.y);
        }
    return a;
}

__device__ __forceinline__ void store_su3(double *U, int site, int mu, const cmat3<double> &a) {
    double2 *p = reinterpret_cast<double2 *>(U) + 9 * (size_t)(3 * site + mu);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) p[i + 3 * j] = double2{a.m[i][j].re, a.m[i][j].im};
}

template <typename T> __device__ __forceinline__ cmat3<T> m3_mul(const cmat3<T> &a, const cmat3<T> &b) {
    cmat3<T> c;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) c.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return c;
}

template <typename T> __device__ __forceinline__ cmat3<T> m3_dag(const cmat3<T> &a) {
    cmat3<T> c;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) c.m[i][j] = conj(a.m[j][i]);
    return c;
}

// t^a alpha^a (MatrixForm, SU3/AlgebraOperations.cpp:89-105)
__device__ __forceinline__ cmat3<double> su3_form(const double *al) {
    const double r3 = 0.57735026918962576451;  // 1/sqrt(3)
    cmat3<double> A;
    A.m[0][0] = mk<double>(0.5 * (al[2] + al[7] * r3), 0.0);
    A.m[1][1] = mk<double>(-0.5 * (al[2] - al[7] * r3), 0.0);
    A.m[2][2] = mk<double>(-al[7] * r3, 0.0);
    A.m[1][0] = mk<double>(0.5 * al[0], 0.5 * al[1]);
    A.m[2][0] = mk<double>(0.5 * al[3], 0.5 * al[4]);
    A.m[2][1] = mk<double>(0.5 * al[5], 0.5 * al[6]);
    A.m[0][1] = conj(A.m[1][0]);
    A.m[0][2] = conj(A.m[2][0]);
    A.m[1][2] = conj(A.m[2][1]);
    return A;
}

// 2 tr(t^a H) for a hermitian H (the inverse of su3_form on traceless H).
__device__ __forceinline__ void su3_components(const cmat3<double> &H, double *out) {
    const double r3 = 0.57735026918962576451;
    out[0] = H.m[0][1].re + H.m[1][0].re;
    out[1] = H.m[1][0].im - H.m[0][1].im;
    out[2] = H.m[0][0].re - H.m[1][1].re;
    out[3] = H.m[0][2].re + H.m[2][0].re;
    out[4] = H.m[2][0].im - H.m[0][2].im;
    out[5] = H.m[1][2].re + H.m[2][1].re;
    out[6] = H.m[2][1].im - H.m[1][2].im;
    out[7] = (H.m[0][0].re + H.m[1][1].re - 2.0 * H.m[2][2].re) * r3;
}

// Re tr(i t^a V) = -Im tr(t^a V) for all a, written out per generator
// (ReTrIGenU, SU3/GroupOperations.cpp:108-119).
__device__ __forceinline__ void su3_retr_ita(const cmat3<double> &V, double *out) {
    const double r3 = 0.57735026918962576451;
    out[0] = -0.5 * (V.m[0][1].im + V.m[1][0].im);
    out[1] = -0.5 * (V.m[0][1].re - V.m[1][0].re);
    out[2] = -0.5 * (V.m[0][0].im - V.m[1][1].im);
    out[3] = -0.5 * (V.m[0][2].im + V.m[2][0].im);
    out[4] = -0.5 * (V.m[0][2].re - V.m[2][0].re);
    out[5] = -0.5 * (V.m[1][2].im + V.m[2][1].im);
    out[6] = -0.5 * (V.m[1][2].re - V.m[2][1].re);
    out[7] = -0.5 * (V.m[0][0].im + V.m[1][1].im - 2.0 * V.m[2][2].im) * r3;
}

// exp(X) for X = i c t^a alpha^a by scaling and squaring of the Taylor series:
// X / 2^s with Frobenius norm <= 1/4, 13 terms (remainder below 1e-17), then
// s squarings.  (The reference diagonalises, SU3/AlgebraOperations.cpp:141-183;
// both are exact to rounding.)
__device__ inline cmat3<double> su3_exp(double c, const double *alpha) {
    cmat3<double> A = su3_form(alpha), X;
    double nrm = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            X.m[i][j] = mk<double>(-c * A.m[i][j].im, c * A.m[i][j].re);  // i c A
            nrm += X.m[i][j].re * X.m[i][j].re + X.m[i][j].im * X.m[i][j].im;
        }
    nrm = sqrt(nrm);
    int s = 0;
    while (nrm > 0.25 && s < 60) {
        nrm *= 0.5;
        s++;
    }
    const double sc = ldexp(1.0, -s);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) X.m[i][j] = sc * X.m[i][j];
    // Horner: 1 + X (1 + X/2 (1 + X/3 (... (1 + X/13))))
    cmat3<double> R = m3_unit<double>();
    for (int k = 13; k >= 1; k--) {
        cmat3<double> t = m3_mul(X, R);
        const double f = 1.0 / k;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) R.m[i][j] = mk<double>((i == j ? 1.0 : 0.0) + f * t.m[i][j].re, f * t.m[i][j].im);
    }
    for (int k = 0; k < s; k++) R = m3_mul(R, R);
    return R;
}

// Gram-Schmidt onto SU(3): rows 0 and 1 orthonormalised, row 2 the conjugated
// cross product (unit determinant).
__device__ inline cmat3<double> su3_reunitarize(const cmat3<double> &U) {
    cmat3<double> R;
    double n0 = 0.0;
    for (int j = 0; j < 3; j++) n0 += U.m[0][j].re * U.m[0][j].re + U.m[0][j].im * U.m[0][j].im;
    n0 = 1.0 / sqrt(n0);
    for (int j = 0; j < 3; j++) R.m[0][j] = n0 * U.m[0][j];
    cpx<double> d = mk<double>(0.0, 0.0);
    for (int j = 0; j < 3; j++) d = d + cdot(R.m[0][j], U.m[1][j]);
    double n1 = 0.0;
    for (int j = 0; j < 3; j++) {
        R.m[1][j] = U.m[1][j] - d * R.m[0][j];
        n1 += R.m[1][j].re * R.m[1][j].re + R.m[1][j].im * R.m[1][j].im;
    }
    n1 = 1.0 / sqrt(n1);
    for (int j = 0; j < 3; j++) R.m[1][j] = n1 * R.m[1][j];
    R.m[2][0] = conj(R.m[0][1] * R.m[1][2] - R.m[0][2] * R.m[1][1]);
    R.m[2][1] = conj(R.m[0][2] * R.m[1][0] - R.m[0][0] * R.m[1][2]);
    R.m[2][2] = conj(R.m[0][0] * R.m[1][1] - R.m[0][1] * R.m[1][0]);
    return R;
}

// ---------------------------------------------------------------- stencil --
// Where the three-colour hop kernels read links from: FP64 links, or (F32)
// the FP32 copy; U1: x and y links dressed with the U(1) background phase.
template <bool F32, bool U1> struct Links3 {
    const void *U;
    const void *u1;
    int n01;
    template <typename T> __device__ __forceinline__ cmat3<T> get(int site, int mu) const {
        cmat3<T> M;
        if (F32) {  // 80-byte records: five 16-byte loads
            const float4 *p = reinterpret_cast<const float4 *>(U) + kLink32Vec4 * (size_t)(3 * site + mu);
            float f[20];
#pragma unroll
            for (int k = 0; k < 5; k++) {
                const float4 v = __ldg(p + k);
                f[4 * k] = v.x;
                f[4 * k + 1] = v.y;
                f[4 * k + 2] = v.z;
                f[4 * k + 3] = v.w;
            }
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) M.m[i][j] = mk<T>((T)f[2 * (i + 3 * j)], (T)f[2 * (i + 3 * j) + 1]);
        } else {
            const double2 *p = reinterpret_cast<const double2 *>(U) + 9 * (size_t)(3 * site + mu);
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    const double2 v = __ldg(p + i + 3 * j);
                    M.m[i][j] = mk<T>((T)v.x, (T)v.y);
                }
        }
        if (U1 && mu < 2) {
            cpx<T> ph;
            if (F32) {
                const float2 v = __ldg(reinterpret_cast<const float2 *>(u1) + 2 * (site % n01) + mu);
                ph = mk<T>((T)v.x, (T)v.y);
            } else {
                const double2 v = __ldg(reinterpret_cast<const double2 *>(u1) + 2 * (site % n01) + mu);
                ph = mk<T>((T)v.x, (T)v.y);
            }
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) M.m[i][j] = ph * M.m[i][j];
        }
        return M;
    }
};

// acc -= (1 - G_mu) U phi(x+mu) (forward) or (1 + G_mu) U^+ phi(x-mu)
// (backward) for one neighbour, read component by component: the two
// projected colour vectors h0, h1 are formed as the spinor arrives, multiplied
// by the link, and the lower spin components rebuilt (the projections of hop()
// in ovl_stencil.cuh).
// a0 h0 + a1 h1 + a2 h2 (CONJ: conj(a_k) h_k) as two chains of fused
// multiply-adds, one per real and imaginary part (the signs of the im * im
// terms are operand negations, no extra instructions).
template <typename T, bool CONJ>
__device__ __forceinline__ cpx<T> row3(const cpx<T> &a0, const cpx<T> &a1, const cpx<T> &a2, const cpx<T> (&h)[3]) {
    const T s = CONJ ? (T)1 : (T)-1;  // sign of a.im * h.im in the real part
    cpx<T> k;
    k.re = fma(a0.re, h[0].re, fma(s * a0.im, h[0].im, fma(a1.re, h[1].re, fma(s * a1.im, h[1].im,
                                                                                fma(a2.re, h[2].re, s * a2.im * h[2].im)))));
    k.im = fma(a0.re, h[0].im, fma(-s * a0.im, h[0].re, fma(a1.re, h[1].im, fma(-s * a1.im, h[1].re,
                                                                                 fma(a2.re, h[2].im, -s * a2.im * h[2].re)))));
    return k;
}

// COH false: read-only data (ld.global.nc); true: data the same launch writes
// (coherent ld.global.ca, ordered after an acquire).
template <bool COH, typename T> __device__ __forceinline__ cpx<T> ld3(const cpx<T> *p) {
    if (!COH) return ld(p);
    using V2 = typename vec2_of<T>::type;
    const V2 v = __ldca(reinterpret_cast<const V2 *>(p));
    return mk<T>(v.x, v.y);
}

// STRIDE: elements between consecutive components of one spinor (the mode
// block's 32 lanes, or 1 for a single vector stored component by component).
template <typename T, int MU, bool FWD, bool COH = false, int STRIDE = kModeBlock>
__device__ __forceinline__ void hop3(Spinor3<T> &acc, const cpx<T> *__restrict__ f, const cmat3<T> &M) {
    cpx<T> h0[3], h1[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const cpx<T> *p = f + c * kSpin * STRIDE;
        const cpx<T> p0 = ld3<COH>(p), p1 = ld3<COH>(p + STRIDE), p2 = ld3<COH>(p + 2 * STRIDE),
                     p3 = ld3<COH>(p + 3 * STRIDE);
        if (MU == 0) {
            h0[c] = FWD ? p0 + times_i(p3) : p0 - times_i(p3);
            h1[c] = FWD ? p1 + times_i(p2) : p1 - times_i(p2);
        } else if (MU == 1) {
            h0[c] = FWD ? p0 + p3 : p0 - p3;
            h1[c] = FWD ? p1 - p2 : p1 + p2;
        } else {
            h0[c] = FWD ? p0 + times_i(p2) : p0 - times_i(p2);
            h1[c] = FWD ? p1 - times_i(p3) : p1 + times_i(p3);
        }
    }
    cpx<T> k0[3], k1[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (FWD) {
            k0[i] = row3<T, false>(M.m[i][0], M.m[i][1], M.m[i][2], h0);
            k1[i] = row3<T, false>(M.m[i][0], M.m[i][1], M.m[i][2], h1);
        } else {
            k0[i] = row3<T, true>(M.m[0][i], M.m[1][i], M.m[2][i], h0);
            k1[i] = row3<T, true>(M.m[0][i], M.m[1][i], M.m[2][i], h1);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        cpx<T> *a = acc.c[c];
        a[0] = a[0] - k0[c];
        a[1] = a[1] - k1[c];
        if (MU == 0) {
            a[2] = FWD ? a[2] - times_mi(k1[c]) : a[2] - times_i(k1[c]);
            a[3] = FWD ? a[3] - times_mi(k0[c]) : a[3] - times_i(k0[c]);
        } else if (MU == 1) {
            a[2] = FWD ? a[2] + k1[c] : a[2] - k1[c];
            a[3] = FWD ? a[3] - k0[c] : a[3] + k0[c];
        } else {
            a[2] = FWD ? a[2] - times_mi(k0[c]) : a[2] - times_i(k0[c]);
            a[3] = FWD ? a[3] - times_i(k1[c]) : a[3] - times_mi(k1[c]);
        }
    }
}

// (D phi)(site) before the -i gamma_0 / 2 factor, for the 32 modes of block mb.
template <typename T, class LK, bool COH = false>
__device__ __forceinline__ void wilson_site3(const LK &lk, const cpx<T> *__restrict__ src, const Lattice &L, int site,
                                             int mb, int lane, T amass, Spinor3<T> &acc) {
    int x, y, z;
    site_coords(L, site, x, y, z);
    const int n01 = L.N0 * L.N1, V = L.V;
    const int xp = x + 1 == L.N0 ? site + 1 - L.N0 : site + 1;
    const int xm = x == 0 ? site - 1 + L.N0 : site - 1;
    const int yp = y + 1 == L.N1 ? site + L.N0 - n01 : site + L.N0;
    const int ym = y == 0 ? site - L.N0 + n01 : site - L.N0;
    const int zp = z + 1 == L.N2 ? site + n01 - V : site + n01;
    const int zm = z == 0 ? site - n01 + V : site - n01;
    const cpx<T> *f = src + field_index3(V, mb, site, 0, lane);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) acc.c[c][a] = amass * ld3<COH>(f + (c * kSpin + a) * kModeBlock);
    hop3<T, 0, true, COH>(acc, src + field_index3(V, mb, xp, 0, lane), lk.template get<T>(site, 0));
    hop3<T, 0, false, COH>(acc, src + field_index3(V, mb, xm, 0, lane), lk.template get<T>(xm, 0));
    hop3<T, 1, true, COH>(acc, src + field_index3(V, mb, yp, 0, lane), lk.template get<T>(site, 1));
    hop3<T, 1, false, COH>(acc, src + field_index3(V, mb, ym, 0, lane), lk.template get<T>(ym, 1));
    hop3<T, 2, true, COH>(acc, src + field_index3(V, mb, zp, 0, lane), lk.template get<T>(site, 2));
    hop3<T, 2, false, COH>(acc, src + field_index3(V, mb, zm, 0, lane), lk.template get<T>(zm, 2));
}

}  // namespace ovl
