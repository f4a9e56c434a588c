// The packed-pair FP32 Wilson half step (hop variant 3), shared by the
// single-context kernel (ovl_wilson.cu) and the batched ensemble kernel
// (ovl_batch.cu), and the FP64 local charges the observing half steps sum.
#pragma once

#include "ovl_stencil.cuh"

namespace ovl {

constexpr int kObsVals = 3;

// Vacuum-weighted local charges of one mode at one site (FP64 products; FP32
// inputs multiply exactly in FP64): N_V += w |psi|^2, N_5 += w 2 Re z,
// PS += -w 2 Im z with z = sum_c conj(psi_c0) psi_c2 + conj(psi_c1) psi_c3
// (psi^+ g5 psi = 2 Re z, psi^+ i g0 g5 psi = -2 Im z in the Dirac basis).
__device__ __forceinline__ void local_charges(const cpx<double> (&f)[kColours][kSpin], double w, double (&o)[kObsVals]) {
    double nv = 0.0;
    cpx<double> zz = mk<double>(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < kColours; c++) {
#pragma unroll
        for (int a = 0; a < kSpin; a++) nv += f[c][a].re * f[c][a].re + f[c][a].im * f[c][a].im;
        zz = zz + cdot(f[c][0], f[c][2]) + cdot(f[c][1], f[c][3]);
    }
    o[0] = w * nv;
    o[1] = w * 2.0 * zz.re;
    o[2] = w * -2.0 * zz.im;
}

// ------------------------------------------- packed FP32 pairs (variant 3) --
// The FP32 half step with two modes per thread and the colour and spin
// arithmetic on (mode a, mode b) pairs, one sm_100 paired FP32 instruction
// (__ffma2_rn, __fmul2_rn) per two lanes of work.  Same operator, link
// matrices and field layout as the stencil of ovl_stencil.cuh:
//   - a thread owns lanes (2q, 2q+1) of a mode block and loads a component as
//     one float4 (re_a, im_a, re_b, im_b); the spin projection (scalar adds)
//     writes its results straight into the pairs (re_a, re_b) and (im_a, im_b);
//   - the link multiply and the accumulation run on those pairs;
//   - the six links of each of the CTA's sites (FP32 copy, dressed with the
//     U(1) phase as LinksF32 does, daggered for the backward hops) are built
//     once per CTA in shared memory as broadcast pairs, so a hop reads its
//     matrix with six shared loads and no arithmetic.
// A warp covers two sites (one per half warp) x 32 modes, a CTA 16 consecutive
// sites of one mode block.
constexpr int kPkSites = 2 * kSitesPerCta;
constexpr int kPkRecVec = 6;  // float4 per link record

struct cpair {
    float2 R, I;  // (re_a, re_b), (im_a, im_b)
};

__device__ __forceinline__ float2 pr(float a, float b) { return make_float2(a, b); }
// a - b in one paired fma: b * (-1) is exact, so the result is a - b rounded once
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }

// The matrix a hop applies: dir 0..2 the link U_mu(site), 3..5 the dagger of
// U_mu(site - mu).  Record: [a00, a01, a10, a11] as (re, re, im, im), then
// (-im a00, -im a00, -im a01, -im a01) and the same for a10, a11.
template <bool U1>
__device__ __forceinline__ void build_link_record(const float4 *__restrict__ U32, const float2 *__restrict__ u1,
                                                  const Lattice &L, int site, int dir, float4 *__restrict__ rec) {
    const int mu = dir % 3;
    int ls = site;
    if (dir >= 3) {
        const Nbrs n = neighbours(L, site);
        ls = mu == 0 ? n.xm : (mu == 1 ? n.ym : n.zm);
    }
    const cmat2<float> M = LinksF32<U1>{U32, u1, L.N0 * L.N1}.template get<float>(ls, mu);
    cpx<float> a00 = M.m00, a01 = M.m01, a10 = M.m10, a11 = M.m11;
    if (dir >= 3) {
        a00 = conj(M.m00);
        a01 = conj(M.m10);
        a10 = conj(M.m01);
        a11 = conj(M.m11);
    }
    rec[0] = make_float4(a00.re, a00.re, a00.im, a00.im);
    rec[1] = make_float4(a01.re, a01.re, a01.im, a01.im);
    rec[2] = make_float4(a10.re, a10.re, a10.im, a10.im);
    rec[3] = make_float4(a11.re, a11.re, a11.im, a11.im);
    rec[4] = make_float4(-a00.im, -a00.im, -a01.im, -a01.im);
    rec[5] = make_float4(-a10.im, -a10.im, -a11.im, -a11.im);
}

// k = A h for the colour two-vector h (pairs), A from a record.
__device__ __forceinline__ void pmul(const float4 *__restrict__ rec, const cpair (&h)[kColours], cpair (&k)[kColours]) {
    const float4 a00 = rec[0], a01 = rec[1], a10 = rec[2], a11 = rec[3], n0 = rec[4], n1 = rec[5];
    k[0].R = __ffma2_rn(pr(a00.x, a00.y), h[0].R,
                        __ffma2_rn(pr(n0.x, n0.y), h[0].I,
                                   __ffma2_rn(pr(a01.x, a01.y), h[1].R, __fmul2_rn(pr(n0.z, n0.w), h[1].I))));
    k[0].I = __ffma2_rn(pr(a00.x, a00.y), h[0].I,
                        __ffma2_rn(pr(a00.z, a00.w), h[0].R,
                                   __ffma2_rn(pr(a01.x, a01.y), h[1].I, __fmul2_rn(pr(a01.z, a01.w), h[1].R))));
    k[1].R = __ffma2_rn(pr(a10.x, a10.y), h[0].R,
                        __ffma2_rn(pr(n1.x, n1.y), h[0].I,
                                   __ffma2_rn(pr(a11.x, a11.y), h[1].R, __fmul2_rn(pr(n1.z, n1.w), h[1].I))));
    k[1].I = __ffma2_rn(pr(a10.x, a10.y), h[0].I,
                        __ffma2_rn(pr(a10.z, a10.w), h[0].R,
                                   __ffma2_rn(pr(a11.x, a11.y), h[1].I, __fmul2_rn(pr(a11.z, a11.w), h[1].R))));
}

// One projected hop on pairs, in two parts so that the next neighbour's loads
// can be issued between them (the spinor registers are free once projected):
// pproject forms h0, h1 from the neighbour's 8 components (c * 4 + spin),
// pmulacc multiplies them by the link and adds them into acc.  The same
// projections and reconstruction as hop() in ovl_stencil.cuh.
template <int MU, bool FWD>
__device__ __forceinline__ void pproject(const float4 (&v)[kComp], cpair (&h0)[kColours], cpair (&h1)[kColours]) {
#pragma unroll
    for (int c = 0; c < kColours; c++) {
        const float4 p0 = v[c * kSpin], p1 = v[c * kSpin + 1], p2 = v[c * kSpin + 2], p3 = v[c * kSpin + 3];
        if (MU == 0) {  // h0 = p0 +- i p3, h1 = p1 +- i p2
            h0[c].R = FWD ? pr(p0.x - p3.y, p0.z - p3.w) : pr(p0.x + p3.y, p0.z + p3.w);
            h0[c].I = FWD ? pr(p0.y + p3.x, p0.w + p3.z) : pr(p0.y - p3.x, p0.w - p3.z);
            h1[c].R = FWD ? pr(p1.x - p2.y, p1.z - p2.w) : pr(p1.x + p2.y, p1.z + p2.w);
            h1[c].I = FWD ? pr(p1.y + p2.x, p1.w + p2.z) : pr(p1.y - p2.x, p1.w - p2.z);
        } else if (MU == 1) {  // h0 = p0 +- p3, h1 = p1 -+ p2
            h0[c].R = FWD ? pr(p0.x + p3.x, p0.z + p3.z) : pr(p0.x - p3.x, p0.z - p3.z);
            h0[c].I = FWD ? pr(p0.y + p3.y, p0.w + p3.w) : pr(p0.y - p3.y, p0.w - p3.w);
            h1[c].R = FWD ? pr(p1.x - p2.x, p1.z - p2.z) : pr(p1.x + p2.x, p1.z + p2.z);
            h1[c].I = FWD ? pr(p1.y - p2.y, p1.w - p2.w) : pr(p1.y + p2.y, p1.w + p2.w);
        } else {  // h0 = p0 +- i p2, h1 = p1 -+ i p3
            h0[c].R = FWD ? pr(p0.x - p2.y, p0.z - p2.w) : pr(p0.x + p2.y, p0.z + p2.w);
            h0[c].I = FWD ? pr(p0.y + p2.x, p0.w + p2.z) : pr(p0.y - p2.x, p0.w - p2.z);
            h1[c].R = FWD ? pr(p1.x + p3.y, p1.z + p3.w) : pr(p1.x - p3.y, p1.z - p3.w);
            h1[c].I = FWD ? pr(p1.y - p3.x, p1.w - p3.z) : pr(p1.y + p3.x, p1.w + p3.z);
        }
    }
}

template <int MU, bool FWD>
__device__ __forceinline__ void pmulacc(cpair (&acc)[kColours][kSpin], const cpair (&h0)[kColours],
                                        const cpair (&h1)[kColours], const float4 *__restrict__ rec) {
    cpair k0[kColours], k1[kColours];
    pmul(rec, h0, k0);
    pmul(rec, h1, k1);
#pragma unroll
    for (int c = 0; c < kColours; c++) {
        cpair *a = acc[c];
        a[0].R = psub(a[0].R, k0[c].R);
        a[0].I = psub(a[0].I, k0[c].I);
        a[1].R = psub(a[1].R, k1[c].R);
        a[1].I = psub(a[1].I, k1[c].I);
        if (MU == 0) {  // forward: spin 2 = -i h1, spin 3 = -i h0; backward: +i
            a[2].R = FWD ? psub(a[2].R, k1[c].I) : padd(a[2].R, k1[c].I);
            a[2].I = FWD ? padd(a[2].I, k1[c].R) : psub(a[2].I, k1[c].R);
            a[3].R = FWD ? psub(a[3].R, k0[c].I) : padd(a[3].R, k0[c].I);
            a[3].I = FWD ? padd(a[3].I, k0[c].R) : psub(a[3].I, k0[c].R);
        } else if (MU == 1) {  // forward: spin 2 = -h1, spin 3 = +h0; backward: +h1, -h0
            a[2].R = FWD ? padd(a[2].R, k1[c].R) : psub(a[2].R, k1[c].R);
            a[2].I = FWD ? padd(a[2].I, k1[c].I) : psub(a[2].I, k1[c].I);
            a[3].R = FWD ? psub(a[3].R, k0[c].R) : padd(a[3].R, k0[c].R);
            a[3].I = FWD ? psub(a[3].I, k0[c].I) : padd(a[3].I, k0[c].I);
        } else {  // forward: spin 2 = -i h0, spin 3 = +i h1; backward: +i h0, -i h1
            a[2].R = FWD ? psub(a[2].R, k0[c].I) : padd(a[2].R, k0[c].I);
            a[2].I = FWD ? padd(a[2].I, k0[c].R) : psub(a[2].I, k0[c].R);
            a[3].R = FWD ? padd(a[3].R, k1[c].I) : psub(a[3].R, k1[c].I);
            a[3].I = FWD ? psub(a[3].I, k1[c].R) : padd(a[3].I, k1[c].R);
        }
    }
}

// The local charges (local_charges) of the two modes of v, colour by colour
// with independent partial sums: the FP64 products are exact (FP32 inputs),
// only the order of the FP64 additions differs from local_charges.
__device__ __forceinline__ void pair_charges(const float4 (&v)[kComp], int mode, int n_modes, int first_mode,
                                             double (&o)[kObsVals]) {
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const double w = mode + j >= n_modes ? 0.0 : (((first_mode + mode + j) & 1) == 0 ? 1.0 : -1.0);
        double nv[kColours], zr[kColours], zi[kColours];
#pragma unroll
        for (int c = 0; c < kColours; c++) {
            double re[kSpin], im[kSpin];
#pragma unroll
            for (int a = 0; a < kSpin; a++) {
                const float4 x = v[c * kSpin + a];
                re[a] = j == 0 ? (double)x.x : (double)x.z;
                im[a] = j == 0 ? (double)x.y : (double)x.w;
            }
            nv[c] = fma(re[0], re[0], im[0] * im[0]) + fma(re[1], re[1], im[1] * im[1]) +
                    (fma(re[2], re[2], im[2] * im[2]) + fma(re[3], re[3], im[3] * im[3]));
            // conj(f0) f2 + conj(f1) f3
            zr[c] = fma(re[0], re[2], im[0] * im[2]) + fma(re[1], re[3], im[1] * im[3]);
            zi[c] = fma(re[0], im[2], -im[0] * re[2]) + fma(re[1], im[3], -im[1] * re[3]);
        }
        o[0] += w * (nv[0] + nv[1]);
        o[1] += w * 2.0 * (zr[0] + zr[1]);
        o[2] += w * -2.0 * (zi[0] + zi[1]);
    }
}

// COH false: read-only data of the launch, through the non-coherent path
// (ld.global.nc).  COH true: data that the same launch writes as well (the
// pipelined step's fields), read with ordinary coherent loads (ld.global.ca),
// which the memory model orders after an acquire.
template <bool COH = false>
__device__ __forceinline__ void load_spinor4(const float4 *__restrict__ p, float4 (&v)[kComp]) {
#pragma unroll
    for (int k = 0; k < kComp; k++) v[k] = COH ? __ldca(p + k * (kModeBlock / 2)) : __ldg(p + k * (kModeBlock / 2));
}

// A CTA runs kPkBlocks mode blocks of its 16 sites one after the other on the
// same link records; the first block's own-site spinor is in flight while the
// records are built.
constexpr int kPkBlocks = 8;

// One CTA's tile: sites [site0, site0 + 16) x mode blocks [mb0, mb1) of the
// fields src/dst (float4 views, mode block 0 at the pointers).  MODE 0:
// dst = D src; 1: dst += dt D src (hdt = dt / 2, the 1/2 of D folded in,
// exact).  OBS (and observe, uniform over the CTA): the local charges of src
// are added into o (weights +-1 by the parity of first_mode + mode, 0 beyond
// n_modes).  Every thread of the CTA calls it (it holds a barrier); rec is the
// CTA's shared link records.
// W: warps per CTA (2 W sites); DEPTH: neighbour spinors in flight per thread
// (2: two register buffers alternate, each refilled two hops ahead).  COH:
// src is written elsewhere in the same launch (load_spinor4).
template <int MODE, bool U1, bool OBS, int W = kSitesPerCta, int DEPTH = 1, bool COH = false>
__device__ __forceinline__ void packed_tile(float4 (*__restrict__ rec)[6][kPkRecVec], const float4 *__restrict__ U32,
                                            const float2 *__restrict__ u1, const float4 *__restrict__ src,
                                            float4 *__restrict__ dst, const Lattice &L, int site0, int mb0, int mb1,
                                            float amass, float hdt, int n_modes, int first_mode,
                                            double (&o)[kObsVals], bool observe = true) {
    const int t = threadIdx.y * kModeBlock + threadIdx.x;
    const int sl = 2 * threadIdx.y + (threadIdx.x >> 4), q = threadIdx.x & 15;
    const int site = site0 + sl;
    const bool live = site < L.V;
    // float4 index of component 0 of (mb, s) for this thread's lane pair
    auto at = [&](int mb, int s) { return (((size_t)mb * L.V + s) * kComp) * (kModeBlock / 2) + q; };
    float4 v[kComp];
    if (live) load_spinor4<COH>(src + at(mb0, site), v);
    if (t < 2 * W * 6) {
        const int s = site0 + t / 6;
        if (s < L.V) build_link_record<U1>(U32, u1, L, s, t % 6, rec[t / 6][t % 6]);
    }
    __syncthreads();
    if (live) {
        const Nbrs n = neighbours(L, site);
        const float4(*r)[kPkRecVec] = rec[sl];
        for (int mb = mb0; mb < mb1; mb++) {
            if (mb > mb0) load_spinor4<COH>(src + at(mb, site), v);
            cpair acc[kColours][kSpin];
#pragma unroll
            for (int c = 0; c < kColours; c++)
#pragma unroll
                for (int a = 0; a < kSpin; a++) {
                    const float4 f = v[c * kSpin + a];
                    acc[c][a].R = pr(amass * f.x, amass * f.z);
                    acc[c][a].I = pr(amass * f.y, amass * f.w);
                }
            float4 w[kComp];  // the second buffer (DEPTH 2): the first neighbour is in flight during the sums
            if (DEPTH == 2) load_spinor4<COH>(src + at(mb, n.xp), w);
            if (OBS && observe) pair_charges(v, mb * kModeBlock + 2 * q, n_modes, first_mode, o);
            cpair h0[kColours], h1[kColours];
            if (DEPTH == 1) {
                load_spinor4<COH>(src + at(mb, n.xp), v);
                pproject<0, true>(v, h0, h1);
                load_spinor4<COH>(src + at(mb, n.xm), v);
                pmulacc<0, true>(acc, h0, h1, r[0]);
                pproject<0, false>(v, h0, h1);
                load_spinor4<COH>(src + at(mb, n.yp), v);
                pmulacc<0, false>(acc, h0, h1, r[3]);
                pproject<1, true>(v, h0, h1);
                load_spinor4<COH>(src + at(mb, n.ym), v);
                pmulacc<1, true>(acc, h0, h1, r[1]);
                pproject<1, false>(v, h0, h1);
                load_spinor4<COH>(src + at(mb, n.zp), v);
                pmulacc<1, false>(acc, h0, h1, r[4]);
                pproject<2, true>(v, h0, h1);
                load_spinor4<COH>(src + at(mb, n.zm), v);
                pmulacc<2, true>(acc, h0, h1, r[2]);
                pproject<2, false>(v, h0, h1);
                pmulacc<2, false>(acc, h0, h1, r[5]);
            } else {  // w holds xp (issued above), v is free once the site's own spinor is used
                load_spinor4<COH>(src + at(mb, n.xm), v);
                pproject<0, true>(w, h0, h1);
                load_spinor4<COH>(src + at(mb, n.yp), w);
                pmulacc<0, true>(acc, h0, h1, r[0]);
                pproject<0, false>(v, h0, h1);
                load_spinor4<COH>(src + at(mb, n.ym), v);
                pmulacc<0, false>(acc, h0, h1, r[3]);
                pproject<1, true>(w, h0, h1);
                load_spinor4<COH>(src + at(mb, n.zp), w);
                pmulacc<1, true>(acc, h0, h1, r[1]);
                pproject<1, false>(v, h0, h1);
                load_spinor4<COH>(src + at(mb, n.zm), v);
                pmulacc<1, false>(acc, h0, h1, r[4]);
                pproject<2, true>(w, h0, h1);
                pmulacc<2, true>(acc, h0, h1, r[2]);
                pproject<2, false>(v, h0, h1);
                pmulacc<2, false>(acc, h0, h1, r[5]);
            }
            // -i gamma_0 / 2: spins 0, 1 times -i/2, spins 2, 3 times +i/2
            float4 *out = dst + at(mb, site);
#pragma unroll
            for (int c = 0; c < kColours; c++)
#pragma unroll
                for (int a = 0; a < kSpin; a++) {
                    const cpair &x = acc[c][a];
                    const float sg = a < 2 ? 1.0f : -1.0f;
                    float4 *o4 = out + (c * kSpin + a) * (kModeBlock / 2);
                    if (MODE == 0) {
                        const float h = 0.5f * sg;
                        *o4 = make_float4(h * x.I.x, -h * x.R.x, h * x.I.y, -h * x.R.y);
                    } else {
                        const float h = hdt * sg;
                        const float4 d = *o4;
                        *o4 = make_float4(fmaf(h, x.I.x, d.x), fmaf(-h, x.R.x, d.y), fmaf(h, x.I.y, d.z),
                                          fmaf(-h, x.R.y, d.w));
                    }
                }
        }
    }
}

}  // namespace ovl
