// The three-colour FP32 Wilson stencil on packed pairs: two modes per thread
// with the colour and spin arithmetic on (mode a, mode b) pairs, one sm_100
// paired FP32 instruction (__ffma2_rn, __fmul2_rn, __fadd2_rn) per two lanes of
// work -- the two-colour packed kernel of ovl_packed.cuh with 3x3 links.  Same
// operator, links and field layout as the scalar stencil of ovl_su3.cuh:
//   - a thread owns lanes (2q, 2q+1) of a mode block and loads a component as
//     one float4 (re_a, im_a, re_b, im_b); the spin projection (scalar adds)
//     writes its results straight into the pairs (re_a, re_b), (im_a, im_b);
//   - the link multiply and the accumulation run on those pairs;
//   - the six links of each of the CTA's sites (FP32 copy, dressed with the
//     U(1) phase as Links3 does, daggered for the backward hops) are built once
//     per CTA in shared memory as broadcast pairs, so a hop reads its matrix
//     from shared memory and does no link arithmetic.
// A warp covers two sites (one per half warp) x 32 modes.
#pragma once

#include "ovl_packed.cuh"
#include "ovl_su3.cuh"

namespace ovl {

constexpr int kPk3RecVec = 14;  // float4 per link record: 9 (re, re, im, im) + 9 (-im, -im) pairs, padded

// The matrix a hop applies: dir 0..2 the link U_mu(site), 3..5 the dagger of
// U_mu(site - mu).  Record: rec[3 i + j] = (re, re, im, im) of A_ij; then the
// pairs (-im A_ij, -im A_ij) at float2 index 3 i + j of rec + 9.
template <bool U1>
__device__ __forceinline__ void build_link_record3(const float4 *__restrict__ U32, const float2 *__restrict__ u1,
                                                   const Lattice &L, int site, int dir, float4 *__restrict__ rec) {
    const int mu = dir % 3;
    int ls = site;
    if (dir >= 3) {
        const Nbrs n = neighbours(L, site);
        ls = mu == 0 ? n.xm : (mu == 1 ? n.ym : n.zm);
    }
    const cmat3<float> M = Links3<true, U1>{U32, u1, L.N0 * L.N1}.template get<float>(ls, mu);
    float2 *nim = reinterpret_cast<float2 *>(rec + 9);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const cpx<float> a = dir >= 3 ? conj(M.m[j][i]) : M.m[i][j];
            rec[3 * i + j] = make_float4(a.re, a.re, a.im, a.im);
            nim[3 * i + j] = make_float2(-a.im, -a.im);
        }
    nim[9] = make_float2(0.0f, 0.0f);
}

// Row i of k0 = A h0, k1 = A h1 for colour three-vectors of pairs.
__device__ __forceinline__ void pmul3_row(const float4 *__restrict__ rec, int i, const cpair (&h0)[kColours3],
                                          const cpair (&h1)[kColours3], cpair &k0, cpair &k1) {
    const float2 *nim = reinterpret_cast<const float2 *>(rec + 9);
    const float4 a0 = rec[3 * i], a1 = rec[3 * i + 1], a2 = rec[3 * i + 2];
    const float2 n0 = nim[3 * i], n1 = nim[3 * i + 1], n2 = nim[3 * i + 2];
    const float2 r0 = pr(a0.x, a0.y), r1 = pr(a1.x, a1.y), r2 = pr(a2.x, a2.y);
    const float2 m0 = pr(a0.z, a0.w), m1 = pr(a1.z, a1.w), m2 = pr(a2.z, a2.w);
    k0.R = __ffma2_rn(r0, h0[0].R, __ffma2_rn(n0, h0[0].I, __ffma2_rn(r1, h0[1].R, __ffma2_rn(n1, h0[1].I,
           __ffma2_rn(r2, h0[2].R, __fmul2_rn(n2, h0[2].I))))));
    k0.I = __ffma2_rn(r0, h0[0].I, __ffma2_rn(m0, h0[0].R, __ffma2_rn(r1, h0[1].I, __ffma2_rn(m1, h0[1].R,
           __ffma2_rn(r2, h0[2].I, __fmul2_rn(m2, h0[2].R))))));
    k1.R = __ffma2_rn(r0, h1[0].R, __ffma2_rn(n0, h1[0].I, __ffma2_rn(r1, h1[1].R, __ffma2_rn(n1, h1[1].I,
           __ffma2_rn(r2, h1[2].R, __fmul2_rn(n2, h1[2].I))))));
    k1.I = __ffma2_rn(r0, h1[0].I, __ffma2_rn(m0, h1[0].R, __ffma2_rn(r1, h1[1].I, __ffma2_rn(m1, h1[1].R,
           __ffma2_rn(r2, h1[2].I, __fmul2_rn(m2, h1[2].R))))));
}

// The projections of pproject (ovl_packed.cuh) for three colours.
template <int MU, bool FWD>
__device__ __forceinline__ void pproject3(const float4 (&v)[kComp3], cpair (&h0)[kColours3],
                                          cpair (&h1)[kColours3]) {
#pragma unroll
    for (int c = 0; c < kColours3; c++) {
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

// acc -= the rebuilt four-spinor of the hop (pmulacc of ovl_packed.cuh, three
// colours), row by row, so one row of products is live at a time.
template <int MU, bool FWD>
__device__ __forceinline__ void pmulacc3(cpair (&acc)[kColours3][kSpin], const cpair (&h0)[kColours3],
                                         const cpair (&h1)[kColours3], const float4 *__restrict__ rec) {
#pragma unroll
    for (int c = 0; c < kColours3; c++) {
        cpair k0, k1;
        pmul3_row(rec, c, h0, h1, k0, k1);
        cpair *a = acc[c];
        a[0].R = psub(a[0].R, k0.R);
        a[0].I = psub(a[0].I, k0.I);
        a[1].R = psub(a[1].R, k1.R);
        a[1].I = psub(a[1].I, k1.I);
        if (MU == 0) {  // forward: spin 2 = -i h1, spin 3 = -i h0; backward: +i
            a[2].R = FWD ? psub(a[2].R, k1.I) : padd(a[2].R, k1.I);
            a[2].I = FWD ? padd(a[2].I, k1.R) : psub(a[2].I, k1.R);
            a[3].R = FWD ? psub(a[3].R, k0.I) : padd(a[3].R, k0.I);
            a[3].I = FWD ? padd(a[3].I, k0.R) : psub(a[3].I, k0.R);
        } else if (MU == 1) {  // forward: spin 2 = -h1, spin 3 = +h0; backward: +h1, -h0
            a[2].R = FWD ? padd(a[2].R, k1.R) : psub(a[2].R, k1.R);
            a[2].I = FWD ? padd(a[2].I, k1.I) : psub(a[2].I, k1.I);
            a[3].R = FWD ? psub(a[3].R, k0.R) : padd(a[3].R, k0.R);
            a[3].I = FWD ? psub(a[3].I, k0.I) : padd(a[3].I, k0.I);
        } else {  // forward: spin 2 = -i h0, spin 3 = +i h1; backward: +i h0, -i h1
            a[2].R = FWD ? psub(a[2].R, k0.I) : padd(a[2].R, k0.I);
            a[2].I = FWD ? padd(a[2].I, k0.R) : psub(a[2].I, k0.R);
            a[3].R = FWD ? padd(a[3].R, k1.I) : psub(a[3].R, k1.I);
            a[3].I = FWD ? psub(a[3].I, k1.R) : padd(a[3].I, k1.R);
        }
    }
}

template <bool COH = false>
__device__ __forceinline__ void load_spinor4_3(const float4 *__restrict__ p, float4 (&v)[kComp3]) {
#pragma unroll
    for (int k = 0; k < kComp3; k++) v[k] = COH ? __ldca(p + k * (kModeBlock / 2)) : __ldg(p + k * (kModeBlock / 2));
}

// The constants of the overlap-combination epilogue (MODE 3 of packed_tile3,
// OverlapU.cpp:188-202) with D chi the stencil on src:
// o = mdw [ -i g0 cp phi + cm D chi ] into out (accumulate 0) or out += dt o
// (accumulate 1).
struct ClenshawArgs {
    const float4 *phi;
    float mdw, cp, cm, dt;
    int accumulate;
};

// One CTA's tile: sites [site0, site0 + 2W) x mode blocks [mb0, mb1) of src
// and dst (float4 views, mode block 0 at the pointers).  MODE 0: dst = D src;
// 1: dst += dt D src (hdt = dt / 2: the 1/2 of D folded in, exact); 3: the
// overlap combination (cl).  COH: src is written elsewhere in the same launch
// (coherent loads).  Every thread of the CTA calls it (it holds a barrier).
template <int MODE, bool U1, int W, bool COH = false>
__device__ __forceinline__ void packed_tile3(float4 (*__restrict__ rec)[6][kPk3RecVec],
                                             const float4 *__restrict__ U32, const float2 *__restrict__ u1,
                                             const float4 *__restrict__ src, float4 *__restrict__ dst,
                                             const Lattice &L, int site0, int mb0, int mb1, float amass, float hdt,
                                             const ClenshawArgs &cl) {
    const int t = threadIdx.y * kModeBlock + threadIdx.x;
    const int sl = 2 * threadIdx.y + (threadIdx.x >> 4), q = threadIdx.x & 15;
    const int site = site0 + sl;
    const bool live = site < L.V;
    // float4 index of component 0 of (mb, s) for this thread's lane pair
    auto at = [&](int mb, int s) { return (((size_t)mb * L.V + s) * kComp3) * (kModeBlock / 2) + q; };
    if (t < 2 * W * 6) {
        const int s = site0 + t / 6;
        if (s < L.V) build_link_record3<U1>(U32, u1, L, s, t % 6, rec[t / 6][t % 6]);
    }
    __syncthreads();
    if (!live) return;
    const Nbrs n = neighbours(L, site);
    const float4(*r)[kPk3RecVec] = rec[sl];
    for (int mb = mb0; mb < mb1; mb++) {
        float4 v[kComp3];
        load_spinor4_3<COH>(src + at(mb, site), v);
        cpair acc[kColours3][kSpin];
#pragma unroll
        for (int c = 0; c < kColours3; c++)
#pragma unroll
            for (int a = 0; a < kSpin; a++) {
                const float4 f = v[c * kSpin + a];
                acc[c][a].R = pr(amass * f.x, amass * f.z);
                acc[c][a].I = pr(amass * f.y, amass * f.w);
            }
        cpair h0[kColours3], h1[kColours3];
        load_spinor4_3<COH>(src + at(mb, n.xp), v);
        pproject3<0, true>(v, h0, h1);
        load_spinor4_3<COH>(src + at(mb, n.xm), v);
        pmulacc3<0, true>(acc, h0, h1, r[0]);
        pproject3<0, false>(v, h0, h1);
        load_spinor4_3<COH>(src + at(mb, n.yp), v);
        pmulacc3<0, false>(acc, h0, h1, r[3]);
        pproject3<1, true>(v, h0, h1);
        load_spinor4_3<COH>(src + at(mb, n.ym), v);
        pmulacc3<1, true>(acc, h0, h1, r[1]);
        pproject3<1, false>(v, h0, h1);
        load_spinor4_3<COH>(src + at(mb, n.zp), v);
        pmulacc3<1, false>(acc, h0, h1, r[4]);
        pproject3<2, true>(v, h0, h1);
        load_spinor4_3<COH>(src + at(mb, n.zm), v);
        pmulacc3<2, true>(acc, h0, h1, r[2]);
        pproject3<2, false>(v, h0, h1);
        pmulacc3<2, false>(acc, h0, h1, r[5]);
        // -i gamma_0 / 2: spins 0, 1 times -i/2, spins 2, 3 times +i/2
        const size_t o = at(mb, site);
#pragma unroll
        for (int c = 0; c < kColours3; c++)
#pragma unroll
            for (int a = 0; a < kSpin; a++) {
                const cpair &x = acc[c][a];
                const float sg = a < 2 ? 1.0f : -1.0f;
                const size_t i = o + (c * kSpin + a) * (kModeBlock / 2);
                if (MODE == 0) {
                    const float h = 0.5f * sg;
                    dst[i] = make_float4(h * x.I.x, -h * x.R.x, h * x.I.y, -h * x.R.y);
                } else if (MODE == 1) {
                    const float h = hdt * sg;
                    const float4 d = dst[i];
                    dst[i] = make_float4(fmaf(h, x.I.x, d.x), fmaf(-h, x.R.x, d.y), fmaf(h, x.I.y, d.z),
                                         fmaf(-h, x.R.y, d.w));
                } else {  // MODE 3
                    // -i g0 phi = sg (im, -re);  D chi = (1/2) sg (I, -R)
                    const float4 f = __ldg(cl.phi + i);
                    const float g = cl.mdw * sg, hc = 0.5f * cl.cm;
                    const float4 o4 = make_float4(g * fmaf(cl.cp, f.y, hc * x.I.x), -g * fmaf(cl.cp, f.x, hc * x.R.x),
                                                  g * fmaf(cl.cp, f.w, hc * x.I.y), -g * fmaf(cl.cp, f.z, hc * x.R.y));
                    if (cl.accumulate) {
                        const float4 d = dst[i];
                        dst[i] = make_float4(fmaf(cl.dt, o4.x, d.x), fmaf(cl.dt, o4.y, d.y), fmaf(cl.dt, o4.z, d.z),
                                             fmaf(cl.dt, o4.w, d.w));
                    } else {
                        dst[i] = o4;
                    }
                }
            }
    }
}

}  // namespace ovl
