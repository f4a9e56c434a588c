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

// Where the hop kernels read links from.  LinksF64: the FP64 4-real links
// (converted to the arithmetic precision at use); LinksF32: an FP32 copy kept
// next to them for the FP32 path (one 16-byte load per link, no conversion).
// Both give the same matrices: each component is rounded to T once.  U1: the
// x and y links carry the U(1) background phase (compiled in only when set).
template <bool U1> struct LinksF64 {
    const double *U;
    const double2 *u1;
    int n01;
    template <typename T> __device__ __forceinline__ cmat2<T> get(int site, int mu) const {
        if (U1) return dressed_link<T>(U, u1, site, mu, n01);
        return link_matrix<T>(load_link(U, site, mu));
    }
};

template <bool U1> struct LinksF32 {
    const float4 *U;
    const float2 *u1;
    int n01;
    template <typename T> __device__ __forceinline__ cmat2<T> get(int site, int mu) const {
        const float4 q = __ldg(U + 3 * site + mu);
        cmat2<T> M = {mk<T>(q.w, q.z), mk<T>(q.y, q.x), mk<T>(-q.y, q.x), mk<T>(q.w, -q.z)};
        if (U1 && mu < 2) {
            const float2 ph = __ldg(u1 + 2 * (site % n01) + mu);
            const cpx<T> p = mk<T>(ph.x, ph.y);
            M.m00 = p * M.m00;
            M.m01 = p * M.m01;
            M.m10 = p * M.m10;
            M.m11 = p * M.m11;
        }
        return M;
    }
};

// Neighbour sites of `site` (periodic).
struct Nbrs {
    int xp, xm, yp, ym, zp, zm;
};
__device__ __forceinline__ Nbrs neighbours(const Lattice &L, int site) {
    int x, y, z;
    site_coords(L, site, x, y, z);
    const int n01 = L.N0 * L.N1, V = L.V;
    Nbrs n;
    n.xp = x + 1 == L.N0 ? site + 1 - L.N0 : site + 1;
    n.xm = x == 0 ? site - 1 + L.N0 : site - 1;
    n.yp = y + 1 == L.N1 ? site + L.N0 - n01 : site + L.N0;
    n.ym = y == 0 ? site - L.N0 + n01 : site - L.N0;
    n.zp = z + 1 == L.N2 ? site + n01 - V : site + n01;
    n.zm = z == 0 ? site - n01 + V : site - n01;
    return n;
}

// The six FP64 link matrices of one site's hops, gathered once per CTA in
// shared memory and reused over the CTA's mode blocks: entries 0..2 the links
// U_mu(site), 3..5 the links U_mu(site - mu) (the backward hop takes their
// dagger itself), each as LK delivers it (dressed with the U(1) phase when one
// is set).  get() is called by the stencil with the site itself for the
// forward hops and with its backward neighbours, which differ from the site on
// every lattice the library accepts (N >= 3).
// Mode blocks a CTA of the FP64 stencils runs on one gathering of its sites'
// links: kLinkBlocks, halved while the grid would hold fewer than 4 CTAs per
// SM (small lattices or few modes); 1 selects the stencil without the table.
constexpr int kLinkBlocks = 8;
inline int link_blocks(int site_ctas, int n_mb, int sm_count) {
    int m = kLinkBlocks;
    while (m > 1 && (long long)site_ctas * ((n_mb + m - 1) / m) < 4LL * sm_count) m /= 2;
    return m;
}
// SMs of the current device (cached per device).
inline int current_sm_count() {
    static int cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
    if (cache[dev] == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 1;
    }
    return cache[dev];
}

struct LinksTable {
    const cmat2<double> *t;
    int site;
    template <typename T> __device__ __forceinline__ cmat2<T> get(int s, int mu) const {
        static_assert(sizeof(T) == 8, "the link table holds FP64 matrices");
        return t[(s == site ? 0 : 3) + mu];
    }
};

// Fills tab[j][dir] for the CTA's sites site_of(j) (j < SITES; a negative
// site: none) from lk; every thread of the CTA calls it (it holds a barrier).
template <int SITES, class LK, class SiteOf>
__device__ __forceinline__ void fill_link_table(const LK &lk, const Lattice &L, const SiteOf &site_of,
                                                cmat2<double> (*tab)[6]) {
    const int t = threadIdx.y * kModeBlock + threadIdx.x;
    if (t < SITES * 6) {
        const int s = site_of(t / 6), dir = t % 6, mu = dir % 3;
        if (s >= 0) {
            int ls = s;
            if (dir >= 3) {
                const Nbrs n = neighbours(L, s);
                ls = mu == 0 ? n.xm : (mu == 1 ? n.ym : n.zm);
            }
            tab[t / 6][dir] = lk.template get<double>(ls, mu);
        }
    }
    __syncthreads();
}

// (D phi)(site) for the 32 modes of block mb (one per lane), before the
// -i gamma_0 / 2 factor: amass phi(x) - sum of the six projected hops.
template <typename T, class LK>
__device__ __forceinline__ void wilson_site_lk(const LK &lk, const cpx<T> *__restrict__ src, const Lattice &L, int site,
                                               int mb, int lane, T amass, Spinor<T> &acc) {
    const int V = L.V;
    const Nbrs n = neighbours(L, site);
    Spinor<T> f;
    load_spinor(src, V, mb, site, lane, f);
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) acc.c[c][a] = amass * f.c[c][a];
    load_spinor(src, V, mb, n.xp, lane, f);
    hop<T, 0, true>(acc, f, lk.template get<T>(site, 0));
    load_spinor(src, V, mb, n.xm, lane, f);
    hop<T, 0, false>(acc, f, lk.template get<T>(n.xm, 0));
    load_spinor(src, V, mb, n.yp, lane, f);
    hop<T, 1, true>(acc, f, lk.template get<T>(site, 1));
    load_spinor(src, V, mb, n.ym, lane, f);
    hop<T, 1, false>(acc, f, lk.template get<T>(n.ym, 1));
    load_spinor(src, V, mb, n.zp, lane, f);
    hop<T, 2, true>(acc, f, lk.template get<T>(site, 2));
    load_spinor(src, V, mb, n.zm, lane, f);
    hop<T, 2, false>(acc, f, lk.template get<T>(n.zm, 2));
}

template <typename T>
__device__ __forceinline__ void wilson_site(const double *__restrict__ links, const double2 *__restrict__ u1,
                                            const cpx<T> *__restrict__ src, const Lattice &L, int site, int mb,
                                            int lane, T amass, Spinor<T> &acc) {
    if (u1 != nullptr) wilson_site_lk(LinksF64<true>{links, u1, L.N0 * L.N1}, src, L, site, mb, lane, amass, acc);
    else wilson_site_lk(LinksF64<false>{links, nullptr, L.N0 * L.N1}, src, L, site, mb, lane, amass, acc);
}

// Component (c, a) of -i gamma_0 / 2 acc: spins 0,1 times -i/2, spins 2,3 times +i/2.
template <typename T> __device__ __forceinline__ cpx<T> finish_component(const cpx<T> &v, int a) {
    const cpx<T> d = a < 2 ? times_mi(v) : times_i(v);
    return (T)0.5 * d;
}

}  // namespace ovl
