// Ensembles: independent trajectories (members) of their own lattice size,
// mode count and colour count, stepped together.  One launch per group of
// members (colours x U(1) background, at most kParamMembers each) advances
// their hop work by a half step and one launch updates every member's links,
// so a leapfrog step of the whole ensemble is a handful of kernels (the half
// steps, two link updates, the step counters), captured once as a CUDA graph.
//
// Work is cut into tiles of SITES sites x one block of 32 modes (a warp per
// site, as the single-trajectory kernels); tiles are numbered member by member
// and a CTA finds its member by binary search over the members' first tiles.
// The Update.cpp:57 gate (links move while qs t < tSphaleron) is evaluated on
// the device from each member's step counter, so the captured step needs no
// host decisions.
#include "ovl_fp40.cuh"
#include "ovl_internal.h"
#include "ovl_packed.cuh"
#include "ovl_stencil.cuh"
#include "ovl_su3.cuh"

namespace ovl {

__device__ __forceinline__ int find_member(const BatchMember *__restrict__ m, int count, long long key,
                                           long long BatchMember::*first) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {  // last member whose first index <= key
        const int mid = (lo + hi + 1) >> 1;
        if (m[mid].*first <= key) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// CTAs per SM the register allocation must allow: FP32 64 registers, FP64 128
// (as the single-context kernels).
template <typename T, int SITES> struct BatchOcc {
    static constexpr int kMinBlocks = (sizeof(T) == 4 ? 1024 : 512) / (kModeBlock * SITES);
};

// phase 0: psi += dt D psimid; phase 1: psimid += dt D psi.  One launch covers
// the members of one group (all with a U(1) background, U1, or all without;
// at most kParamMembers), their descriptors passed by value (kernel parameter
// space, read through the constant cache: no dependent global loads before a
// CTA finds its member); tiles numbered on from the first member's tile0.
template <typename T, int SITES, bool U1>
__global__ void __launch_bounds__(kModeBlock *SITES, BatchOcc<T, SITES>::kMinBlocks)
    wilson_batch_param_kernel(const __grid_constant__ BatchGroup g, int phase) {
    const long long key = (long long)blockIdx.x + g.m[0].tile0;
    int lo = 0, hi = g.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (g.m[mid].tile0 <= key) lo = mid;
        else hi = mid - 1;
    }
    const BatchMember &m = g.m[lo];
    const Lattice L{m.N0, m.N1, m.N2, m.V};
    const int nsb = (L.V + SITES - 1) / SITES;
    // a member's tiles number below 2^31: two fields of 32 B per mode-site and colour
    // in 180 GB hold at most ~1.4e9 mode-sites, ~1.1e7 tiles of 4 sites x 32 modes
    const int local = (int)(key - m.tile0);
    const int mb = local / nsb;
    const int site = (local - mb * nsb) * SITES + threadIdx.y;
    if (site >= L.V) return;
    const int lane = threadIdx.x;
    const cpx<T> *src = reinterpret_cast<const cpx<T> *>(phase == 0 ? m.psimid : m.psi);
    cpx<T> *dst = reinterpret_cast<cpx<T> *>(phase == 0 ? m.psi : m.psimid);
    const int n01 = L.N0 * L.N1;
    Spinor<T> acc;
    if constexpr (sizeof(T) == 4)
        wilson_site_lk(LinksF32<U1>{reinterpret_cast<const float4 *>(m.U32), reinterpret_cast<const float2 *>(m.u1_32),
                                    n01},
                       src, L, site, mb, lane, (T)m.amass, acc);
    else
        wilson_site_lk(LinksF64<U1>{m.U, reinterpret_cast<const double2 *>(m.u1), n01}, src, L, site, mb, lane,
                       (T)m.amass, acc);
    cpx<T> *out = dst + field_index(L.V, mb, site, 0, lane);
    const T dt = (T)m.dt;
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) {
            const cpx<T> d = finish_component(acc.c[c][a], a);
            cpx<T> *o = out + (c * kSpin + a) * kModeBlock;
            const cpx<T> v = ld(o);
            st(o, v + dt * d);
        }
}

// FP32 two-colour members in packed-pair tiles: a CTA covers kBatchPkSites
// sites x kPkBlocks mode blocks of one member with the arithmetic and shape
// of hop variant 3 (packed_tile: two modes per thread on the paired FP32
// instructions, the tile's links built once in shared memory, CTAs of
// kBatchPkWarps warps with two neighbour spinors in flight per thread).
constexpr int kBatchPkWarps = 4, kBatchPkSites = 2 * kBatchPkWarps;

template <bool U1>
__global__ void __launch_bounds__(kModeBlock *kBatchPkWarps, 3)
    wilson_batch_packed_kernel(const __grid_constant__ BatchGroup g, int phase) {
    __shared__ float4 rec[kBatchPkSites][6][kPkRecVec];
    const long long key = (long long)blockIdx.x + g.m[0].tile0;
    int lo = 0, hi = g.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (g.m[mid].tile0 <= key) lo = mid;
        else hi = mid - 1;
    }
    const BatchMember &m = g.m[lo];
    const Lattice L{m.N0, m.N1, m.N2, m.V};
    const int nst = (L.V + kBatchPkSites - 1) / kBatchPkSites;
    const int local = (int)(key - m.tile0);  // below 2^31 (see wilson_batch_param_kernel)
    const int mbt = local / nst;
    const int mb0 = mbt * kPkBlocks;
    const float4 *src = reinterpret_cast<const float4 *>(phase == 0 ? m.psimid : m.psi);
    float4 *dst = reinterpret_cast<float4 *>(phase == 0 ? m.psi : m.psimid);
    double o[kObsVals] = {0.0, 0.0, 0.0};  // not observing
    packed_tile<1, U1, false, kBatchPkWarps, 2>(rec, reinterpret_cast<const float4 *>(m.U32),
                                                reinterpret_cast<const float2 *>(m.u1_32), src, dst, L,
                                                (local - mbt * nst) * kBatchPkSites, mb0, min(m.n_mb, mb0 + kPkBlocks),
                                                (float)m.amass, (float)(0.5 * m.dt), 0, 0, o);
}

// Three-colour members (SU(3) links, 12-component modes), one group per U(1)
// setting; descriptors by value as above.  FP32 modes read the padded FP32
// link copy, FP64 modes the FP64 links.
template <typename T, int SITES, bool U1>
__global__ void __launch_bounds__(kModeBlock *SITES, BatchOcc<T, SITES>::kMinBlocks / 2)
    wilson_batch3_kernel(const __grid_constant__ BatchGroup g, int phase) {
    const long long key = (long long)blockIdx.x + g.m[0].tile0;
    int lo = 0, hi = g.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (g.m[mid].tile0 <= key) lo = mid;
        else hi = mid - 1;
    }
    const BatchMember &m = g.m[lo];
    const Lattice L{m.N0, m.N1, m.N2, m.V};
    const int nsb = (L.V + SITES - 1) / SITES;
    // a member's tiles number below 2^31: two fields of 32 B per mode-site and colour
    // in 180 GB hold at most ~1.4e9 mode-sites, ~1.1e7 tiles of 4 sites x 32 modes
    const int local = (int)(key - m.tile0);
    const int mb = local / nsb;
    const int site = (local - mb * nsb) * SITES + threadIdx.y;
    if (site >= L.V) return;
    const int lane = threadIdx.x;
    const cpx<T> *src = reinterpret_cast<const cpx<T> *>(phase == 0 ? m.psimid : m.psi);
    cpx<T> *dst = reinterpret_cast<cpx<T> *>(phase == 0 ? m.psi : m.psimid);
    constexpr bool F32 = sizeof(T) == 4;
    const Links3<F32, U1> lk{F32 ? (const void *)m.U32 : (const void *)m.U, F32 ? (const void *)m.u1_32 : (const void *)m.u1,
                             L.N0 * L.N1};
    Spinor3<T> acc;
    wilson_site3(lk, src, L, site, mb, lane, (T)m.amass, acc);
    cpx<T> *out = dst + field_index3(L.V, mb, site, 0, lane);
    const T dt = (T)m.dt;
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) {
            const cpx<T> v = acc.c[c][a];
            const cpx<T> d = (T)0.5 * (a < 2 ? times_mi(v) : times_i(v));
            cpx<T> *o = out + (c * kSpin + a) * kModeBlock;
            st(o, ld(o) + dt * d);
        }
}

// Link updates of every member, U <- exp(-i dt/2 E^a t^a) U where the member's
// links move (Update.cpp:57 on its own step counter), with the FP32 copy kept.
__global__ void links_batch_kernel(const BatchMember *__restrict__ members, int count, long long total) {
    const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (l >= total) return;
    const int mi = find_member(members, count, l, &BatchMember::link0);
    const BatchMember &m = members[mi];
    const int k = (int)(l - m.link0);  // link of the member: 3 site + mu
    if (!(m.qs * (*m.tsteps * m.dt) < m.t_sphaleron)) return;
    if (m.nc == 3) {  // SU(3): Dynamics.cpp:97-138 with the 3x3 exponential
        const int site = k / 3, mu = k % 3;
        cmat3<double> u = m3_mul(su3_exp(-0.5 * m.dt, m.E + 8 * (size_t)k), load_su3(m.U, site, mu));
        if (m.reunit) u = su3_reunitarize(u);
        store_su3(m.U, site, mu, u);
        if (m.U32) {
            float2 *p = reinterpret_cast<float2 *>(m.U32 + (size_t)kLink32Floats * k);
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) p[i + 3 * j] = float2{(float)u.m[i][j].re, (float)u.m[i][j].im};
            p[9] = float2{0.0f, 0.0f};
        }
        return;
    }
    const double *e = m.E + 3 * k;
    const quat g = qexp(-0.5 * m.dt, e[0], e[1], e[2]);
    const int site = k / 3, mu = k % 3;
    quat u = qmul(g, load_link(m.U, site, mu));
    if (m.reunit) {
        const double nrm = sqrt(u.v0 * u.v0 + u.v1 * u.v1 + u.v2 * u.v2 + u.s * u.s);
        u = {u.v0 / nrm, u.v1 / nrm, u.v2 / nrm, u.s / nrm};
    }
    store_link(m.U, site, mu, u);
    if (m.U32) reinterpret_cast<float4 *>(m.U32)[k] = float4{(float)u.v0, (float)u.v1, (float)u.v2, (float)u.s};
}

__global__ void advance_batch_kernel(const BatchMember *__restrict__ members, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) *members[i].tsteps += 1;
}

long long batch_tiles(int V, int n_mb, int sites, int nc, bool fp32) {
    if (sites == kBatchPacked) {
        if (nc == 2 && fp32)
            return (long long)((V + kBatchPkSites - 1) / kBatchPkSites) * ((n_mb + kPkBlocks - 1) / kPkBlocks);
        sites = 8;
    }
    return (long long)((V + sites - 1) / sites) * n_mb;
}

template <int SITES, bool U1>
static void launch_hop_param(const BatchGroup &g, long long tiles, int phase, bool fp32, cudaStream_t s, int nc) {
    const dim3 block(kModeBlock, SITES);
    if (nc == 3) {
        if (fp32) wilson_batch3_kernel<float, SITES, U1><<<(unsigned)tiles, block, 0, s>>>(g, phase);
        else wilson_batch3_kernel<double, SITES, U1><<<(unsigned)tiles, block, 0, s>>>(g, phase);
        return;
    }
    if (fp32) wilson_batch_param_kernel<float, SITES, U1><<<(unsigned)tiles, block, 0, s>>>(g, phase);
    else wilson_batch_param_kernel<double, SITES, U1><<<(unsigned)tiles, block, 0, s>>>(g, phase);
}

template <bool U1> static void launch_hop_packed(const BatchGroup &g, long long tiles, int phase, cudaStream_t s) {
    wilson_batch_packed_kernel<U1><<<(unsigned)tiles, dim3(kModeBlock, kBatchPkWarps), 0, s>>>(g, phase);
}

void launch_batch_hop_param(const BatchGroup &g, long long tiles, int sites, int phase, bool fp32, bool u1,
                            cudaStream_t stream, int nc) {
    if (g.count <= 0 || tiles <= 0) return;
    if (sites == kBatchPacked) {
        if (nc == 2 && fp32) {
            if (u1) launch_hop_packed<true>(g, tiles, phase, stream);
            else launch_hop_packed<false>(g, tiles, phase, stream);
            return;
        }
        sites = 8;
    }
    if (u1) {
        if (sites == 4) launch_hop_param<4, true>(g, tiles, phase, fp32, stream, nc);
        else launch_hop_param<8, true>(g, tiles, phase, fp32, stream, nc);
    } else {
        if (sites == 4) launch_hop_param<4, false>(g, tiles, phase, fp32, stream, nc);
        else launch_hop_param<8, false>(g, tiles, phase, fp32, stream, nc);
    }
}

void launch_batch_links(const BatchMember *members, int count, long long total_links, cudaStream_t stream) {
    links_batch_kernel<<<(unsigned)((total_links + 255) / 256), 256, 0, stream>>>(members, count, total_links);
}

void launch_batch_advance(const BatchMember *members, int count, cudaStream_t stream) {
    advance_batch_kernel<<<(count + 127) / 128, 128, 0, stream>>>(members, count);
}

}  // namespace ovl
