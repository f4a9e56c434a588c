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

#include <algorithm>
#include <type_traits>

#include "ovl_fp40.cuh"
#include "ovl_internal.h"
#include "ovl_packed.cuh"
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

// Variants of the same half step for the autotuner (identical arithmetic):
//   VARIANT 0  one site per warp, the 8 warps of a CTA on 8 consecutive sites
//   VARIANT 1  one site per warp, the 8 warps of a CTA on a 4 x 2 (x, y) tile, so
//              that x and y neighbours are read by warps of the same CTA (L1)
//   VARIANT 2  one (x, y) column per thread marching in z: the z neighbours and
//              the site itself come from registers (5 spinor loads per site
//              instead of 7)
// LK selects FP64 links or the FP32 copy (FP32 path).
template <typename T, int MODE>
__device__ __forceinline__ void store_result(cpx<T> *__restrict__ dst, int V, int mb, int site, int lane,
                                             const Spinor<T> &acc, T dt) {
    cpx<T> *out = dst + field_index(V, mb, site, 0, lane);
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

// CTAs of 8 warps per SM the compiler must fit: FP32 4 (<= 64 registers), FP64 2.
template <typename T, int VARIANT> struct HopOccupancy {
    static constexpr int kMinBlocks = sizeof(T) == 4 ? 4 : 2;
};

constexpr int kTileX = 4, kTileY = kSitesPerCta / kTileX;  // the (x, y) tile of variant 1

// TABLE (FP64, variants 0 and 1): a CTA runs its 8 sites for mblk mode blocks
// [mblk blockIdx.y, ...) of the n_mb, with the sites' links gathered once in
// shared memory (fill_link_table): the link loads and the U(1) dressing are
// done once per CTA instead of once per mode block.
template <typename T, int MODE, int VARIANT, class LK, bool TABLE = false>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta, HopOccupancy<T, VARIANT>::kMinBlocks)
    wilson_tuned_kernel(LK lk, const cpx<T> *__restrict__ src, cpx<T> *__restrict__ dst, Lattice L, T amass, T dt,
                        int n_mb = 0, int mblk = 1) {
    const int lane = threadIdx.x;
    // the site of warp j of this CTA, or -1
    auto site_of = [&](int j) {
        if (VARIANT == 1) {
            const int ntx = (L.N0 + kTileX - 1) / kTileX, nty = (L.N1 + kTileY - 1) / kTileY;
            const int t = blockIdx.x;
            const int x = (t % ntx) * kTileX + j % kTileX;
            const int y = ((t / ntx) % nty) * kTileY + j / kTileX;
            const int z = t / (ntx * nty);
            return x < L.N0 && y < L.N1 ? x + L.N0 * (y + L.N1 * z) : -1;
        }
        const int s = blockIdx.x * kSitesPerCta + j;
        return s < L.V ? s : -1;
    };
    const int site = site_of(threadIdx.y);
    if constexpr (TABLE) {
        static_assert(VARIANT <= 1 && sizeof(T) == 8, "the link table serves the FP64 tiles");
        __shared__ cmat2<double> tab[kSitesPerCta][6];
        fill_link_table<kSitesPerCta>(lk, L, site_of, tab);
        if (site < 0) return;
        const LinksTable lt{tab[threadIdx.y], site};
        const int mb0 = blockIdx.y * mblk, mb1 = min(n_mb, mb0 + mblk);
        for (int mb = mb0; mb < mb1; mb++) {
            Spinor<T> acc;
            wilson_site_lk(lt, src, L, site, mb, lane, amass, acc);
            store_result<T, MODE>(dst, L.V, mb, site, lane, acc, dt);
        }
        return;
    }
    const int mb = blockIdx.y;
    if (site < 0) return;
    Spinor<T> acc;
    wilson_site_lk(lk, src, L, site, mb, lane, amass, acc);
    store_result<T, MODE>(dst, L.V, mb, site, lane, acc, dt);
}

// ------------------------------------------------- observing half step --
// The CTA's sums of o (warp shuffles, then the warps in a fixed order) into
// row[0..kObsVals) (thread (0, 0) writes).
__device__ __forceinline__ void cta_sum_row(double (&o)[kObsVals], double *__restrict__ row) {
    __shared__ double sh[kSitesPerCta][kObsVals];
#pragma unroll
    for (int k = 0; k < kObsVals; k++) {
        double t = o[k];
        for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
        o[k] = t;
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < kObsVals; k++) sh[threadIdx.y][k] = o[k];
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int k = 0; k < kObsVals; k++) {
            double t = 0.0;
            for (int j = 0; j < (int)blockDim.y; j++) t += sh[j][k];  // the CTA's warps (at most kSitesPerCta)
            row[k] = t;
        }
    }
    __syncthreads();  // sh is reused by the CTA's next call
}

// Per-CTA sums into partial, one row per CTA of the grid.
__device__ __forceinline__ void cta_partial(double (&o)[kObsVals], double *__restrict__ partial) {
    cta_sum_row(o, partial + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * kObsVals);
}

// The packed-pair half step over all sites and mode blocks (packed_tile):
// CTAs of kPkWarps warps (2 kPkWarps sites), kPkDepth neighbour spinors in
// flight per thread, kPkMinBlocks CTAs per SM.
constexpr int kPkWarps = 4, kPkDepth = 2, kPkMinBlocks = 3;
constexpr int kPkCtaSites = 2 * kPkWarps;

template <int MODE, bool U1, bool OBS>
__global__ void __launch_bounds__(kModeBlock *kPkWarps, kPkMinBlocks)
    wilson_packed_kernel(const float4 *__restrict__ U32, const float2 *__restrict__ u1, const float4 *__restrict__ src,
                         float4 *__restrict__ dst, Lattice L, int n_mb, float amass, float hdt, int n_modes,
                         int first_mode, double *__restrict__ partial) {
    __shared__ float4 rec[kPkCtaSites][6][kPkRecVec];
    const int mb0 = blockIdx.y * kPkBlocks;
    double o[kObsVals] = {0.0, 0.0, 0.0};
    packed_tile<MODE, U1, OBS, kPkWarps, kPkDepth>(rec, U32, u1, src, dst, L, blockIdx.x * kPkCtaSites, mb0,
                                                   min(n_mb, mb0 + kPkBlocks), amass, hdt, n_modes, first_mode, o);
    if (OBS) cta_partial(o, partial);
}


// Rows of kObsVals partial sums the packed observing launch writes.
size_t packed_obs_rows(const Lattice &L, int n_mb) {
    return (size_t)((L.V + kPkCtaSites - 1) / kPkCtaSites) * ((n_mb + kPkBlocks - 1) / kPkBlocks);
}

template <int MODE, bool OBS>
static void launch_packed(const HopConfig &hc, const void *src, void *dst, const Lattice &L, int n_mb, double amass,
                          double dt, int n_modes, int first_mode, double *partial, cudaStream_t stream) {
    const dim3 block(kModeBlock, kPkWarps),
        grid((L.V + kPkCtaSites - 1) / kPkCtaSites, (n_mb + kPkBlocks - 1) / kPkBlocks);
    const float4 *U = reinterpret_cast<const float4 *>(hc.U32);
    const float4 *s = reinterpret_cast<const float4 *>(src);
    float4 *d = reinterpret_cast<float4 *>(dst);
    const float a = (float)amass, h = (float)(0.5 * dt);
    if (hc.u1_32)
        wilson_packed_kernel<MODE, true, OBS><<<grid, block, 0, stream>>>(
            U, reinterpret_cast<const float2 *>(hc.u1_32), s, d, L, n_mb, a, h, n_modes, first_mode, partial);
    else
        wilson_packed_kernel<MODE, false, OBS><<<grid, block, 0, stream>>>(U, nullptr, s, d, L, n_mb, a, h, n_modes,
                                                                          first_mode, partial);
}

// ---------------------------------------------- pipelined grouped step --
// The grouped fused step (both half steps, group by group of `group` mode
// blocks) in one persistent launch of the packed-pair tile: CTAs take tiles
// (16 sites x the group's mode blocks, of one half step) by ticket, in the
// order
//   H1(0), H1(1), H2(0), H1(2), H2(1), ..., H1(n-1), H2(n-2), H2(n-1)
// (H1: b += dt D a with links U1; H2: c += dt D b with links U2), so that a
// group's second half step runs two phases after its first, while the group's
// fields are still in L2: 4 instead of 6 passes over HBM per leapfrog step.
// A tile of H2(g) waits until every tile of H1(g) is done (a counter per
// group, released after the tile's stores); those tiles hold earlier tickets,
// taken by running CTAs whose H1 tiles never wait, so the wait ends.  It is
// bounded all the same (wait_count: 1 s of the GPU's %globaltimer, or a
// poll count, whichever comes first): the CTA then sets the error word and
// leaves the tile undone, and the host reports the step as failed.  Both half steps read fields the launch also writes (H1's source is
// H2's destination, H2's source is H1's destination), so their spinor loads
// are coherent ones (packed_tile with COH), not the read-only path.
struct PipeArgs {
    const float4 *U1, *U2;  // FP32 links of the two half steps
    const float2 *u1;       // U(1) phases or null
    const float4 *a;        // H1 source
    float4 *b, *c;          // H1 destination = H2 source; H2 destination
    Lattice L;
    int n_mb, group, n_groups, tiles;  // tiles per (group, half step)
    float amass, hdt;
    int n_modes, first_mode;
    int *done, *ticket, *err;  // counters: done[n_groups], ticket, error word
    double *partial;           // OBS: kObsVals per (group, tile) of H2
};




template <bool U1, bool OBS>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta, 2) wilson_pipeline_kernel(const __grid_constant__ PipeArgs p) {
    __shared__ float4 rec[kPkSites][6][kPkRecVec];
    __shared__ int s_item, s_go;
    const int t = threadIdx.y * kModeBlock + threadIdx.x;
    const int total = 2 * p.n_groups * p.tiles;
    // the next ticket is taken while the current tile runs (its latency hidden);
    // a CTA works its tickets in increasing order, so the smallest unfinished
    // ticket is always a running tile whose dependencies are done: no deadlock
    int next = 0;
    if (t == 0) next = atomicAdd(p.ticket, 1);
    for (;;) {
        if (t == 0) {
            s_item = next;
            if (next < total) next = atomicAdd(p.ticket, 1);
        }
        __syncthreads();
        const int item = s_item;
        if (item >= total) break;  // the same for every thread of the CTA
        const int j = item / p.tiles, tile = item - j * p.tiles;
        int g, h;
        pipe_phase(j, p.n_groups, g, h);
        if (t == 0) {
            int go = 1;
            if (h == 1) go = wait_count(p.done + g, p.tiles, p.err) ? 1 : 0;
            s_go = go;
        }
        __syncthreads();
        if (s_go) {  // the same for every thread of the CTA
            const int mb0 = g * p.group, mb1 = min(p.n_mb, mb0 + p.group);
            double o[kObsVals] = {0.0, 0.0, 0.0};
            // one inlined tile body for both half steps (links and fields by h)
            packed_tile<1, U1, OBS, kSitesPerCta, 1, true>(rec, h ? p.U2 : p.U1, p.u1, h ? p.b : p.a, h ? p.c : p.b, p.L,
                                                           tile * kPkSites, mb0, mb1, p.amass, p.hdt, p.n_modes,
                                                           p.first_mode, o, h == 1);
            if (OBS && h == 1) cta_sum_row(o, p.partial + ((size_t)g * p.tiles + tile) * kObsVals);
        }
        __syncthreads();  // every thread's stores of the tile are issued
        if (t == 0 && h == 0) red_release_add(p.done + g, 1);
    }
}

int pipeline_counters(int n_mb) { return n_mb + 2; }

size_t pipeline_obs_rows(const Lattice &L, int n_mb, int group) {
    return (size_t)((n_mb + group - 1) / group) * ((L.V + kPkSites - 1) / kPkSites);
}

__global__ void set_int_kernel(int *p, int v) { *p = v; }

void launch_wilson_pipeline(const HopConfig &h1, const HopConfig &h2, const void *a, void *b, void *c,
                            const Lattice &L, int n_mb, int group, double amass, double dt, int *counters, int sm_count,
                            int n_modes, int first_mode, double *partial, cudaStream_t stream, int first_ticket) {
    PipeArgs p;
    p.U1 = reinterpret_cast<const float4 *>(h1.U32);
    p.U2 = reinterpret_cast<const float4 *>(h2.U32);
    p.u1 = reinterpret_cast<const float2 *>(h1.u1_32);
    p.a = reinterpret_cast<const float4 *>(a);
    p.b = reinterpret_cast<float4 *>(b);
    p.c = reinterpret_cast<float4 *>(c);
    p.L = L;
    p.n_mb = n_mb;
    p.group = group;
    p.n_groups = (n_mb + group - 1) / group;
    p.tiles = (L.V + kPkSites - 1) / kPkSites;
    p.amass = (float)amass;
    p.hdt = (float)(0.5 * dt);
    p.n_modes = n_modes;
    p.first_mode = first_mode;
    p.done = counters;
    p.ticket = counters + p.n_groups;
    p.err = counters + n_mb + 1;  // sticky: reset by the caller after it reads it
    p.partial = partial;
    cudaMemsetAsync(counters, 0, sizeof(int) * (p.n_groups + 1), stream);
    if (first_ticket) set_int_kernel<<<1, 1, 0, stream>>>(p.ticket, first_ticket);
    const long long items = 2LL * p.n_groups * p.tiles;
    const int grid = (int)std::min<long long>(items, 2LL * sm_count);  // 2 CTAs per SM (128 registers)
    const dim3 block(kModeBlock, kSitesPerCta);
    if (p.u1) {
        if (partial) wilson_pipeline_kernel<true, true><<<grid, block, 0, stream>>>(p);
        else wilson_pipeline_kernel<true, false><<<grid, block, 0, stream>>>(p);
    } else {
        if (partial) wilson_pipeline_kernel<false, true><<<grid, block, 0, stream>>>(p);
        else wilson_pipeline_kernel<false, false><<<grid, block, 0, stream>>>(p);
    }
}

template <typename T, class LK>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta, HopOccupancy<T, 0>::kMinBlocks)
    wilson_observe_kernel(LK lk, const cpx<T> *__restrict__ src, cpx<T> *__restrict__ dst, Lattice L, T amass, T dt,
                          int n_modes, int first_mode, double *__restrict__ partial) {
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSitesPerCta + threadIdx.y;
    const int mb = blockIdx.y;
    double o[kObsVals] = {0.0, 0.0, 0.0};
    if (site < L.V) {
        Spinor<T> acc;
        wilson_site_lk(lk, src, L, site, mb, lane, amass, acc);
        store_result<T, 1>(dst, L.V, mb, site, lane, acc, dt);
        // the site's own spinor again: an L1 hit, the stencil has just read it
        const int mode = mb * kModeBlock + lane;
        const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
        const cpx<T> *p = src + field_index(L.V, mb, site, 0, lane);
        cpx<double> f[kColours][kSpin];
#pragma unroll
        for (int c = 0; c < kColours; c++)
#pragma unroll
            for (int a = 0; a < kSpin; a++) {
                const cpx<T> v = ld(p + (c * kSpin + a) * kModeBlock);
                f[c][a] = mk<double>((double)v.re, (double)v.im);
            }
        local_charges(f, w, o);
    }
    cta_partial(o, partial);
}

size_t obs_partial_doubles(const Lattice &L, int n_mb) {
    return (size_t)kObsVals * ((L.V + kSitesPerCta - 1) / kSitesPerCta) * n_mb;
}

template <typename T>
size_t launch_wilson_observe(const HopConfig &hc, const void *src, void *dst, const Lattice &L, int n_mb, double amass,
                             double dt, int n_modes, int first_mode, double *partial, cudaStream_t stream) {
    if (std::is_same<T, float>::value && hc.variant == kPackedVariant && hc.U32 != nullptr) {
        launch_packed<1, true>(hc, src, dst, L, n_mb, amass, dt, n_modes, first_mode, partial, stream);
        return packed_obs_rows(L, n_mb);
    }
    const cpx<T> *s = reinterpret_cast<const cpx<T> *>(src);
    cpx<T> *d = reinterpret_cast<cpx<T> *>(dst);
    const dim3 block(kModeBlock, kSitesPerCta), grid((L.V + kSitesPerCta - 1) / kSitesPerCta, n_mb);
    const int n01 = L.N0 * L.N1;
    auto go = [&](const auto &lk) {
        using LK = std::decay_t<decltype(lk)>;
        wilson_observe_kernel<T, LK><<<grid, block, 0, stream>>>(lk, s, d, L, (T)amass, (T)dt, n_modes, first_mode,
                                                                 partial);
    };
    if (std::is_same<T, float>::value && hc.U32 != nullptr) {
        const float4 *u = reinterpret_cast<const float4 *>(hc.U32);
        if (hc.u1_32) go(LinksF32<true>{u, reinterpret_cast<const float2 *>(hc.u1_32), n01});
        else go(LinksF32<false>{u, nullptr, n01});
    } else {
        if (hc.u1) go(LinksF64<true>{hc.U, reinterpret_cast<const double2 *>(hc.u1), n01});
        else go(LinksF64<false>{hc.U, nullptr, n01});
    }
    return obs_partial_doubles(L, n_mb) / kObsVals;
}

// Two-level fixed-order sum of `rows` rows of kObsVals: 256 CTAs sum
// contiguous runs into scratch, one CTA sums those (compensated), scaled.
__global__ void obs_rows_kernel(const double *__restrict__ partial, size_t rows, double *__restrict__ scratch) {
    const size_t per = (rows + gridDim.x - 1) / gridDim.x, r0 = blockIdx.x * per;
    const size_t r1 = r0 + per < rows ? r0 + per : rows;
    __shared__ double sh[kObsVals][256];
    CompSum t[kObsVals];
    for (size_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
        for (int k = 0; k < kObsVals; k++) t[k].add(partial[r * kObsVals + k]);
    for (int k = 0; k < kObsVals; k++) sh[k][threadIdx.x] = t[k].value();
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < kObsVals; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < kObsVals; k++) scratch[blockIdx.x * kObsVals + k] = sh[k][0];
}

__global__ void obs_final_kernel(const double *__restrict__ scratch, int n, double scale, double *__restrict__ out3) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    CompSum t[kObsVals];
    for (int i = 0; i < n; i++)
        for (int k = 0; k < kObsVals; k++) t[k].add(scratch[i * kObsVals + k]);
    for (int k = 0; k < kObsVals; k++) out3[k] = scale * t[k].value();
}

constexpr int kObsRowBlocks = 256;

void launch_obs_finish(const double *partial, size_t rows, double *scratch, double scale, double *out3,
                       cudaStream_t stream) {
    obs_rows_kernel<<<kObsRowBlocks, 256, 0, stream>>>(partial, rows, scratch);
    obs_final_kernel<<<1, 32, 0, stream>>>(scratch, kObsRowBlocks, scale, out3);
}

constexpr int kZChunk = 4;  // z sites per thread in the z-marching variant

template <typename T, int MODE, class LK>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta, 2)
    wilson_zmarch_kernel(LK lk, const cpx<T> *__restrict__ src, cpx<T> *__restrict__ dst, Lattice L, T amass, T dt) {
    const int lane = threadIdx.x;
    const int n01 = L.N0 * L.N1;
    const int pxy = blockIdx.x * kSitesPerCta + threadIdx.y;  // site in the (x, y) plane
    const int mb = blockIdx.y;
    const int z0 = blockIdx.z * kZChunk;
    if (pxy >= n01 || z0 >= L.N2) return;
    const int z1 = min(z0 + kZChunk, L.N2);
    const int V = L.V;
    Spinor<T> fm, f0, fp, f;
    load_spinor(src, V, mb, pxy + n01 * ((z0 - 1 + L.N2) % L.N2), lane, fm);
    load_spinor(src, V, mb, pxy + n01 * z0, lane, f0);
    for (int z = z0; z < z1; z++) {
        const int site = pxy + n01 * z;
        const int zp = pxy + n01 * (z + 1 == L.N2 ? 0 : z + 1);
        const int zm = pxy + n01 * (z == 0 ? L.N2 - 1 : z - 1);
        load_spinor(src, V, mb, zp, lane, fp);
        const Nbrs n = neighbours(L, site);
        Spinor<T> acc;
#pragma unroll
        for (int c = 0; c < kColours; c++)
#pragma unroll
            for (int a = 0; a < kSpin; a++) acc.c[c][a] = amass * f0.c[c][a];
        load_spinor(src, V, mb, n.xp, lane, f);
        hop<T, 0, true>(acc, f, lk.template get<T>(site, 0));
        load_spinor(src, V, mb, n.xm, lane, f);
        hop<T, 0, false>(acc, f, lk.template get<T>(n.xm, 0));
        load_spinor(src, V, mb, n.yp, lane, f);
        hop<T, 1, true>(acc, f, lk.template get<T>(site, 1));
        load_spinor(src, V, mb, n.ym, lane, f);
        hop<T, 1, false>(acc, f, lk.template get<T>(n.ym, 1));
        hop<T, 2, true>(acc, fp, lk.template get<T>(site, 2));
        hop<T, 2, false>(acc, fm, lk.template get<T>(zm, 2));
        store_result<T, MODE>(dst, V, mb, site, lane, acc, dt);
        fm = f0;
        f0 = fp;
    }
}

template <typename T, int MODE, class LK>
static void launch_variant(int variant, const LK &lk, const cpx<T> *s, cpx<T> *d, const Lattice &L, int n_mb, T amass,
                           T dt, cudaStream_t stream) {
    dim3 block(kModeBlock, kSitesPerCta);
    if (variant == 2) {
        dim3 grid((L.N0 * L.N1 + kSitesPerCta - 1) / kSitesPerCta, n_mb, (L.N2 + kZChunk - 1) / kZChunk);
        wilson_zmarch_kernel<T, MODE, LK><<<grid, block, 0, stream>>>(lk, s, d, L, amass, dt);
        return;
    }
    if (variant == 1) {
        const int tiles = ((L.N0 + kTileX - 1) / kTileX) * ((L.N1 + kTileY - 1) / kTileY) * L.N2;
        if constexpr (sizeof(T) == 8) {
            const int m = link_blocks(tiles, n_mb, current_sm_count());
            if (m > 1) {
                wilson_tuned_kernel<T, MODE, 1, LK, true>
                    <<<dim3(tiles, (n_mb + m - 1) / m), block, 0, stream>>>(lk, s, d, L, amass, dt, n_mb, m);
                return;
            }
        }
        wilson_tuned_kernel<T, MODE, 1, LK><<<dim3(tiles, n_mb), block, 0, stream>>>(lk, s, d, L, amass, dt);
        return;
    }
    dim3 grid((L.V + kSitesPerCta - 1) / kSitesPerCta, n_mb);
    if constexpr (sizeof(T) == 8) {
        const int m = link_blocks(grid.x, n_mb, current_sm_count());
        if (m > 1) {
            wilson_tuned_kernel<T, MODE, 0, LK, true>
                <<<dim3(grid.x, (n_mb + m - 1) / m), block, 0, stream>>>(lk, s, d, L, amass, dt, n_mb, m);
            return;
        }
    }
    wilson_tuned_kernel<T, MODE, 0, LK><<<grid, block, 0, stream>>>(lk, s, d, L, amass, dt);
}

template <typename T>
void launch_wilson_tuned(const HopConfig &hc, const void *src, void *dst, const Lattice &L, int mb_first, int n_mb,
                         double amass, double dt, bool accumulate, cudaStream_t stream) {
    if (n_mb <= 0) return;
    const size_t off = field_index(L.V, mb_first, 0, 0, 0);
    const cpx<T> *s = reinterpret_cast<const cpx<T> *>(src) + off;
    cpx<T> *d = reinterpret_cast<cpx<T> *>(dst) + (accumulate ? off : 0);
    if (std::is_same<T, float>::value && hc.variant == kPackedVariant && hc.U32 != nullptr) {
        if (accumulate) launch_packed<1, false>(hc, s, d, L, n_mb, amass, dt, 0, 0, nullptr, stream);
        else launch_packed<0, false>(hc, s, d, L, n_mb, amass, dt, 0, 0, nullptr, stream);
        return;
    }
    const int n01 = L.N0 * L.N1;
    auto go = [&](const auto &lk) {
        if (accumulate) launch_variant<T, 1>(hc.variant, lk, s, d, L, n_mb, (T)amass, (T)dt, stream);
        else launch_variant<T, 0>(hc.variant, lk, s, d, L, n_mb, (T)amass, (T)dt, stream);
    };
    if (std::is_same<T, float>::value && hc.U32 != nullptr) {
        const float4 *u = reinterpret_cast<const float4 *>(hc.U32);
        if (hc.u1_32) go(LinksF32<true>{u, reinterpret_cast<const float2 *>(hc.u1_32), n01});
        else go(LinksF32<false>{u, nullptr, n01});
    } else {
        if (hc.u1) go(LinksF64<true>{hc.U, reinterpret_cast<const double2 *>(hc.u1), n01});
        else go(LinksF64<false>{hc.U, nullptr, n01});
    }
}

// ------------------------------------------------------ 40-bit storage --
// Half step on fields in 40-bit storage (ovl_fp40.cuh): a spinor is 8 uint2
// high words plus one uint4 of extension bytes per lane (9 loads); the raw
// words of the next neighbour are loaded one hop ahead (20 registers in
// flight), decode to FP64 by register moves, and the stencil runs in FP64 with
// the FP64 links; the destination is rounded back to 40 bits.  MODE 0:
// dst = D src; MODE 1: dst += dt D src.  Same launch shape as variant 0.
struct Raw40 {
    uint2 h[kComp];
    uint4 l;
};

__device__ __forceinline__ void load_raw40(const uint2 *__restrict__ hi, const uint4 *__restrict__ lo, int V, int mb,
                                           int site, int lane, Raw40 &r) {
    const size_t base = field_index(V, mb, site, 0, lane);
#pragma unroll
    for (int k = 0; k < kComp; k++) r.h[k] = __ldg(hi + base + k * kModeBlock);
    r.l = __ldg(lo + ((size_t)mb * V + site) * kModeBlock + lane);
}

// Extension byte b of the packed word, moved to the top byte of a 32-bit word
// (the low word of the decoded double) by one byte permute.
__device__ __forceinline__ unsigned ext_low(const uint4 &l, int b) {
    const unsigned w = b < 4 ? l.x : b < 8 ? l.y : b < 12 ? l.z : l.w;
    return __byte_perm(w, 0u, 0x0444u | ((unsigned)(b & 3) << 12));
}

__device__ __forceinline__ void decode40(const Raw40 &r, Spinor<double> &s) {
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) {
            const int k = c * kSpin + a;
            s.c[c][a] = mk<double>(__hiloint2double((int)r.h[k].x, (int)ext_low(r.l, 2 * k)),
                                   __hiloint2double((int)r.h[k].y, (int)ext_low(r.l, 2 * k + 1)));
        }
}

// MINB: CTAs of 8 warps per SM the register allocation must allow (2: 128
// registers, 3: 80 registers with a few spills); the autotuner picks.
// OBS: also sum the local charges of src into partial (as wilson_observe_kernel).
// One site and mode block of the FP40 half step (lane = the mode in the block);
// OBS: the local charges of src are added into o.
template <int MODE, bool OBS, class LK>
__device__ __forceinline__ void fp40_site(const LK &lk, const uint2 *__restrict__ src, const uint4 *__restrict__ src_lo,
                                          uint2 *__restrict__ dst, uint4 *__restrict__ dst_lo, const Lattice &L,
                                          int site, int mb, double amass, double dt, int n_modes, int first_mode,
                                          double (&o)[kObsVals]) {
    const int lane = threadIdx.x;
    const int V = L.V;
    const Nbrs n = neighbours(L, site);
    Raw40 a, b;
    Spinor<double> acc, f;
    load_raw40(src, src_lo, V, mb, site, lane, a);
    load_raw40(src, src_lo, V, mb, n.xp, lane, b);
    decode40(a, f);
    if (OBS) {
        const int mode = mb * kModeBlock + lane;
        const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
        local_charges(f.c, w, o);
    }
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int s2 = 0; s2 < kSpin; s2++) acc.c[c][s2] = amass * f.c[c][s2];
    load_raw40(src, src_lo, V, mb, n.xm, lane, a);
    decode40(b, f);
    hop<double, 0, true>(acc, f, lk.template get<double>(site, 0));
    load_raw40(src, src_lo, V, mb, n.yp, lane, b);
    decode40(a, f);
    hop<double, 0, false>(acc, f, lk.template get<double>(n.xm, 0));
    load_raw40(src, src_lo, V, mb, n.ym, lane, a);
    decode40(b, f);
    hop<double, 1, true>(acc, f, lk.template get<double>(site, 1));
    load_raw40(src, src_lo, V, mb, n.zp, lane, b);
    decode40(a, f);
    hop<double, 1, false>(acc, f, lk.template get<double>(n.ym, 1));
    load_raw40(src, src_lo, V, mb, n.zm, lane, a);
    decode40(b, f);
    hop<double, 2, true>(acc, f, lk.template get<double>(site, 2));
    if (MODE == 1) load_raw40(dst, dst_lo, V, mb, site, lane, b);  // the destination, one hop ahead
    decode40(a, f);
    hop<double, 2, false>(acc, f, lk.template get<double>(n.zm, 2));
    const size_t base = field_index(V, mb, site, 0, lane);
    unsigned lw[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int s2 = 0; s2 < kSpin; s2++) {
            const int k = c * kSpin + s2;
            cpx<double> d = finish_component(acc.c[c][s2], s2);
            if (MODE == 1) {
                d.re = __hiloint2double((int)b.h[k].x, (int)ext_low(b.l, 2 * k)) + dt * d.re;
                d.im = __hiloint2double((int)b.h[k].y, (int)ext_low(b.l, 2 * k + 1)) + dt * d.im;
            }
            // round to 40 bits: add half a unit of the last kept bit, keep the
            // high word and the top byte of the low word
            const unsigned long long bre = (unsigned long long)__double_as_longlong(d.re) + (1ull << 23);
            const unsigned long long bim = (unsigned long long)__double_as_longlong(d.im) + (1ull << 23);
            dst[base + k * kModeBlock] = make_uint2((unsigned)(bre >> 32), (unsigned)(bim >> 32));
            // bytes 3 of the two low words -> bytes 2(k&1), 2(k&1)+1 of word k/2
            const unsigned pair = __byte_perm((unsigned)bre, (unsigned)bim, 0x0073u) & 0xffffu;
            lw[k >> 1] |= pair << (16 * (k & 1));
        }
    dst_lo[((size_t)mb * V + site) * kModeBlock + lane] = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

// TABLE (not observing): a CTA runs its 8 sites for mblk mode blocks
// [mblk blockIdx.y, ...) of the n_mb, with the sites' links gathered once in
// shared memory (fill_link_table) instead of loaded and dressed with the U(1)
// phase once per mode block.
template <int MODE, int MINB, class LK, bool OBS = false, bool TABLE = false>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta, MINB)
    wilson_fp40_kernel(LK lk, const uint2 *__restrict__ src, const uint4 *__restrict__ src_lo, uint2 *__restrict__ dst,
                       uint4 *__restrict__ dst_lo, Lattice L, double amass, double dt, int n_modes = 0,
                       int first_mode = 0, double *__restrict__ partial = nullptr, int n_mb = 0, int mblk = 1) {
    const int site = blockIdx.x * kSitesPerCta + threadIdx.y;
    double o[kObsVals] = {0.0, 0.0, 0.0};
    if constexpr (TABLE) {
        static_assert(!OBS, "the observing half step keeps one mode block per CTA row");
        __shared__ cmat2<double> tab[kSitesPerCta][6];
        const int site0 = blockIdx.x * kSitesPerCta;
        fill_link_table<kSitesPerCta>(lk, L, [&](int j) { return site0 + j < L.V ? site0 + j : -1; }, tab);
        if (site >= L.V) return;
        const LinksTable lt{tab[threadIdx.y], site};
        const int mb0 = blockIdx.y * mblk, mb1 = min(n_mb, mb0 + mblk);
        for (int mb = mb0; mb < mb1; mb++) fp40_site<MODE, false>(lt, src, src_lo, dst, dst_lo, L, site, mb, amass, dt, 0, 0, o);
        return;
    }
    if (site >= L.V) {
        if (OBS) cta_partial(o, partial);
        return;
    }
    fp40_site<MODE, OBS>(lk, src, src_lo, dst, dst_lo, L, site, blockIdx.y, amass, dt, n_modes, first_mode, o);
    if (OBS) cta_partial(o, partial);
}

void launch_wilson40(const HopConfig &hc, const void *src, const void *src_lo, void *dst, void *dst_lo,
                     const Lattice &L, int mb_first, int n_mb, double amass, double dt, bool accumulate,
                     cudaStream_t stream) {
    if (n_mb <= 0) return;
    const size_t off = field_index(L.V, mb_first, 0, 0, 0);    // complex numbers
    const size_t loff = (size_t)mb_first * L.V * kModeBlock;  // uint4 words
    const uint2 *s = reinterpret_cast<const uint2 *>(src) + off;
    const uint4 *sl = reinterpret_cast<const uint4 *>(src_lo) + loff;
    uint2 *d = reinterpret_cast<uint2 *>(dst) + (accumulate ? off : 0);
    uint4 *dl = reinterpret_cast<uint4 *>(dst_lo) + (accumulate ? loff : 0);
    dim3 block(kModeBlock, kSitesPerCta);
    dim3 grid((L.V + kSitesPerCta - 1) / kSitesPerCta, n_mb);
    const int m = link_blocks(grid.x, n_mb, current_sm_count());
    const int n01 = L.N0 * L.N1;
    auto go = [&](const auto &lk) {
        using LK = std::decay_t<decltype(lk)>;
        if (m > 1) {
            const dim3 g2(grid.x, (n_mb + m - 1) / m);
            if (!accumulate)
                wilson_fp40_kernel<0, 2, LK, false, true><<<g2, block, 0, stream>>>(lk, s, sl, d, dl, L, amass, dt, 0, 0,
                                                                                   nullptr, n_mb, m);
            else if (hc.variant == 1)
                wilson_fp40_kernel<1, 3, LK, false, true><<<g2, block, 0, stream>>>(lk, s, sl, d, dl, L, amass, dt, 0, 0,
                                                                                   nullptr, n_mb, m);
            else
                wilson_fp40_kernel<1, 2, LK, false, true><<<g2, block, 0, stream>>>(lk, s, sl, d, dl, L, amass, dt, 0, 0,
                                                                                   nullptr, n_mb, m);
            return;
        }
        if (accumulate) {
            if (hc.variant == 1) wilson_fp40_kernel<1, 3, LK><<<grid, block, 0, stream>>>(lk, s, sl, d, dl, L, amass, dt);
            else wilson_fp40_kernel<1, 2, LK><<<grid, block, 0, stream>>>(lk, s, sl, d, dl, L, amass, dt);
        } else {
            wilson_fp40_kernel<0, 2, LK><<<grid, block, 0, stream>>>(lk, s, sl, d, dl, L, amass, dt);
        }
    };
    if (hc.u1) go(LinksF64<true>{hc.U, reinterpret_cast<const double2 *>(hc.u1), n01});
    else go(LinksF64<false>{hc.U, nullptr, n01});
}

void launch_wilson40_observe(const HopConfig &hc, const void *src, const void *src_lo, void *dst, void *dst_lo,
                             const Lattice &L, int n_mb, double amass, double dt, int n_modes, int first_mode,
                             double *partial, cudaStream_t stream) {
    const uint2 *s = reinterpret_cast<const uint2 *>(src);
    const uint4 *sl = reinterpret_cast<const uint4 *>(src_lo);
    uint2 *d = reinterpret_cast<uint2 *>(dst);
    uint4 *dl = reinterpret_cast<uint4 *>(dst_lo);
    const dim3 block(kModeBlock, kSitesPerCta), grid((L.V + kSitesPerCta - 1) / kSitesPerCta, n_mb);
    const int n01 = L.N0 * L.N1;
    auto go = [&](const auto &lk) {
        using LK = std::decay_t<decltype(lk)>;
        wilson_fp40_kernel<1, 2, LK, true><<<grid, block, 0, stream>>>(lk, s, sl, d, dl, L, amass, dt, n_modes,
                                                                        first_mode, partial);
    };
    if (hc.u1) go(LinksF64<true>{hc.U, reinterpret_cast<const double2 *>(hc.u1), n01});
    else go(LinksF64<false>{hc.U, nullptr, n01});
}

// FP32 copy of the links (and of the U(1) phases) for the FP32 path.
__global__ void links_to_f32_kernel(const double *__restrict__ U, float *U32, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) U32[i] = (float)U[i];
}

void launch_links_to_f32(const double *U, float *U32, size_t n, cudaStream_t stream) {
    links_to_f32_kernel<<<(int)((n + 255) / 256), 256, 0, stream>>>(U, U32, (int)n);
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
    if constexpr (sizeof(T) == 8) {
        // the same site function and store as wilson_kernel, on links gathered once per CTA
        const int m = link_blocks(grid.x, n_mb, current_sm_count());
        if (m > 1) {
            const dim3 g2(grid.x, (n_mb + m - 1) / m);
            auto go = [&](const auto &lk) {
                using LK = std::decay_t<decltype(lk)>;
                if (accumulate)
                    wilson_tuned_kernel<T, 1, 0, LK, true><<<g2, block, 0, stream>>>(lk, s + off, d + off, L, (T)amass,
                                                                                    (T)dt, n_mb, m);
                else
                    wilson_tuned_kernel<T, 0, 0, LK, true><<<g2, block, 0, stream>>>(lk, s + off, d, L, (T)amass, (T)dt,
                                                                                    n_mb, m);
            };
            if (ph) go(LinksF64<true>{links, ph, L.N0 * L.N1});
            else go(LinksF64<false>{links, nullptr, L.N0 * L.N1});
            return;
        }
    }
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
template void launch_wilson_tuned<double>(const HopConfig &, const void *, void *, const Lattice &, int, int, double,
                                          double, bool, cudaStream_t);
template void launch_wilson_tuned<float>(const HopConfig &, const void *, void *, const Lattice &, int, int, double,
                                         double, bool, cudaStream_t);
template void launch_axpy<float>(void *, const void *, size_t, double, int, cudaStream_t);
template size_t launch_wilson_observe<float>(const HopConfig &, const void *, void *, const Lattice &, int, double, double,
                                           int, int, double *, cudaStream_t);
template size_t launch_wilson_observe<double>(const HopConfig &, const void *, void *, const Lattice &, int, double,
                                            double, int, int, double *, cudaStream_t);

}  // namespace ovl
