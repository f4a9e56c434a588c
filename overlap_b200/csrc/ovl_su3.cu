// Three-colour kernels: the Wilson leapfrog half step (plain and fused), the
// link update, the Chebyshev overlap operator, the charges, the improved E.B,
// the geodesic interpolation of Delta N_CS and the bulk observables, for
// 12-component modes and SU(3) links (layouts in ovl_su3.cuh).  Each follows
// the two-colour kernel of the same job (ovl_wilson.cu, ovl_chebyshev.cu,
// ovl_modes.cu, ovl_gauge.cu) with 3x3 links; the reference routines are
// cited there.
#include <algorithm>
#include <cmath>

#include "ovl_internal.h"
#include "ovl_su3.cuh"
#include "ovl_su3_packed.cuh"

namespace ovl {

// ------------------------------------------------------------ hop kernel --
// MODE 0: out = D src; MODE 1: out += dt D src (the fused half step).
// CTAs per SM the register allocation must allow: FP32 6 (85 registers; 64 for 8 spill).
template <typename T> struct Occ3 { static constexpr int kMinBlocks = sizeof(T) == 4 ? 6 : 1; };

template <typename T, int MODE, class LK>
__global__ void __launch_bounds__(kModeBlock *kSites3, Occ3<T>::kMinBlocks)
    su3_wilson_kernel(LK lk, const cpx<T> *__restrict__ src, cpx<T> *__restrict__ out, Lattice L, int mb0, T amass,
                      T dt) {
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSites3 + threadIdx.y;
    const int mb = mb0 + blockIdx.y;
    if (site >= L.V) return;
    Spinor3<T> acc;
    wilson_site3(lk, src, L, site, mb, lane, amass, acc);
    cpx<T> *o = out + field_index3(L.V, MODE == 1 ? mb : blockIdx.y, site, 0, lane);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) {
            const cpx<T> v = acc.c[c][a];
            const cpx<T> d = (T)0.5 * (a < 2 ? times_mi(v) : times_i(v));  // -i gamma_0 / 2
            cpx<T> *p = o + (c * kSpin + a) * kModeBlock;
            if (MODE == 1) {
                const cpx<T> w = ld(p);
                st(p, w + dt * d);
            } else {
                st(p, d);
            }
        }
}

template <typename T, int MODE, bool F32, bool U1>
static void hop3_launch(const Su3Links &lk, const void *src, void *dst, const Lattice &L, int mb0, int n_mb, double amass,
                        double dt, cudaStream_t s) {
    const dim3 block(kModeBlock, kSites3), grid((L.V + kSites3 - 1) / kSites3, n_mb);
    Links3<F32, U1> links{F32 ? (const void *)lk.U32 : (const void *)lk.U, F32 ? (const void *)lk.u1_32 : (const void *)lk.u1,
                          L.N0 * L.N1};
    su3_wilson_kernel<T, MODE, Links3<F32, U1>><<<grid, block, 0, s>>>(
        links, reinterpret_cast<const cpx<T> *>(src), reinterpret_cast<cpx<T> *>(dst), L, mb0, (T)amass, (T)dt);
}

// The packed-pair stencil (variant 3, FP32): CTAs of kPk3Warps warps (2
// kPk3Warps sites) running kPk3Blocks mode blocks each on one set of link
// records.  MODE 0: dst = D src, 1: dst += dt D src, 2: the Clenshaw term.
constexpr int kPk3Warps = 4, kPk3Sites = 2 * kPk3Warps, kPk3Blocks = 8, kPk3MinBlocks = 3;

template <int MODE, bool U1>
__global__ void __launch_bounds__(kModeBlock *kPk3Warps, kPk3MinBlocks)
    su3_packed_kernel(const float4 *__restrict__ U32, const float2 *__restrict__ u1, const float4 *__restrict__ src,
                      float4 *__restrict__ dst, Lattice L, int n_mb, float amass, float hdt, const ClenshawArgs cl) {
    __shared__ float4 rec[kPk3Sites][6][kPk3RecVec];
    const int mb0 = blockIdx.y * kPk3Blocks;
    packed_tile3<MODE, U1, kPk3Warps>(rec, U32, u1, src, dst, L, blockIdx.x * kPk3Sites, mb0,
                                      min(n_mb, mb0 + kPk3Blocks), amass, hdt, cl);
}

template <int MODE>
static void packed3_launch(const Su3Links &lk, const void *src, void *dst, const Lattice &L, int n_mb, double amass,
                           double dt, const ClenshawArgs &cl, cudaStream_t s) {
    const dim3 block(kModeBlock, kPk3Warps), grid((L.V + kPk3Sites - 1) / kPk3Sites, (n_mb + kPk3Blocks - 1) / kPk3Blocks);
    const float4 *U = reinterpret_cast<const float4 *>(lk.U32);
    const float4 *a = reinterpret_cast<const float4 *>(src);
    float4 *d = reinterpret_cast<float4 *>(dst);
    const float am = (float)amass, h = (float)(0.5 * dt);
    if (lk.u1_32)
        su3_packed_kernel<MODE, true><<<grid, block, 0, s>>>(U, reinterpret_cast<const float2 *>(lk.u1_32), a, d, L,
                                                             n_mb, am, h, cl);
    else
        su3_packed_kernel<MODE, false><<<grid, block, 0, s>>>(U, nullptr, a, d, L, n_mb, am, h, cl);
}

static bool packed3(const Su3Links &lk, size_t elem) { return elem == 4 && lk.variant == kPackedVariant && lk.U32; }

template <typename T>
void su3_launch_hop(const Su3Links &lk, const void *src, void *dst, const Lattice &L, int mb0, int n_mb, double amass,
                    double dt, bool accumulate, cudaStream_t s) {
    constexpr bool F32 = sizeof(T) == 4;
    if (packed3(lk, sizeof(T))) {
        const size_t off = field_index3(L.V, mb0, 0, 0, 0);
        const cpx<T> *a = reinterpret_cast<const cpx<T> *>(src) + off;
        cpx<T> *d = reinterpret_cast<cpx<T> *>(dst) + (accumulate ? off : 0);
        if (accumulate) packed3_launch<1>(lk, a, d, L, n_mb, amass, dt, ClenshawArgs{}, s);
        else packed3_launch<0>(lk, a, d, L, n_mb, amass, 0.0, ClenshawArgs{}, s);
        return;
    }
    const bool u1 = F32 ? lk.u1_32 != nullptr : lk.u1 != nullptr;
    if (accumulate) {
        if (u1) hop3_launch<T, 1, F32, true>(lk, src, dst, L, mb0, n_mb, amass, dt, s);
        else hop3_launch<T, 1, F32, false>(lk, src, dst, L, mb0, n_mb, amass, dt, s);
    } else {
        if (u1) hop3_launch<T, 0, F32, true>(lk, src, dst, L, mb0, n_mb, amass, dt, s);
        else hop3_launch<T, 0, F32, false>(lk, src, dst, L, mb0, n_mb, amass, dt, s);
    }
}

// ----------------------------------------------------------- link update --
// U <- exp(i cU t^a E^a) U (Dynamics.cpp:97-138, cU = -dt_step), optionally
// projected back onto SU(3), with the FP32 copy kept.
__global__ void su3_links_kernel(double *U, const double *__restrict__ E, int n_links, double c, float *U32, int reunit) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_links) return;
    const int site = l / 3, mu = l % 3;
    double e[8];
#pragma unroll
    for (int a = 0; a < 8; a++) e[a] = E[8 * (size_t)l + a];
    cmat3<double> u = m3_mul(su3_exp(c, e), load_su3(U, site, mu));
    if (reunit) u = su3_reunitarize(u);
    store_su3(U, site, mu, u);
    if (U32) {
        float2 *p = reinterpret_cast<float2 *>(U32 + (size_t)kLink32Floats * l);
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) p[i + 3 * j] = float2{(float)u.m[i][j].re, (float)u.m[i][j].im};
        p[9] = float2{0.0f, 0.0f};
    }
}

void su3_launch_update_links(double *U, const double *E, const Lattice &L, double dt_step, float *U32, bool reunit,
                             cudaStream_t s) {
    const int n = 3 * L.V;
    su3_links_kernel<<<(n + 127) / 128, 128, 0, s>>>(U, E, n, -dt_step, U32, reunit ? 1 : 0);
}

// --------------------------------------------------------- Chebyshev sign --
// One Clenshaw term b_out = factor (a (-D w) + beta b1) - b2 + ck phi, -D w
// the stencil applied to w = D b1 (ovl_chebyshev.cu, three colours).
template <typename T, class LK>
__global__ void __launch_bounds__(kModeBlock *kSites3, Occ3<T>::kMinBlocks)
    su3_clenshaw_kernel(LK lk, const cpx<T> *__restrict__ w, const cpx<T> *__restrict__ b1,
                        const cpx<T> *__restrict__ b2, const cpx<T> *__restrict__ phi, cpx<T> *__restrict__ bout,
                        Lattice L, T amass, T a, T beta, T factor, T ck) {
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSites3 + threadIdx.y;
    const int mb = blockIdx.y;
    if (site >= L.V) return;
    Spinor3<T> acc;
    wilson_site3(lk, w, L, site, mb, lane, amass, acc);
    const size_t base = field_index3(L.V, mb, site, 0, lane);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int s = 0; s < kSpin; s++) {
            const size_t i = base + (c * kSpin + s) * kModeBlock;
            const cpx<T> v = acc.c[c][s];
            const cpx<T> dw = (T)0.5 * (s < 2 ? times_mi(v) : times_i(v));
            const cpx<T> v1 = ld(b1 + i), v2 = ld(b2 + i), f = ld(phi + i);
            const cpx<T> tx = mk<T>(-a * dw.re + beta * v1.re, -a * dw.im + beta * v1.im);
            st(bout + i, mk<T>(factor * tx.re - v2.re + ck * f.re, factor * tx.im - v2.im + ck * f.im));
        }
}

// out = M [ -i g0 (1 + m/2) phi + (1 - m/2) dchi ];  dst = out or dst += dt out
template <typename T>
__global__ void su3_overlap_finish_kernel(const cpx<T> *__restrict__ phi, const cpx<T> *__restrict__ dchi, cpx<T> *dst,
                                          size_t n, T mdw, T mf, T dt, int accumulate) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int spin = (int)((e / kModeBlock) % kSpin);
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

template <typename T, bool F32, bool U1>
static void cheb3(ChebyshevWork &w, const Su3Links &lk, const void *src, void *dst, const Lattice &L, int n_mb,
                  const double *coeff, int K, double eps, double lambda_max, double amass, double mdw, double mf,
                  double dt, bool accumulate, int sm_count, cudaStream_t stream, uint64_t *launches) {
    const size_t n = (size_t)n_mb * L.V * kComp3 * kModeBlock;
    const dim3 block(kModeBlock, kSites3), grid((L.V + kSites3 - 1) / kSites3, n_mb);
    Links3<F32, U1> links{F32 ? (const void *)lk.U32 : (const void *)lk.U, F32 ? (const void *)lk.u1_32 : (const void *)lk.u1,
                          L.N0 * L.N1};
    const cpx<T> *phi = reinterpret_cast<const cpx<T> *>(src);
    cpx<T> *b[3] = {reinterpret_cast<cpx<T> *>(w.b0), reinterpret_cast<cpx<T> *>(w.b1), reinterpret_cast<cpx<T> *>(w.b2)};
    cpx<T> *tmp = reinterpret_cast<cpx<T> *>(w.w);
    const double scale = 1.0 / std::sqrt(lambda_max);
    const T a = (T)(2.0 / ((1.0 - eps) * lambda_max)), beta = (T)(-(1.0 + eps) / (1.0 - eps)), am = (T)amass;
    cudaMemsetAsync(b[1], 0, n * sizeof(cpx<T>), stream);
    cudaMemsetAsync(b[2], 0, n * sizeof(cpx<T>), stream);
    int i1 = 1, i2 = 2, io = 0;
    uint64_t nl = 0;
    // variant 3 (FP32): the D passes in the packed stencil, and the overlap
    // combination fused into the last one
    const bool pk = packed3(lk, sizeof(T));
    for (int k = K; k >= 0; k--) {
        const T factor = (T)(k > 0 ? 2 : 1), ck = (T)((k > 0 ? coeff[k] : 0.5 * coeff[0]) * scale);
        if (pk) packed3_launch<0>(lk, b[i1], tmp, L, n_mb, amass, 0.0, ClenshawArgs{}, stream);
        else su3_wilson_kernel<T, 0, Links3<F32, U1>><<<grid, block, 0, stream>>>(links, b[i1], tmp, L, 0, am, (T)0);
        su3_clenshaw_kernel<T, Links3<F32, U1>><<<grid, block, 0, stream>>>(links, tmp, b[i1], b[i2], phi, b[io], L, am,
                                                                            a, beta, factor, ck);
        nl += 2;
        const int t = i2;
        i2 = i1;
        i1 = io;
        io = t;
    }
    // chi = b[i1]; D chi, then the overlap combination (one pass of the
    // packed stencil with the combination in its epilogue)
    if (pk) {
        ClenshawArgs cl{};
        cl.phi = reinterpret_cast<const float4 *>(phi);
        cl.mdw = (float)mdw;
        cl.cp = (float)(1.0 + 0.5 * mf);
        cl.cm = (float)(1.0 - 0.5 * mf);
        cl.dt = (float)dt;
        cl.accumulate = accumulate ? 1 : 0;
        packed3_launch<3>(lk, b[i1], dst, L, n_mb, amass, 0.0, cl, stream);
        nl += 1;
        if (launches) *launches += nl;
        return;
    }
    su3_wilson_kernel<T, 0, Links3<F32, U1>><<<grid, block, 0, stream>>>(links, b[i1], tmp, L, 0, am, (T)0);
    const size_t blocks = (n + 255) / 256, cap = (size_t)sm_count * 16;
    su3_overlap_finish_kernel<T><<<(int)std::min(blocks, cap), 256, 0, stream>>>(
        phi, tmp, reinterpret_cast<cpx<T> *>(dst), n, (T)mdw, (T)mf, (T)dt, accumulate ? 1 : 0);
    nl += 2;
    if (launches) *launches += nl;
}

template <typename T>
void su3_chebyshev_apply(ChebyshevWork &w, const Su3Links &lk, const void *src, void *dst, const Lattice &L, int n_mb,
                         const double *coeff, int K, double eps, double lambda_max, double amass, double mdw, double mf,
                         double dt, bool accumulate, int sm_count, cudaStream_t stream, uint64_t *launches) {
    constexpr bool F32 = sizeof(T) == 4;
    const bool u1 = F32 ? lk.u1_32 != nullptr : lk.u1 != nullptr;
    if (u1)
        cheb3<T, F32, true>(w, lk, src, dst, L, n_mb, coeff, K, eps, lambda_max, amass, mdw, mf, dt, accumulate, sm_count,
                            stream, launches);
    else
        cheb3<T, F32, false>(w, lk, src, dst, L, n_mb, coeff, K, eps, lambda_max, amass, mdw, mf, dt, accumulate, sm_count,
                             stream, launches);
}

// ---------------------------------------------------------------- charges --
// Lattice sums {sum jV^0, N_5, sum PS, sum WA} (Currents.cpp:7-394 for three
// colours; the bilinears of charges_kernel in ovl_modes.cu).  Bilinears in
// FP64 for every mode precision.  One CTA per (group of kSites3 sites, slice
// of mode blocks); partial sums per CTA, summed in a fixed order.
constexpr int kCharge3Groups = 8;  // mode-block slices per site group

template <typename T>
__global__ void __launch_bounds__(kModeBlock *kSites3)
    su3_charges_kernel(const double *__restrict__ U, const double2 *__restrict__ u1, const cpx<T> *__restrict__ psi,
                       Lattice L, int n_mb, int n_modes, int first_mode, double r, double *__restrict__ partial) {
    __shared__ double sh[kSites3][4];
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSites3 + threadIdx.y;
    CompSum sum[4];
    if (site < L.V) {
        int x, y, z;
        site_coords(L, site, x, y, z);
        int nb[3];
        for (int mu = 0; mu < 3; mu++) {
            int c[3] = {x, y, z};
            c[mu] += 1;
            nb[mu] = site_index(L, c[0], c[1], c[2]);
        }
        const Links3<false, true> lk1{U, u1, L.N0 * L.N1};
        const Links3<false, false> lk0{U, nullptr, L.N0 * L.N1};
        cmat3<double> M[3];
        for (int mu = 0; mu < 3; mu++) M[mu] = u1 ? lk1.get<double>(site, mu) : lk0.get<double>(site, mu);
        for (int mb = blockIdx.y; mb < n_mb; mb += gridDim.y) {
            const int mode = mb * kModeBlock + lane;
            const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
            cpx<double> f[3][kSpin];
            const cpx<T> *p = psi + field_index3(L.V, mb, site, 0, lane);
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int a = 0; a < kSpin; a++) {
                    const cpx<T> v = ld(p + (c * kSpin + a) * kModeBlock);
                    f[c][a] = mk<double>((double)v.re, (double)v.im);
                }
            double nv = 0.0;
            cpx<double> zz = mk<double>(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < 3; c++) {
#pragma unroll
                for (int a = 0; a < kSpin; a++) nv += f[c][a].re * f[c][a].re + f[c][a].im * f[c][a].im;
                zz = zz + cdot(f[c][0], f[c][2]) + cdot(f[c][1], f[c][3]);
            }
            double hop = 0.0;
            for (int mu = 0; mu < 3; mu++) {
                const cpx<T> *q = psi + field_index3(L.V, mb, nb[mu], 0, lane);
                cpx<double> ht[3][kSpin];
#pragma unroll
                for (int c = 0; c < 3; c++)
#pragma unroll
                    for (int a = 0; a < kSpin; a++) {
                        const cpx<T> v = ld(q + (c * kSpin + a) * kModeBlock);
                        ht[c][a] = mk<double>((double)v.re, (double)v.im);
                    }
                cpx<double> b = mk<double>(0.0, 0.0);
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    cpx<double> chi[kSpin];
#pragma unroll
                    for (int a = 0; a < kSpin; a++)
                        chi[a] = M[mu].m[i][0] * ht[0][a] + M[mu].m[i][1] * ht[1][a] + M[mu].m[i][2] * ht[2][a];
                    b = b + cdot(f[i][0], chi[2]) + cdot(f[i][1], chi[3]) - cdot(f[i][2], chi[0]) - cdot(f[i][3], chi[1]);
                }
                hop += b.im;
            }
            sum[0].add(w * nv);
            sum[1].add(w * 2.0 * zz.re);
            sum[2].add(w * -2.0 * zz.im);
            sum[3].add(w * (r * (-12.0 * zz.im + 2.0 * hop)));
        }
    }
    double acc[4];
#pragma unroll
    for (int k = 0; k < 4; k++) acc[k] = sum[k].value();
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double t = acc[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        acc[k] = t;
    }
    if (lane == 0)
        for (int k = 0; k < 4; k++) sh[threadIdx.y][k] = acc[k];
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        double *q = partial + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 4;
        for (int k = 0; k < 4; k++) {
            double t = 0.0;
            for (int j = 0; j < kSites3; j++) t += sh[j][k];
            q[k] = t;
        }
    }
}

// Per-site Wilson currents for three colours (currents_kernel of ovl_modes.cu,
// Currents.cpp:7-394): per site the 18 vacuum-weighted mode sums jV^0..3,
// jA^0..3, jVw^1..3, jAw^1..3, PS, WA (slots as kCurrentsPerSite), per group of
// mode blocks into partial[g][site][18]; launch_currents_finish adds the groups.
template <typename T>
__device__ __forceinline__ cpx<double> colour_bilinear3(const mono &G, const cpx<double> (&f)[3][kSpin],
                                                        const cpx<double> (&h)[3][kSpin]) {
    return bilinear<double>(G, f[0], h[0]) + bilinear<double>(G, f[1], h[1]) + bilinear<double>(G, f[2], h[2]);
}

template <typename T>
__device__ __forceinline__ void load_site3(const cpx<T> *__restrict__ psi, int V, int mb, int site, int lane,
                                           cpx<double> (&f)[3][kSpin]) {
    const cpx<T> *p = psi + field_index3(V, mb, site, 0, lane);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) {
            const cpx<T> v = ld(p + (c * kSpin + a) * kModeBlock);
            f[c][a] = mk<double>((double)v.re, (double)v.im);
        }
}

template <typename T, bool U1>
__global__ void __launch_bounds__(kModeBlock *kSites3)
    su3_currents_kernel(const double *__restrict__ U, const double *__restrict__ u1, const cpx<T> *__restrict__ psi,
                        Lattice L, int n_mb, int n_modes, int first_mode, int groups, double r,
                        double *__restrict__ partial) {
    constexpr mono G1 = {{0, 1, 2, 3}, {0, 0, 0, 0}};
    constexpr mono G5 = kGamma5;
    constexpr mono G05 = mono_mul(kGamma0, kGamma5);
    constexpr mono G0 = kGamma0;
    constexpr mono GV[3] = {mono_mul(kGamma0, kGammaX), mono_mul(kGamma0, kGammaY), mono_mul(kGamma0, kGammaZ)};
    constexpr mono GA[3] = {mono_mul(GV[0], kGamma5), mono_mul(GV[1], kGamma5), mono_mul(GV[2], kGamma5)};
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSites3 + threadIdx.y;
    const int g = blockIdx.y;
    if (site >= L.V) return;  // whole warps exit together
    int x, y, z;
    site_coords(L, site, x, y, z);
    const int V = L.V;
    int nb[3][2];
    for (int mu = 0; mu < 3; mu++) {
        int cp[3] = {x, y, z}, cm[3] = {x, y, z};
        cp[mu] += 1;
        cm[mu] -= 1;
        nb[mu][0] = site_index(L, cp[0], cp[1], cp[2]);
        nb[mu][1] = site_index(L, cm[0], cm[1], cm[2]);
    }
    const Links3<false, U1> lk{U, u1, L.N0 * L.N1};
    CompSum acc[kCurrentsPerSite];
    for (int mb = g; mb < n_mb; mb += groups) {
        const int mode = mb * kModeBlock + lane;
        const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
        cpx<double> f[3][kSpin];
        load_site3(psi, V, mb, site, lane, f);
        double v[kCurrentsPerSite];
#pragma unroll
        for (int k = 0; k < kCurrentsPerSite; k++) v[k] = 0.0;
        v[0] = colour_bilinear3<T>(G1, f, f).re;
        v[4] = colour_bilinear3<T>(G5, f, f).re;
        const cpx<double> b05 = colour_bilinear3<T>(G05, f, f);
        v[16] = -b05.im;
        double wa = -6.0 * r * b05.im;
        for (int mu = 0; mu < 3; mu++) {
            cpx<double> h[3][kSpin], chi[3][kSpin];
            load_site3(psi, V, mb, nb[mu][0], lane, h);  // forward: chi = U_mu(x) psi(x+mu)
            {
                const cmat3<double> M = lk.template get<double>(site, mu);
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int a = 0; a < kSpin; a++)
                        chi[i][a] = M.m[i][0] * h[0][a] + M.m[i][1] * h[1][a] + M.m[i][2] * h[2][a];
            }
            v[1 + mu] = colour_bilinear3<T>(GV[mu], f, chi).re;
            v[5 + mu] = colour_bilinear3<T>(GA[mu], f, chi).re;
            v[9 + mu] = r * colour_bilinear3<T>(G0, f, chi).im;
            const double aw = r * colour_bilinear3<T>(G05, f, chi).im;
            v[13 + mu] = aw;
            wa += aw;
            load_site3(psi, V, mb, nb[mu][1], lane, h);  // backward: chi = U_mu(x-mu)^+ psi(x-mu)
            {
                const cmat3<double> M = lk.template get<double>(nb[mu][1], mu);
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int a = 0; a < kSpin; a++)
                        chi[i][a] = cdot(M.m[0][i], h[0][a]) + cdot(M.m[1][i], h[1][a]) + cdot(M.m[2][i], h[2][a]);
            }
            wa += r * colour_bilinear3<T>(G05, f, chi).im;
        }
        v[17] = wa;
#pragma unroll
        for (int k = 0; k < kCurrentsPerSite; k++) acc[k].add(w * v[k]);
    }
#pragma unroll
    for (int k = 0; k < kCurrentsPerSite; k++) {
        double t = acc[k].value();
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) partial[((size_t)g * V + site) * kCurrentsPerSite + k] = t;
    }
}

template <typename T>
void su3_launch_currents(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                         int first_mode, double r, double *partial, double *per_site, cudaStream_t s) {
    const int groups = currents_groups(n_mb);
    const dim3 block(kModeBlock, kSites3), grid((L.V + kSites3 - 1) / kSites3, groups);
    const cpx<T> *p = reinterpret_cast<const cpx<T> *>(psi);
    if (u1) su3_currents_kernel<T, true><<<grid, block, 0, s>>>(U, u1, p, L, n_mb, n_modes, first_mode, groups, r, partial);
    else su3_currents_kernel<T, false><<<grid, block, 0, s>>>(U, u1, p, L, n_mb, n_modes, first_mode, groups, r, partial);
    launch_currents_finish(partial, groups, L, per_site, s);
}

// Sums `n` partial rows of `nv` values in a fixed order (one CTA: a strided
// sum per thread, then a tree), scaled.
template <int NV>
__global__ void su3_sum_rows_kernel(const double *__restrict__ partial, int n, double scale, double *__restrict__ out) {
    __shared__ double sh[256][NV];
    CompSum t[NV];
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int k = 0; k < NV; k++) t[k].add(partial[(size_t)i * NV + k]);
    for (int k = 0; k < NV; k++) sh[threadIdx.x][k] = t[k].value();
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < NV; k++) sh[threadIdx.x][k] += sh[threadIdx.x + w][k];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < NV; k++) out[k] = scale * sh[0][k];
}

size_t su3_charges_partial_doubles(const Lattice &L, int n_mb) {
    return (size_t)4 * ((L.V + kSites3 - 1) / kSites3) * std::min(n_mb, kCharge3Groups);
}

template <typename T>
void su3_launch_charges(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                        int first_mode, double r, double *partial, double *out4, cudaStream_t s) {
    const dim3 block(kModeBlock, kSites3), grid((L.V + kSites3 - 1) / kSites3, std::min(n_mb, kCharge3Groups));
    su3_charges_kernel<T><<<grid, block, 0, s>>>(U, reinterpret_cast<const double2 *>(u1),
                                                 reinterpret_cast<const cpx<T> *>(psi), L, n_mb, n_modes, first_mode, r,
                                                 partial);
    su3_sum_rows_kernel<4><<<1, 256, 0, s>>>(partial, (int)(grid.x * grid.y), 1.0 / (2.0 * L.V), out4);
}

// ----------------------------------------------------------- Wilson loops --
__device__ inline cmat3<double> su3_step(const double *__restrict__ U, const Lattice &L, int c[3], int mu, int dir,
                                         const cmat3<double> &acc) {
    if (dir > 0) {
        const cmat3<double> u = load_su3(U, site_index(L, c[0], c[1], c[2]), mu);
        c[mu] += 1;
        return m3_mul(acc, u);
    }
    c[mu] -= 1;
    return m3_mul(acc, m3_dag(load_su3(U, site_index(L, c[0], c[1], c[2]), mu)));
}

// Counter-clockwise lmu x lnu loop in the (mu, nu) plane with (x, y, z) at its
// corner in quadrant (smu, snu), holonomy based at that corner (loop() in
// ovl_gauge.cu).
__device__ cmat3<double> su3_loop(const double *__restrict__ U, const Lattice &L, int x, int y, int z, int mu, int nu,
                                  int smu, int snu, int lmu, int lnu) {
    const int dmu[4] = {mu, nu, mu, nu}, ddir[4] = {+1, +1, -1, -1}, dlen[4] = {lmu, lnu, lmu, lnu};
    const int start = (smu > 0 && snu > 0) ? 0 : (smu < 0 && snu > 0) ? 1 : (smu < 0 && snu < 0) ? 2 : 3;
    int c[3] = {x, y, z};
    cmat3<double> acc = m3_unit<double>();
    for (int k = 0; k < 4; k++) {
        const int j = (start + k) & 3;
        for (int n = 0; n < dlen[j]; n++) acc = su3_step(U, L, c, dmu[j], ddir[j], acc);
    }
    return acc;
}

// V (t^b e^b) V^+ as components: the adjoint transport R(V) e, R_ab = 2 tr(t^a V t^b V^+).
__device__ inline void su3_transport(const cmat3<double> &V, const double *e, double *out) {
    const cmat3<double> A = su3_form(e);
    su3_components(m3_mul(m3_mul(V, A), m3_dag(V)), out);
}

constexpr int kReduce3Threads = 128;

__device__ inline double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
    __syncthreads();
    return t;
}

// Improved E.B (ChernSimonsOperators.cpp:128-439; improved_e / improved_b of
// ovl_gauge.cu), one thread per (site, direction): E_mu . B_mu, B_mu from the
// plane orthogonal to mu; CTA partial sums.
__global__ void __launch_bounds__(kReduce3Threads)
    su3_ncsdot_kernel(const double *__restrict__ U, const double *__restrict__ E, Lattice L, double *partial) {
    __shared__ double sh[32];
    double v = 0.0;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 3 * L.V) {
        const int s = t / 3, mu = t % 3;
        int x, y, z;
        site_coords(L, s, x, y, z);
        const int plane[3][2] = {{1, 2}, {2, 0}, {0, 1}};
        // improved E_mu: -1/12, 7/12, 7/12, -1/12 of E_mu at x+mu, x, x-mu, x-2mu transported to x
        int c[3] = {x, y, z};
        c[mu] += 1;
        const int sp = site_index(L, c[0], c[1], c[2]);
        c[mu] -= 2;
        const int sm = site_index(L, c[0], c[1], c[2]);
        c[mu] -= 1;
        const int smm = site_index(L, c[0], c[1], c[2]);
        const cmat3<double> umd = m3_dag(load_su3(U, sm, mu));
        double e[8], w[8];
        for (int a = 0; a < 8; a++) e[a] = (7.0 / 12.0) * E[a + 8 * (mu + 3 * s)];
        su3_transport(load_su3(U, s, mu), E + 8 * (mu + 3 * sp), w);
        for (int a = 0; a < 8; a++) e[a] -= (1.0 / 12.0) * w[a];
        su3_transport(umd, E + 8 * (mu + 3 * sm), w);
        for (int a = 0; a < 8; a++) e[a] += (7.0 / 12.0) * w[a];
        su3_transport(m3_mul(umd, m3_dag(load_su3(U, smm, mu))), E + 8 * (mu + 3 * smm), w);
        for (int a = 0; a < 8; a++) e[a] -= (1.0 / 12.0) * w[a];
        // improved B: 5/12 of the four plaquettes, -1/24 of the eight 2x1 rectangles
        const int pm = plane[mu][0], pn = plane[mu][1];
        cmat3<double> avg;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) avg.m[i][j] = mk<double>(0.0, 0.0);
        const int sg[4][2] = {{+1, +1}, {-1, +1}, {-1, -1}, {+1, -1}};
        for (int q = 0; q < 4; q++) {
            const cmat3<double> box = su3_loop(U, L, x, y, z, pm, pn, sg[q][0], sg[q][1], 1, 1);
            const cmat3<double> r1 = su3_loop(U, L, x, y, z, pm, pn, sg[q][0], sg[q][1], 2, 1);
            const cmat3<double> r2 = su3_loop(U, L, x, y, z, pm, pn, sg[q][0], sg[q][1], 1, 2);
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    avg.m[i][j] = avg.m[i][j] + (5.0 / 12.0) * box.m[i][j] - (1.0 / 24.0) * (r1.m[i][j] + r2.m[i][j]);
        }
        double b[8];
        su3_retr_ita(avg, b);
        for (int a = 0; a < 8; a++) v += e[a] * 2.0 * b[a];
    }
    const double tot = block_sum(v, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

size_t su3_reduce_partial_doubles(const Lattice &L) {
    return (size_t)std::max(11 * ((L.V + kReduce3Threads - 1) / kReduce3Threads), 1);
}

void su3_launch_ncsdot(const double *U, const double *E, const Lattice &L, double *partial, double *out, cudaStream_t s) {
    const int nb = (3 * L.V + kReduce3Threads - 1) / kReduce3Threads;
    su3_ncsdot_kernel<<<nb, kReduce3Threads, 0, s>>>(U, E, L, partial);
    su3_sum_rows_kernel<1><<<1, 256, 0, s>>>(partial, nb, 0.125 / (M_PI * M_PI), out);
}

// ---------------------------------------------------- geodesic interpolation --
// Eigensystem of a hermitian 3x3 matrix by cyclic Jacobi rotations (each
// rotation diag(1, e^{-i phi}) R(theta) on a pair (p, q), a_pq = r e^{i phi},
// tan 2 theta = 2 r / (a_qq - a_pp)); columns of Vec are the eigenvectors.
__device__ inline void herm3_eigen(cmat3<double> A, cmat3<double> &Vec) {
    Vec = m3_unit<double>();
    for (int sweep = 0; sweep < 32; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < 3; i++) {
            diag += A.m[i][i].re * A.m[i][i].re;
            for (int j = i + 1; j < 3; j++) off += A.m[i][j].re * A.m[i][j].re + A.m[i][j].im * A.m[i][j].im;
        }
        if (off <= 1e-34 * diag || off < 1e-300) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                const double r = sqrt(A.m[p][q].re * A.m[p][q].re + A.m[p][q].im * A.m[p][q].im);
                if (r == 0.0) continue;
                const cpx<double> phc = mk<double>(A.m[p][q].re / r, -A.m[p][q].im / r);  // e^{-i phi}
                const double th = 0.5 * atan2(2.0 * r, A.m[q][q].re - A.m[p][p].re);
                double sn, cs;
                sincos(th, &sn, &cs);
                cmat3<double> J = m3_unit<double>();
                J.m[p][p] = mk<double>(cs, 0.0);
                J.m[p][q] = mk<double>(sn, 0.0);
                J.m[q][p] = -sn * phc;
                J.m[q][q] = cs * phc;
                A = m3_mul(m3_dag(J), m3_mul(A, J));
                Vec = m3_mul(Vec, J);
            }
    }
}

// A^a with exp(-i A^a t^a) = W (MatrixILog with C = -1,
// SU3/AlgebraOperations.cpp:186-234), through the eigenvectors of the hermitian
// H = (W + W^+)/2 + (W - W^+)/2i, which are W's while no two of its
// eigenphases add up to pi/2 (nearby links); phases made to sum to zero.
__device__ inline void su3_log(const cmat3<double> &W, double *out) {
    const cmat3<double> Wd = m3_dag(W);
    cmat3<double> H, Vec;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const cpx<double> s = W.m[i][j] + Wd.m[i][j], d = W.m[i][j] - Wd.m[i][j];
            H.m[i][j] = mk<double>(0.5 * s.re - 0.5 * d.im, 0.5 * s.im + 0.5 * d.re);  // s/2 - i d/2
        }
    herm3_eigen(H, Vec);
    double th[3], sum = 0.0;
    for (int j = 0; j < 3; j++) {
        cpx<double> e = mk<double>(0.0, 0.0);
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++) e = e + conj(Vec.m[i][j]) * W.m[i][k] * Vec.m[k][j];
        th[j] = atan2(e.im, e.re);
        sum += th[j];
    }
    if (fabs(sum) > M_PI) {
        int big = 0;
        for (int j = 1; j < 3; j++)
            if (fabs(th[j]) > fabs(th[big])) big = j;
        th[big] -= sum > 0 ? 2.0 * M_PI : -2.0 * M_PI;
        sum = th[0] + th[1] + th[2];
    }
    cmat3<double> G;  // -sum_j theta_j v_j v_j^+ = A^a t^a
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            cpx<double> t = mk<double>(0.0, 0.0);
            for (int j = 0; j < 3; j++) t = t + (th[j] - sum / 3.0) * (Vec.m[i][j] * conj(Vec.m[k][j]));
            G.m[i][k] = mk<double>(-t.re, -t.im);
        }
    su3_components(G, out);
}

// GeodesicInterpolation (SUNc/AdvancedOperations.cpp:432-443) for three
// colours: E_mid = A with exp(-i A t) = U_new U_old^+, U_mid = exp(-i c A t) U_old.
__global__ void su3_geodesic_kernel(const double *__restrict__ Uold, const double *__restrict__ Unew, double c,
                                    double *Umid, double *Emid, int n_links) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_links) return;
    const int site = l / 3, mu = l % 3;
    const cmat3<double> uo = load_su3(Uold, site, mu);
    double e[8];
    su3_log(m3_mul(load_su3(Unew, site, mu), m3_dag(uo)), e);
    for (int a = 0; a < 8; a++) Emid[8 * (size_t)l + a] = e[a];
    store_su3(Umid, site, mu, m3_mul(su3_exp(-c, e), uo));
}

void su3_launch_geodesic(const double *Uold, const double *Unew, double c, double *Umid, double *Emid, const Lattice &L,
                         cudaStream_t s) {
    const int n = 3 * L.V;
    su3_geodesic_kernel<<<(n + 127) / 128, 128, 0, s>>>(Uold, Unew, c, Umid, Emid, n);
}

// ------------------------------------------------------------------- bulk --
// E^2 (3), B^2 = 4 Re tr(1 - U_plaq) (3), Gauss squares, unitarity squares,
// Gauss max, unitarity max per CTA (bulk_kernel of ovl_gauge.cu for three colours).
__global__ void __launch_bounds__(kReduce3Threads)
    su3_bulk_kernel(const double *__restrict__ U, const double *__restrict__ E, Lattice L, double *partial) {
    __shared__ double sh[32];
    double v[10];
    for (int k = 0; k < 10; k++) v[k] = 0.0;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < L.V) {
        int x, y, z;
        site_coords(L, s, x, y, z);
        for (int mu = 0; mu < 3; mu++)
            for (int a = 0; a < 8; a++) {
                const double e = E[a + 8 * (mu + 3 * s)];
                v[mu] += e * e;
            }
        const int plane[3][2] = {{1, 2}, {2, 0}, {0, 1}};
        for (int k = 0; k < 3; k++) {
            const cmat3<double> pl = su3_loop(U, L, x, y, z, plane[k][0], plane[k][1], +1, +1, 1, 1);
            v[3 + k] = 4.0 * (3.0 - (pl.m[0][0].re + pl.m[1][1].re + pl.m[2][2].re));
        }
        double g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int mu = 0; mu < 3; mu++) {
            int c[3] = {x, y, z};
            c[mu] -= 1;
            const int sm = site_index(L, c[0], c[1], c[2]);
            double t[8];
            su3_transport(m3_dag(load_su3(U, sm, mu)), E + 8 * (mu + 3 * sm), t);
            for (int a = 0; a < 8; a++) g[a] += E[a + 8 * (mu + 3 * s)] - t[a];
        }
        double gmax = -1e300;
        for (int a = 0; a < 8; a++) {
            gmax = fmax(gmax, g[a]);
            v[6] += g[a] * g[a];
        }
        v[8] = gmax;
        double umax = 0.0;
        for (int mu = 0; mu < 3; mu++) {
            const cmat3<double> u = load_su3(U, s, mu), cc = m3_mul(u, m3_dag(u));
            double n = 0.0;
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    const double re = cc.m[i][j].re - (i == j ? 1.0 : 0.0), im = cc.m[i][j].im;
                    n += re * re + im * im;
                }
            umax = fmax(umax, sqrt(n));
            v[7] += n;
        }
        v[9] = umax;
    } else {
        v[8] = -1e300;
    }
    // sums of slots 0..7, maxima of 8 (Gauss, signed) and 9 (unitarity)
    double out[10];
    for (int k = 0; k < 8; k++) out[k] = block_sum(v[k], sh);
    for (int k = 8; k < 10; k++) {
        double t = v[k];
        for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_down_sync(0xffffffffu, t, o));
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
        __syncthreads();
        t = -1e300;
        if (threadIdx.x == 0)
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = fmax(t, sh[w]);
        __syncthreads();
        out[k] = t;
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 10; k++) partial[(size_t)blockIdx.x * 10 + k] = out[k];
}

__global__ void su3_bulk_finish_kernel(const double *__restrict__ partial, int n, Lattice L, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    CompSum cs[8];
    double gmax = -1e300, umax = 0.0;
    for (int i = 0; i < n; i++) {
        const double *p = partial + (size_t)i * 10;
        for (int k = 0; k < 8; k++) cs[k].add(p[k]);
        gmax = fmax(gmax, p[8]);
        umax = fmax(umax, p[9]);
    }
    double s[8];
    for (int k = 0; k < 8; k++) s[k] = cs[k].value();
    const double V = (double)L.V;
    double e2[3], b2[3];
    for (int k = 0; k < 3; k++) { e2[k] = s[k] / V; b2[k] = s[3 + k] / V; }
    out[0] = 0.5 * (e2[0] + e2[1] + e2[2] + b2[0] + b2[1] + b2[2]);
    out[1] = 0.5 * ((e2[1] + e2[2] + b2[1] + b2[2]) - (e2[0] + b2[0]));
    out[2] = 0.5 * ((e2[0] + e2[2] + b2[0] + b2[2]) - (e2[1] + b2[1]));
    out[3] = 0.5 * ((e2[0] + e2[1] + b2[0] + b2[1]) - (e2[2] + b2[2]));
    out[4] = 0.5 * (e2[0] + e2[1] + e2[2]);
    out[5] = 0.5 * (b2[0] + b2[1] + b2[2]);
    out[6] = fmax(gmax, 0.0);
    out[7] = sqrt(s[6] / (8.0 * V));  // over the Nc^2 - 1 components (GaussLawViolation.cpp:64)
    out[8] = umax;
    out[9] = sqrt(s[7] / (3.0 * V));
}

void su3_launch_bulk(const double *U, const double *E, const Lattice &L, double *partial, double *out, cudaStream_t s) {
    const int nb = (L.V + kReduce3Threads - 1) / kReduce3Threads;
    su3_bulk_kernel<<<nb, kReduce3Threads, 0, s>>>(U, E, L, partial);
    su3_bulk_finish_kernel<<<1, 32, 0, s>>>(partial, nb, L, out);
}

// ------------------------------------------------------------ staple force --
// E^a_mu(x) += -2 dt sum_{nu != mu} [Re tr(i t^a U_{mu,nu}) + Re tr(i t^a U_{mu,-nu})]
// (Dynamics.cpp:145-197; update_efield_kernel of ovl_gauge.cu for three colours).
__global__ void su3_efield_kernel(const double *__restrict__ U, double *E, Lattice L, double gamma) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 3 * L.V) return;
    const int site = l / 3, mu = l % 3;
    int x, y, z;
    site_coords(L, site, x, y, z);
    double f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int nu = 0; nu < 3; nu++) {
        if (nu == mu) continue;
        int c[3] = {x, y, z};
        cmat3<double> up = m3_unit<double>();
        up = su3_step(U, L, c, mu, +1, up);
        up = su3_step(U, L, c, nu, +1, up);
        up = su3_step(U, L, c, mu, -1, up);
        up = su3_step(U, L, c, nu, -1, up);
        int d[3] = {x, y, z};
        cmat3<double> dn = m3_unit<double>();
        dn = su3_step(U, L, d, mu, +1, dn);
        dn = su3_step(U, L, d, nu, -1, dn);
        dn = su3_step(U, L, d, mu, -1, dn);
        dn = su3_step(U, L, d, nu, +1, dn);
        double a[8], b[8];
        su3_retr_ita(up, a);
        su3_retr_ita(dn, b);
        for (int k = 0; k < 8; k++) f[k] += a[k] + b[k];
    }
    for (int k = 0; k < 8; k++) E[8 * (size_t)l + k] += gamma * f[k];
}

// The force of every link reads the links only, so one pass updates E in place.
void su3_launch_update_efield(const double *U, double *E, const Lattice &L, double dt_step, cudaStream_t s) {
    const int n = 3 * L.V;
    su3_efield_kernel<<<(n + 127) / 128, 128, 0, s>>>(U, E, L, -2.0 * dt_step);
}

// ------------------------------------------------------ Gauss restoration --
// GaussLawRestoration (GAUSSLAWFIXING/GaussRestore.cpp:13-168) for three
// colours: G^a(x) = sum_mu E_mu(x) - R(U_mu(x-mu)^+) E_mu(x-mu) into G (8 per
// site), CTA partial sums of G^2 and signed maxima (from 0).
__global__ void __launch_bounds__(kReduce3Threads)
    su3_gauss_violation_kernel(const double *__restrict__ U, const double *__restrict__ E, Lattice L, double *G,
                               double *partial) {
    __shared__ double sh[32];
    double sum = 0.0, mx = 0.0;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < L.V) {
        int x, y, z;
        site_coords(L, s, x, y, z);
        double g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int mu = 0; mu < 3; mu++) {
            int c[3] = {x, y, z};
            c[mu] -= 1;
            const int sm = site_index(L, c[0], c[1], c[2]);
            double t[8];
            su3_transport(m3_dag(load_su3(U, sm, mu)), E + 8 * (mu + 3 * sm), t);
            for (int a = 0; a < 8; a++) g[a] += E[a + 8 * (mu + 3 * s)] - t[a];
        }
        for (int a = 0; a < 8; a++) {
            G[a + 8 * (size_t)s] = g[a];
            sum += g[a] * g[a];
            mx = fmax(mx, g[a]);
        }
    }
    const double tsum = block_sum(sum, sh);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sh[w]);
        partial[2 * blockIdx.x] = tsum;
        partial[2 * blockIdx.x + 1] = m;
    }
}

__global__ void su3_gauss_finish_kernel(const double *__restrict__ partial, int n, double *out2) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sum = 0.0, mx = 0.0;
    for (int i = 0; i < n; i++) {
        sum += partial[2 * i];
        mx = fmax(mx, partial[2 * i + 1]);
    }
    out2[0] = sum;
    out2[1] = mx;
}

// E_mu(x) -= gamma (G(x) - R(U_mu(x)) G(x + mu))   (GaussRestore.cpp:72-118)
__global__ void su3_gauss_update_kernel(const double *__restrict__ U, const double *__restrict__ G,
                                        double *__restrict__ E, Lattice L, double gamma) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * L.V) return;
    const int s = t / 3, mu = t % 3;
    int x, y, z;
    site_coords(L, s, x, y, z);
    int c[3] = {x, y, z};
    c[mu] += 1;
    const int sp = site_index(L, c[0], c[1], c[2]);
    double up[8];
    su3_transport(load_su3(U, s, mu), G + 8 * (size_t)sp, up);
    for (int a = 0; a < 8; a++) E[a + 8 * (size_t)t] -= gamma * (G[a + 8 * (size_t)s] - up[a]);
}

void su3_launch_gauss_violation(const double *U, const double *E, const Lattice &L, double *G, double *partial,
                                double *out2, cudaStream_t s) {
    const int nb = (L.V + kReduce3Threads - 1) / kReduce3Threads;
    su3_gauss_violation_kernel<<<nb, kReduce3Threads, 0, s>>>(U, E, L, G, partial);
    su3_gauss_finish_kernel<<<1, 32, 0, s>>>(partial, nb, out2);
}

void su3_launch_gauss_update(const double *U, const double *G, double *E, const Lattice &L, double gamma,
                             cudaStream_t s) {
    const int n = 3 * L.V;
    su3_gauss_update_kernel<<<(n + 127) / 128, 128, 0, s>>>(U, G, E, L, gamma);
}

// ------------------------------------------------------------ back-reaction --
// The fermion force on E for three colours (ovl_force.cu with 3x3 links and
// t^a = lambda^a / 2): per site and mu the link-independent colour bilinears
//   C_ij = sum_m w_m sum_ab conj(psi_ia(x)) [g0 (1 - G_mu)]_ab psi_jb(x+mu),
// then dH_F/dtheta^a = (1/2V) Im tr(t^a Q), Q = M C^T, M the dressed link.
constexpr int kForce3PerSite = 3 * 18;  // mu, (i, j), (re, im)

template <typename T>
__global__ void __launch_bounds__(kModeBlock *kSites3)
    su3_force_modes_kernel(const cpx<T> *__restrict__ psi, Lattice L, int n_mb, int n_modes, int first_mode,
                           double *__restrict__ partial) {
    constexpr mono G0 = kGamma0;
    constexpr mono G0M[3] = {mono_mul(kGamma0, kGammaX), mono_mul(kGamma0, kGammaY), mono_mul(kGamma0, kGammaZ)};
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSites3 + threadIdx.y;
    const int g = blockIdx.y, groups = gridDim.y;
    if (site >= L.V) return;  // whole warps exit together
    int x, y, z;
    site_coords(L, site, x, y, z);
    int nb[3];
    for (int mu = 0; mu < 3; mu++) {
        int c[3] = {x, y, z};
        c[mu] += 1;
        nb[mu] = site_index(L, c[0], c[1], c[2]);
    }
    double acc[kForce3PerSite];
#pragma unroll
    for (int k = 0; k < kForce3PerSite; k++) acc[k] = 0.0;
    for (int mb = g; mb < n_mb; mb += groups) {
        const int mode = mb * kModeBlock + lane;
        const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
        cpx<double> f[3][kSpin];
        const cpx<T> *pf = psi + field_index3(L.V, mb, site, 0, lane);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int a = 0; a < kSpin; a++) {
                const cpx<T> v = ld(pf + (c * kSpin + a) * kModeBlock);
                f[c][a] = mk<double>((double)v.re, (double)v.im);
            }
#pragma unroll
        for (int mu = 0; mu < 3; mu++) {
            cpx<double> h[3][kSpin];
            const cpx<T> *ph = psi + field_index3(L.V, mb, nb[mu], 0, lane);
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int a = 0; a < kSpin; a++) {
                    const cpx<T> v = ld(ph + (c * kSpin + a) * kModeBlock);
                    h[c][a] = mk<double>((double)v.re, (double)v.im);
                }
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    const cpx<double> b0 = bilinear<double>(G0, f[i], h[j]);
                    const cpx<double> b1 = bilinear<double>(G0M[mu], f[i], h[j]);
                    const int k = 18 * mu + 2 * (3 * i + j);  // g0 (1 - G_mu) = g0 + i g0 g_mu
                    acc[k] += w * (b0.re - b1.im);
                    acc[k + 1] += w * (b0.im + b1.re);
                }
        }
    }
#pragma unroll
    for (int k = 0; k < kForce3PerSite; k++) {
        double t = acc[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        acc[k] = t;
    }
    if (lane == 0) {
        double *q = partial + ((size_t)g * L.V + site) * kForce3PerSite;
#pragma unroll
        for (int k = 0; k < kForce3PerSite; k++) q[k] = acc[k];
    }
}

// One thread per (site, mu).  out != null: out[a + 8 (mu + 3 site)] =
// dH_F/dtheta^a; otherwise E[a + 8 (mu + 3 site)] += coef dH_F/dtheta^a.
template <bool U1>
__global__ void su3_force_finish_kernel(const double *__restrict__ partial, int groups, const double *__restrict__ U,
                                        const double *__restrict__ u1, Lattice L, double *__restrict__ out,
                                        double *__restrict__ E, double coef) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * L.V) return;
    const int site = t / 3, mu = t % 3;
    cmat3<double> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C.m[i][j] = mk<double>(0.0, 0.0);
    for (int g = 0; g < groups; g++) {
        const double *p = partial + ((size_t)g * L.V + site) * kForce3PerSite + 18 * mu;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) C.m[i][j] = C.m[i][j] + mk<double>(p[2 * (3 * i + j)], p[2 * (3 * i + j) + 1]);
    }
    const Links3<false, U1> lk{U, u1, L.N0 * L.N1};
    const cmat3<double> M = lk.template get<double>(site, mu);
    cmat3<double> Q;  // M C^T
    for (int k = 0; k < 3; k++)
        for (int i = 0; i < 3; i++) Q.m[k][i] = M.m[k][0] * C.m[i][0] + M.m[k][1] * C.m[i][1] + M.m[k][2] * C.m[i][2];
    // Im tr(t^a Q) per generator (t^a = lambda^a / 2)
    const double r3 = 0.57735026918962576451;
    double f[8];
    f[0] = 0.5 * (Q.m[1][0].im + Q.m[0][1].im);
    f[1] = 0.5 * (Q.m[0][1].re - Q.m[1][0].re);  // Im((-i Q10 + i Q01)/2)
    f[2] = 0.5 * (Q.m[0][0].im - Q.m[1][1].im);
    f[3] = 0.5 * (Q.m[2][0].im + Q.m[0][2].im);
    f[4] = 0.5 * (Q.m[0][2].re - Q.m[2][0].re);
    f[5] = 0.5 * (Q.m[2][1].im + Q.m[1][2].im);
    f[6] = 0.5 * (Q.m[1][2].re - Q.m[2][1].re);
    f[7] = 0.5 * r3 * (Q.m[0][0].im + Q.m[1][1].im - 2.0 * Q.m[2][2].im);
    const double sc = 1.0 / (2.0 * L.V);
    const size_t o = 8 * (size_t)t;
    for (int a = 0; a < 8; a++) {
        if (out) out[o + a] = sc * f[a];
        else E[o + a] += coef * sc * f[a];
    }
}

int su3_force_groups(int n_mb) { return n_mb < 16 ? n_mb : 16; }

size_t su3_force_partial_doubles(const Lattice &L, int n_mb) {
    return (size_t)su3_force_groups(n_mb) * L.V * kForce3PerSite;
}

template <typename T>
void su3_launch_color_force(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                            int first_mode, double *partial, double *out, double *E, double coef, cudaStream_t s) {
    const int groups = su3_force_groups(n_mb);
    const dim3 block(kModeBlock, kSites3), grid((L.V + kSites3 - 1) / kSites3, groups);
    su3_force_modes_kernel<T><<<grid, block, 0, s>>>(reinterpret_cast<const cpx<T> *>(psi), L, n_mb, n_modes,
                                                      first_mode, partial);
    const int n = 3 * L.V;
    if (u1) su3_force_finish_kernel<true><<<(n + 127) / 128, 128, 0, s>>>(partial, groups, U, u1, L, out, E, coef);
    else su3_force_finish_kernel<false><<<(n + 127) / 128, 128, 0, s>>>(partial, groups, U, u1, L, out, E, coef);
}

// sum_m w_m Re <psi_m, i (D psi)_m> / 2V from psi and D psi (ovl_force.cu's
// energy reduction for 12-component modes): CTA partial sums, one CTA adds them.
template <typename T>
__global__ void __launch_bounds__(256)
    su3_energy_partial_kernel(const cpx<T> *__restrict__ psi, const cpx<T> *__restrict__ dpsi, size_t n, int V,
                              int n_modes, int first_mode, double *__restrict__ partial) {
    __shared__ double sh[32];
    const size_t per_mb = (size_t)V * kComp3 * kModeBlock;
    CompSum acc;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int mode = (int)(e / per_mb) * kModeBlock + (int)(e % kModeBlock);
        if (mode >= n_modes) continue;
        const cpx<T> a = ld(psi + e), d = ld(dpsi + e);
        const double im = (double)a.re * (double)d.im - (double)a.im * (double)d.re;  // Im conj(a) d
        acc.add((((first_mode + mode) & 1) == 0) ? -im : im);
    }
    const double t = block_sum(acc.value(), sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

template <typename T>
void su3_launch_fermion_energy(const void *psi, const void *dpsi, const Lattice &L, int n_mb, int n_modes,
                               int first_mode, double *partial, double *out, cudaStream_t s) {
    const size_t n = (size_t)n_mb * L.V * kComp3 * kModeBlock;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 1024);
    su3_energy_partial_kernel<T><<<blocks, 256, 0, s>>>(reinterpret_cast<const cpx<T> *>(psi),
                                                         reinterpret_cast<const cpx<T> *>(dpsi), n, L.V, n_modes,
                                                         first_mode, partial);
    su3_sum_rows_kernel<1><<<1, 256, 0, s>>>(partial, blocks, 1.0 / (2.0 * L.V), out);
}

// ------------------------------------------------------------ FP32 links --
// n = padded floats: link l's 18 doubles into floats [20 l, 20 l + 18), zeros after.
__global__ void su3_links_f32_kernel(const double *__restrict__ U, float *U32, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t l = i / kLink32Floats, k = i % kLink32Floats;
        U32[i] = k < 18 ? (float)U[18 * l + k] : 0.0f;
    }
}

void su3_launch_links_to_f32(const double *U, float *U32, const Lattice &L, cudaStream_t s) {
    const size_t n = (size_t)kLink32Floats * 3 * L.V;
    su3_links_f32_kernel<<<(int)std::min<size_t>((n + 255) / 256, 65535), 256, 0, s>>>(U, U32, n);
}

#define OVL_SU3_INSTANTIATE(T)                                                                                           \
    template void su3_launch_hop<T>(const Su3Links &, const void *, void *, const Lattice &, int, int, double, double,   \
                                    bool, cudaStream_t);                                                                \
    template void su3_chebyshev_apply<T>(ChebyshevWork &, const Su3Links &, const void *, void *, const Lattice &, int, \
                                         const double *, int, double, double, double, double, double, double, bool, int, \
                                         cudaStream_t, uint64_t *);                                                      \
    template void su3_launch_charges<T>(const double *, const double *, const void *, const Lattice &, int, int, int,   \
                                        double, double *, double *, cudaStream_t);                                      \
    template void su3_launch_currents<T>(const double *, const double *, const void *, const Lattice &, int, int, int,  \
                                         double, double *, double *, cudaStream_t);                                     \
    template void su3_launch_color_force<T>(const double *, const double *, const void *, const Lattice &, int, int,    \
                                            int, double *, double *, double *, double, cudaStream_t);                   \
    template void su3_launch_fermion_energy<T>(const void *, const void *, const Lattice &, int, int, int, double *,    \
                                               double *, cudaStream_t);
OVL_SU3_INSTANTIATE(double)
OVL_SU3_INSTANTIATE(float)

}  // namespace ovl
