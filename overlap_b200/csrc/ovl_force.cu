// Fermion back-reaction on the electric field, and the fermion energy.
//
// An extension without reference counterpart: the reference evolves the modes
// in a fixed gauge background (FERMIONS/WILSON/Update.cpp:48-79 moves the links
// with a constant E and never changes E).  With the links parametrised as
// U_mu(x) -> exp(i theta^a t^a) U_mu(x), t^a = sigma^a / 2, and the fermion energy
//   H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m>,   h_W = i D,
// the only terms of h_W that contain U_mu(x) are the hops between x and x+mu,
// and
//   dH_F/dtheta^a_mu(x) = -(1/2V) sum_m w_m Re[psi(x)^+ g0 (1 - G_mu) i t^a U_mu(x) psi(x+mu)]
// with G_mu = -i gamma_mu.  The colour structure separates: per site and mu,
//   C_ij = sum_m w_m sum_ab conj(psi_ia(x)) [g0 (1 - G_mu)]_ab psi_jb(x+mu)
// is link-independent (one pass over the modes, like the currents), and
//   dH_F/dtheta^a = -(1/2V) Re sum_ij (i t^a M)_ij C_ij = (1/4V) Im sum_ij (sigma^a M)_ij C_ij
// with M the (U(1)-dressed) link.  The link update U <- exp(-i dt E^a t^a) U of
// the reference makes d theta / dt = -E, so dE/dt = dH/dtheta conserves
// H_gauge + g^2 H_F.
#include "ovl_device.cuh"
#include "ovl_fp40.cuh"
#include "ovl_internal.h"

namespace ovl {

constexpr int kForceThreadsY = kSitesPerCta;

// One site's spinor of the lane's mode as complex doubles, from a field view
// (SrcPlain<T> or Src40, ovl_fp40.cuh).
template <class SRC>
__device__ __forceinline__ void force_load(const SRC &f, int V, int mb, int site, int lane,
                                           cpx<double> (&s)[kColours][kSpin]) {
    const size_t base = field_index(V, mb, site, 0, lane);
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) s[c][a] = f(base + (c * kSpin + a) * kModeBlock);
}

// partial[(g V + site) kForcePerSite + 8 mu + 2 (2 i + j) + {re, im}] = C_ij of
// mode-block group g (a warp is one site, its lanes the 32 modes of a block).
template <class SRC>
__global__ void __launch_bounds__(kModeBlock *kForceThreadsY)
    color_force_modes_kernel(SRC psi, Lattice L, int n_mb, int n_modes, int first_mode, int groups,
                             double *__restrict__ partial) {
    constexpr mono G0 = kGamma0;
    constexpr mono G0M[3] = {mono_mul(kGamma0, kGammaX), mono_mul(kGamma0, kGammaY), mono_mul(kGamma0, kGammaZ)};
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kForceThreadsY + threadIdx.y;
    const int g = blockIdx.y;
    if (site >= L.V) return;  // whole warps exit together
    int x, y, z;
    site_coords(L, site, x, y, z);
    int nb[3];
#pragma unroll
    for (int mu = 0; mu < 3; mu++) {
        int c[3] = {x, y, z};
        c[mu] += 1;
        nb[mu] = site_index(L, c[0], c[1], c[2]);
    }
    double acc[kForcePerSite];
#pragma unroll
    for (int k = 0; k < kForcePerSite; k++) acc[k] = 0.0;
    for (int mb = g; mb < n_mb; mb += groups) {
        const int mode = mb * kModeBlock + lane;
        const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
        cpx<double> f[kColours][kSpin];
        force_load(psi, L.V, mb, site, lane, f);
#pragma unroll
        for (int mu = 0; mu < 3; mu++) {
            cpx<double> h[kColours][kSpin];
            force_load(psi, L.V, mb, nb[mu], lane, h);
#pragma unroll
            for (int i = 0; i < kColours; i++)
#pragma unroll
                for (int j = 0; j < kColours; j++) {
                    const cpx<double> b0 = bilinear<double>(G0, f[i], h[j]);
                    const cpx<double> b1 = bilinear<double>(G0M[mu], f[i], h[j]);
                    // g0 (1 + i g_mu) = g0 + i g0 g_mu
                    const int k = 8 * mu + 2 * (2 * i + j);
                    acc[k] += w * (b0.re - b1.im);
                    acc[k + 1] += w * (b0.im + b1.re);
                }
        }
    }
#pragma unroll
    for (int k = 0; k < kForcePerSite; k++) {
        double t = acc[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        acc[k] = t;
    }
    if (lane == 0) {
        double *p = partial + ((size_t)g * L.V + site) * kForcePerSite;
#pragma unroll
        for (int k = 0; k < kForcePerSite; k++) p[k] = acc[k];
    }
}

// One thread per (site, mu): sum the groups' C, contract with the dressed link.
// out != null: out[a + 3 (mu + 3 site)] = dH_F/dtheta^a; otherwise
// E[a + 3 (mu + 3 site)] += coef dH_F/dtheta^a.
__global__ void color_force_finish_kernel(const double *__restrict__ partial, int groups, const double *__restrict__ U,
                                          const double2 *__restrict__ u1, Lattice L, double *__restrict__ out,
                                          double *__restrict__ E, double coef) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * L.V) return;
    const int site = t / 3, mu = t % 3;
    double c[8];
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] = 0.0;
    for (int g = 0; g < groups; g++) {
        const double *p = partial + ((size_t)g * L.V + site) * kForcePerSite + 8 * mu;
#pragma unroll
        for (int k = 0; k < 8; k++) c[k] += p[k];
    }
    const cpx<double> C00 = mk<double>(c[0], c[1]), C01 = mk<double>(c[2], c[3]);
    const cpx<double> C10 = mk<double>(c[4], c[5]), C11 = mk<double>(c[6], c[7]);
    const cmat2<double> M = dressed_link<double>(U, u1, site, mu, L.N0 * L.N1);
    // S_a = sum_ij (sigma^a M)_ij C_ij
    const cpx<double> m1c0 = M.m10 * C00 + M.m11 * C01;  // sum_j M_1j C_0j
    const cpx<double> m0c1 = M.m00 * C10 + M.m01 * C11;  // sum_j M_0j C_1j
    const cpx<double> m0c0 = M.m00 * C00 + M.m01 * C01;
    const cpx<double> m1c1 = M.m10 * C10 + M.m11 * C11;
    const double sx = m1c0.im + m0c1.im;
    const double sy = -m1c0.re + m0c1.re;  // Im(-i m1c0 + i m0c1)
    const double sz = m0c0.im - m1c1.im;
    const double s = 1.0 / (4.0 * L.V);
    const double f[3] = {s * sx, s * sy, s * sz};
    const size_t o = 3 * ((size_t)mu + 3 * (size_t)site);
    if (out) {
        out[o] = f[0];
        out[o + 1] = f[1];
        out[o + 2] = f[2];
    } else {
        E[o] += coef * f[0];
        E[o + 1] += coef * f[1];
        E[o + 2] += coef * f[2];
    }
}

int force_groups(int n_mb) { return n_mb < 16 ? n_mb : 16; }

size_t force_partial_doubles(const Lattice &L, int n_mb) { return (size_t)force_groups(n_mb) * L.V * kForcePerSite; }

template <class SRC>
static void color_force_from(const SRC &src, const double *U, const double *u1, const Lattice &L, int n_mb,
                             int n_modes, int first_mode, double *partial, double *out, double *E, double coef,
                             cudaStream_t stream) {
    const int groups = force_groups(n_mb);
    dim3 block(kModeBlock, kForceThreadsY);
    dim3 grid((L.V + kForceThreadsY - 1) / kForceThreadsY, groups);
    color_force_modes_kernel<SRC><<<grid, block, 0, stream>>>(src, L, n_mb, n_modes, first_mode, groups, partial);
    const int n = 3 * L.V;
    color_force_finish_kernel<<<(n + 127) / 128, 128, 0, stream>>>(partial, groups, U,
                                                                   reinterpret_cast<const double2 *>(u1), L, out, E,
                                                                   coef);
}

template <typename T>
void launch_color_force(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                        int first_mode, double *partial, double *out, double *E, double coef, cudaStream_t stream) {
    color_force_from(SrcPlain<T>{reinterpret_cast<const cpx<T> *>(psi)}, U, u1, L, n_mb, n_modes, first_mode, partial,
                     out, E, coef, stream);
}

void launch_color_force40(const double *U, const double *u1, const void *hi, const void *lo, const Lattice &L, int n_mb,
                          int n_modes, int first_mode, double *partial, double *out, double *E, double coef,
                          cudaStream_t stream) {
    color_force_from(Src40{reinterpret_cast<const uint2 *>(hi), reinterpret_cast<const unsigned char *>(lo)}, U, u1, L, n_mb,
                     n_modes, first_mode, partial, out, E, coef, stream);
}

template void launch_color_force<float>(const double *, const double *, const void *, const Lattice &, int, int, int,
                                        double *, double *, double *, double, cudaStream_t);
template void launch_color_force<double>(const double *, const double *, const void *, const Lattice &, int, int, int,
                                         double *, double *, double *, double, cudaStream_t);

// ------------------------------------------------------------ fermion energy --
// sum_m w_m Re <psi_m, i (D psi)_m> = -sum_m w_m Im <psi_m, (D psi)_m>: per CTA
// partial sums over a fixed grid, then one CTA adds them in order and scales
// by 1/(2V).  Element e of the mode-block layout belongs to mode
// 32 (e / (32 kComp V)) + e % 32.
constexpr int kEnergyThreads = 256;
constexpr int kEnergyBlocks = 1024;

template <class SRC>
__global__ void __launch_bounds__(kEnergyThreads)
    energy_partial_kernel(SRC psi, SRC dpsi, size_t n, int V, int n_modes, int first_mode, double *__restrict__ partial) {
    __shared__ double sh[kEnergyThreads];
    const size_t per_mb = (size_t)V * kComp * kModeBlock;
    CompSum acc;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int mode = (int)(e / per_mb) * kModeBlock + (int)(e % kModeBlock);
        if (mode >= n_modes) continue;
        const cpx<double> a = psi(e), d = dpsi(e);
        const double im = a.re * d.im - a.im * d.re;  // Im conj(a) d
        acc.add((((first_mode + mode) & 1) == 0) ? -im : im);
    }
    sh[threadIdx.x] = acc.value();
    __syncthreads();
    for (int s = kEnergyThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(kEnergyThreads)
    energy_finish_kernel(const double *__restrict__ partial, int blocks, double scale, double *__restrict__ out) {
    __shared__ double sh[kEnergyThreads];
    CompSum acc;
    for (int b = threadIdx.x; b < blocks; b += kEnergyThreads) acc.add(partial[b]);
    sh[threadIdx.x] = acc.value();
    __syncthreads();
    for (int s = kEnergyThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = scale * sh[0];
}

size_t energy_partial_doubles() { return kEnergyBlocks; }

template <class SRC>
static void energy_from(const SRC &psi, const SRC &dpsi, const Lattice &L, int n_mb, int n_modes, int first_mode,
                        double *partial, double *out, cudaStream_t stream) {
    const size_t n = (size_t)n_mb * L.V * kComp * kModeBlock;
    const size_t want = (n + kEnergyThreads - 1) / kEnergyThreads;
    const int blocks = (int)(want < (size_t)kEnergyBlocks ? want : (size_t)kEnergyBlocks);
    energy_partial_kernel<SRC><<<blocks, kEnergyThreads, 0, stream>>>(psi, dpsi, n, L.V, n_modes, first_mode, partial);
    energy_finish_kernel<<<1, kEnergyThreads, 0, stream>>>(partial, blocks, 1.0 / (2.0 * L.V), out);
}

template <typename T>
void launch_fermion_energy(const void *psi, const void *dpsi, const Lattice &L, int n_mb, int n_modes, int first_mode,
                           double *partial, double *out, cudaStream_t stream) {
    energy_from(SrcPlain<T>{reinterpret_cast<const cpx<T> *>(psi)}, SrcPlain<T>{reinterpret_cast<const cpx<T> *>(dpsi)},
                L, n_mb, n_modes, first_mode, partial, out, stream);
}

void launch_fermion_energy40(const void *hi, const void *lo, const void *dhi, const void *dlo, const Lattice &L,
                             int n_mb, int n_modes, int first_mode, double *partial, double *out, cudaStream_t stream) {
    energy_from(Src40{reinterpret_cast<const uint2 *>(hi), reinterpret_cast<const unsigned char *>(lo)},
                Src40{reinterpret_cast<const uint2 *>(dhi), reinterpret_cast<const unsigned char *>(dlo)}, L, n_mb, n_modes,
                first_mode, partial, out, stream);
}

template void launch_fermion_energy<float>(const void *, const void *, const Lattice &, int, int, int, double *,
                                           double *, cudaStream_t);
template void launch_fermion_energy<double>(const void *, const void *, const Lattice &, int, int, int, double *,
                                            double *, cudaStream_t);

}  // namespace ovl
