// Kernels over the mode batch other than the Wilson operator: the fermion
// currents and their lattice sums, layout conversion between the reference's
// per-mode arrays and the mode-block layout, and free plane-wave modes.

#include "ovl_device.cuh"
#include "ovl_fp40.cuh"
#include "ovl_internal.h"

namespace ovl {

// ---------------------------------------------------------------- currents --
// Fermions::Observables::ComputeCurrents, Wilson (FERMIONS/WILSON/Currents.cpp:7-309).
// For each mode (vacuum weight w = +1 even / -1 odd global index,
// FermionField.cpp:109-122) and site, with chi_mu = U_mu(x) psi(x+mu) and
// chib_mu = U_mu(x-mu)^+ psi(x-mu):
//   jV^0 = psi^+ psi              jA^0 = psi^+ g5 psi
//   jV^mu = Re psi^+ g0 g_mu chi   jA^mu = Re psi^+ g0 g_mu g5 chi
//   jVw^mu = Re psi^+ (-i r g0) chi, jAw^mu = Re psi^+ (-i r g0 g5) chi
//   PS = Re psi^+ (i g0 g5) psi
//   WA = Re[-6 psi^+ (-i r g0 g5) psi + sum_mu psi^+ (-i r g0 g5) (chi_mu + chib_mu)]
// summed over colours and modes, times 1/(2V) (Currents.cpp:289).
// Output per site: jV[4] jA[4] jVw[4] jAw[4] PS WA (jVw^0 = jAw^0 = 0).

constexpr int kCurrentsThreadsY = kSitesPerCta;

template <typename T>
__device__ __forceinline__ void load_site(const cpx<T> *__restrict__ f, int V, int mb, int site, int lane,
                                          cpx<T> (&s)[kColours][kSpin]) {
    const cpx<T> *p = f + field_index(V, mb, site, 0, lane);
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) s[c][a] = ld(p + (c * kSpin + a) * kModeBlock);
}

// One site's spinor of the lane's mode as complex doubles, from a field view
// (SrcPlain<T> or Src40, ovl_fp40.cuh).
template <class SRC>
__device__ __forceinline__ void load_site_d(const SRC &f, int V, int mb, int site, int lane,
                                            cpx<double> (&s)[kColours][kSpin]) {
    const size_t base = field_index(V, mb, site, 0, lane);
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) s[c][a] = f(base + (c * kSpin + a) * kModeBlock);
}

// sum over colours of psi^+ G h, in double
template <typename T>
__device__ __forceinline__ cpx<double> colour_bilinear(const mono &G, const cpx<T> (&f)[kColours][kSpin],
                                                        const cpx<double> (&h)[kColours][kSpin]) {
    cpx<double> t = mk<double>(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < kColours; c++) {
        cpx<double> fd[kSpin];
#pragma unroll
        for (int a = 0; a < kSpin; a++) fd[a] = mk<double>((double)f[c][a].re, (double)f[c][a].im);
        t = t + bilinear<double>(G, fd, h[c]);
    }
    return t;
}

template <class SRC>
__global__ void __launch_bounds__(kModeBlock *kCurrentsThreadsY)
    currents_kernel(const double *__restrict__ U, const double2 *__restrict__ u1, SRC psi, Lattice L, int n_mb,
                    int n_modes, int first_mode, int groups, double r, double *__restrict__ partial) {
    constexpr mono G1 = {{0, 1, 2, 3}, {0, 0, 0, 0}};
    constexpr mono G5 = kGamma5;
    constexpr mono G05 = mono_mul(kGamma0, kGamma5);
    constexpr mono G0 = kGamma0;
    constexpr mono GV[3] = {mono_mul(kGamma0, kGammaX), mono_mul(kGamma0, kGammaY), mono_mul(kGamma0, kGammaZ)};
    constexpr mono GA[3] = {mono_mul(GV[0], kGamma5), mono_mul(GV[1], kGamma5), mono_mul(GV[2], kGamma5)};

    const int lane = threadIdx.x;
    const int site = blockIdx.x * kCurrentsThreadsY + threadIdx.y;
    const int g = blockIdx.y;
    if (site >= L.V) return;  // whole warps exit together: a warp is one site
    int x, y, z;
    site_coords(L, site, x, y, z);
    const int V = L.V;

    double acc[kCurrentsPerSite];
#pragma unroll
    for (int k = 0; k < kCurrentsPerSite; k++) acc[k] = 0.0;

    int nb[3][2];
    for (int mu = 0; mu < 3; mu++) {
        int cp[3] = {x, y, z}, cm[3] = {x, y, z};
        cp[mu] += 1;
        cm[mu] -= 1;
        nb[mu][0] = site_index(L, cp[0], cp[1], cp[2]);
        nb[mu][1] = site_index(L, cm[0], cm[1], cm[2]);
    }

    for (int mb = g; mb < n_mb; mb += groups) {
        const int mode = mb * kModeBlock + lane;
        const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
        cpx<double> f[kColours][kSpin];
        load_site_d(psi, V, mb, site, lane, f);
        const cpx<double>(&fd)[kColours][kSpin] = f;
        double v[kCurrentsPerSite];
#pragma unroll
        for (int k = 0; k < kCurrentsPerSite; k++) v[k] = 0.0;
        v[0] = colour_bilinear(G1, f, fd).re;
        v[4] = colour_bilinear(G5, f, fd).re;
        const cpx<double> b05 = colour_bilinear(G05, f, fd);
        v[16] = -b05.im;                 // Re(i x)
        double wa = -6.0 * r * b05.im;   // -6 Re(-i r x)
#pragma unroll
        for (int mu = 0; mu < 3; mu++) {
            cpx<double> h[kColours][kSpin];
            cpx<double> chi[kColours][kSpin];
            // forward: chi = U_mu(x) psi(x+mu)
            load_site_d(psi, V, mb, nb[mu][0], lane, h);
            {
                const cmat2<double> M = dressed_link<double>(U, u1, site, mu, L.N0 * L.N1);
#pragma unroll
                for (int a = 0; a < kSpin; a++) mul(M, h[0][a], h[1][a], chi[0][a], chi[1][a]);
            }
            v[1 + mu] = colour_bilinear(GV[mu], f, chi).re;
            v[5 + mu] = colour_bilinear(GA[mu], f, chi).re;
            v[9 + mu] = r * colour_bilinear(G0, f, chi).im;
            const double aw = r * colour_bilinear(G05, f, chi).im;
            v[13 + mu] = aw;
            wa += aw;
            // backward: chib = U_mu(x-mu)^+ psi(x-mu)
            load_site_d(psi, V, mb, nb[mu][1], lane, h);
            {
                const cmat2<double> M = dressed_link<double>(U, u1, nb[mu][1], mu, L.N0 * L.N1);
#pragma unroll
                for (int a = 0; a < kSpin; a++) mul_dag(M, h[0][a], h[1][a], chi[0][a], chi[1][a]);
            }
            wa += r * colour_bilinear(G05, f, chi).im;
        }
        v[17] = wa;
#pragma unroll
        for (int k = 0; k < kCurrentsPerSite; k++) acc[k] += w * v[k];
    }
    // sum over the 32 modes of the warp, fixed order
#pragma unroll
    for (int k = 0; k < kCurrentsPerSite; k++) {
        double t = acc[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        acc[k] = t;
    }
    if (lane == 0) {
        double *p = partial + ((size_t)g * V + site) * kCurrentsPerSite;
#pragma unroll
        for (int k = 0; k < kCurrentsPerSite; k++) p[k] = acc[k];
    }
}

__global__ void currents_finish_kernel(const double *__restrict__ partial, int groups, int V, double scale,
                                       double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = V * kCurrentsPerSite;
    if (i >= n) return;
    double t = 0.0;
    for (int g = 0; g < groups; g++) t += partial[(size_t)g * n + i];
    out[i] = scale * t;
}

int currents_groups(int n_mb) { return n_mb < 16 ? n_mb : 16; }

void launch_currents_finish(const double *partial, int groups, const Lattice &L, double *per_site, cudaStream_t stream) {
    const int n = L.V * kCurrentsPerSite;
    currents_finish_kernel<<<(n + 255) / 256, 256, 0, stream>>>(partial, groups, L.V, 1.0 / (2.0 * L.V), per_site);
}

size_t currents_partial_doubles(const Lattice &L, int n_mb) {
    return (size_t)currents_groups(n_mb) * L.V * kCurrentsPerSite;
}

template <class SRC>
static void currents_from(const SRC &src, const double *U, const double *u1, const Lattice &L, int n_mb, int n_modes,
                          int first_mode, double r_wilson, double *partial, double *per_site, cudaStream_t stream) {
    const int groups = currents_groups(n_mb);
    dim3 block(kModeBlock, kCurrentsThreadsY);
    dim3 grid((L.V + kCurrentsThreadsY - 1) / kCurrentsThreadsY, groups);
    currents_kernel<SRC><<<grid, block, 0, stream>>>(U, reinterpret_cast<const double2 *>(u1), src, L, n_mb, n_modes,
                                                     first_mode, groups, r_wilson, partial);
    const int n = L.V * kCurrentsPerSite;
    currents_finish_kernel<<<(n + 255) / 256, 256, 0, stream>>>(partial, groups, L.V, 1.0 / (2.0 * L.V), per_site);
}

template <typename T>
void launch_currents(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                     int first_mode, double r_wilson, double *partial, double *per_site, cudaStream_t stream) {
    currents_from(SrcPlain<T>{reinterpret_cast<const cpx<T> *>(psi)}, U, u1, L, n_mb, n_modes, first_mode, r_wilson,
                  partial, per_site, stream);
}

void launch_currents40(const double *U, const double *u1, const void *hi, const void *lo, const Lattice &L, int n_mb,
                       int n_modes, int first_mode, double r_wilson, double *partial, double *per_site,
                       cudaStream_t stream) {
    currents_from(Src40{reinterpret_cast<const uint2 *>(hi), reinterpret_cast<const unsigned char *>(lo)}, U, u1, L, n_mb,
                  n_modes, first_mode, r_wilson, partial, per_site, stream);
}

// ----------------------------------------------------------------- charges --
// The lattice sums of the current densities without the per-site maps:
//   N_V = sum psi^+ psi,  N_5 = sum psi^+ g5 psi = 2 Re z,  PS = -2 Im z,
//   z = sum_c conj(psi_0) psi_2 + conj(psi_1) psi_3,
//   WA  = -12 r Im z + 2 r sum_mu Im psi^+(x) g0 g5 U_mu(x) psi(x+mu).
// For the WA sum the backward hop of Currents.cpp:273-283 is not evaluated:
// with Gamma = -i r g0 g5 hermitian, shifting x -> x+mu turns
// sum_x psi^+(x) Gamma U_mu(x-mu)^+ psi(x-mu) into the complex conjugate of the
// forward sum, whose real part is the same.  Each thread evaluates its mode
// and site in double whatever the mode precision; partial sums per CTA are
// added in a fixed order.
constexpr int kChargeVals = 4;

template <class SRC>
__global__ void __launch_bounds__(kModeBlock *kCurrentsThreadsY)
    charges_kernel(const double *__restrict__ U, const double2 *__restrict__ u1, SRC psi, Lattice L, int n_mb,
                   int n_modes, int first_mode, int groups, double r, double *__restrict__ partial) {
    __shared__ double sh[kCurrentsThreadsY][kChargeVals];
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kCurrentsThreadsY + threadIdx.y;
    const int g = blockIdx.y;
    CompSum sum[kChargeVals];
    if (site < L.V) {
        int x, y, z;
        site_coords(L, site, x, y, z);
        int nb[3];
        for (int mu = 0; mu < 3; mu++) {
            int c[3] = {x, y, z};
            c[mu] += 1;
            nb[mu] = site_index(L, c[0], c[1], c[2]);
        }
        cmat2<double> M[3];
        for (int mu = 0; mu < 3; mu++) M[mu] = dressed_link<double>(U, u1, site, mu, L.N0 * L.N1);
        for (int mb = g; mb < n_mb; mb += groups) {
            const int mode = mb * kModeBlock + lane;
            const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
            // the bilinears in double for every mode precision: each of the
            // ~1e8 terms of a lattice sum then carries a 1e-16 rounding error
            cpx<double> f[kColours][kSpin];
            load_site_d(psi, L.V, mb, site, lane, f);
            double nv = 0.0;
            cpx<double> zz = mk<double>(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < kColours; c++) {
#pragma unroll
                for (int a = 0; a < kSpin; a++) nv += f[c][a].re * f[c][a].re + f[c][a].im * f[c][a].im;
                zz = zz + cdot(f[c][0], f[c][2]) + cdot(f[c][1], f[c][3]);
            }
            double hop = 0.0;
#pragma unroll
            for (int mu = 0; mu < 3; mu++) {
                cpx<double> ht[kColours][kSpin];
                load_site_d(psi, L.V, mb, nb[mu], lane, ht);
                cpx<double> chi[kColours][kSpin];
#pragma unroll
                for (int a = 0; a < kSpin; a++) mul(M[mu], ht[0][a], ht[1][a], chi[0][a], chi[1][a]);
                cpx<double> b = mk<double>(0.0, 0.0);
#pragma unroll
                for (int c = 0; c < kColours; c++)
                    b = b + cdot(f[c][0], chi[c][2]) + cdot(f[c][1], chi[c][3]) - cdot(f[c][2], chi[c][0]) -
                        cdot(f[c][3], chi[c][1]);
                hop += b.im;
            }
            sum[0].add(w * nv);
            sum[1].add(w * 2.0 * zz.re);
            sum[2].add(w * -2.0 * zz.im);
            sum[3].add(w * (r * (-12.0 * zz.im + 2.0 * hop)));
        }
    }
    double acc[kChargeVals];
#pragma unroll
    for (int k = 0; k < kChargeVals; k++) acc[k] = sum[k].value();
#pragma unroll
    for (int k = 0; k < kChargeVals; k++) {
        double t = acc[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        acc[k] = t;
    }
    if (lane == 0)
        for (int k = 0; k < kChargeVals; k++) sh[threadIdx.y][k] = acc[k];
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        double *p = partial + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * kChargeVals;
        for (int k = 0; k < kChargeVals; k++) {
            double t = 0.0;
            for (int j = 0; j < kCurrentsThreadsY; j++) t += sh[j][k];
            p[k] = t;
        }
    }
}

__global__ void charges_finish_kernel(const double *__restrict__ partial, int n, double scale, double *__restrict__ out4) {
    __shared__ double sh[kChargeVals][256];
    CompSum t[kChargeVals];
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int k = 0; k < kChargeVals; k++) t[k].add(partial[(size_t)i * kChargeVals + k]);
    for (int k = 0; k < kChargeVals; k++) sh[k][threadIdx.x] = t[k].value();
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if ((int)threadIdx.x < stride)
            for (int k = 0; k < kChargeVals; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + stride];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < kChargeVals; k++) out4[k] = scale * sh[k][0];
}

size_t charges_partial_doubles(const Lattice &L, int n_mb) {
    return (size_t)currents_groups(n_mb) * ((L.V + kCurrentsThreadsY - 1) / kCurrentsThreadsY) * kChargeVals;
}

template <class SRC>
static void charges_from(const SRC &src, const double *U, const double *u1, const Lattice &L, int n_mb, int n_modes,
                         int first_mode, double r, double *partial, double *out4, cudaStream_t stream) {
    const int groups = currents_groups(n_mb);
    dim3 block(kModeBlock, kCurrentsThreadsY);
    dim3 grid((L.V + kCurrentsThreadsY - 1) / kCurrentsThreadsY, groups);
    charges_kernel<SRC><<<grid, block, 0, stream>>>(U, reinterpret_cast<const double2 *>(u1), src, L, n_mb, n_modes,
                                                    first_mode, groups, r, partial);
    charges_finish_kernel<<<1, 256, 0, stream>>>(partial, (int)(grid.x * grid.y), 1.0 / (2.0 * L.V), out4);
}

template <typename T>
void launch_charges(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                    int first_mode, double r_wilson, double *partial, double *out4, cudaStream_t stream) {
    // the arithmetic precision of r as before: the FP32 path rounds it to float
    charges_from(SrcPlain<T>{reinterpret_cast<const cpx<T> *>(psi)}, U, u1, L, n_mb, n_modes, first_mode,
                 (double)(T)r_wilson, partial, out4, stream);
}

void launch_charges40(const double *U, const double *u1, const void *hi, const void *lo, const Lattice &L, int n_mb,
                      int n_modes, int first_mode, double r_wilson, double *partial, double *out4, cudaStream_t stream) {
    charges_from(Src40{reinterpret_cast<const uint2 *>(hi), reinterpret_cast<const unsigned char *>(lo)}, U, u1, L, n_mb,
                 n_modes, first_mode, r_wilson, partial, out4, stream);
}

// Lattice sums of jV^0, jA^0, PS, WA from the per-site array, fixed order.
__global__ void site_sums_kernel(const double *__restrict__ per_site, int V, double *__restrict__ out4) {
    __shared__ double sh[4][256];
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (int s = threadIdx.x; s < V; s += blockDim.x) {
        const double *p = per_site + (size_t)s * kCurrentsPerSite;
        t[0] += p[0];
        t[1] += p[4];
        t[2] += p[16];
        t[3] += p[17];
    }
    for (int k = 0; k < 4; k++) sh[k][threadIdx.x] = t[k];
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if ((int)threadIdx.x < stride)
            for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + stride];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; k++) out4[k] = sh[k][0];
}

void launch_site_sums(const double *per_site, const Lattice &L, double * /*partial*/, double *out4, cudaStream_t stream) {
    site_sums_kernel<<<1, 256, 0, stream>>>(per_site, L.V, out4);
}

// ---------------------------------------------------------- layout change --
// ncomp complex components per mode and site: 8 (two colours) or 12 (three).
__device__ __forceinline__ size_t block_index(int V, int ncomp, int m, int site, int comp) {
    return (((size_t)(m / kModeBlock) * V + site) * ncomp + comp) * kModeBlock + m % kModeBlock;
}

template <typename T>
__global__ void ref_to_blocks_kernel(const double2 *__restrict__ ref, cpx<T> *__restrict__ blocks, int V, int m0,
                                     int count, unsigned char *__restrict__ lo, int ncomp) {
    const size_t n = (size_t)count * V * ncomp;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int comp = (int)(i % ncomp);
        const size_t ms = i / ncomp;
        const int site = (int)(ms % V);
        const int m = m0 + (int)(ms / V);
        const double2 v = ref[i];
        const size_t j = block_index(V, ncomp, m, site, comp);
        if (lo) store40(reinterpret_cast<uint2 *>(blocks), lo, j, v.x, v.y);  // 40-bit storage
        else st(blocks + j, mk<T>((T)v.x, (T)v.y));
    }
}

template <typename T>
__global__ void blocks_to_ref_kernel(const cpx<T> *__restrict__ blocks, double2 *__restrict__ ref, int V, int m0,
                                     int count, const unsigned char *__restrict__ lo, int ncomp) {
    const size_t n = (size_t)count * V * ncomp;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int comp = (int)(i % ncomp);
        const size_t ms = i / ncomp;
        const int site = (int)(ms % V);
        const int m = m0 + (int)(ms / V);
        const size_t j = block_index(V, ncomp, m, site, comp);
        if (lo) {  // 40-bit storage
            const cpx<double> v = Src40{reinterpret_cast<const uint2 *>(blocks), lo}(j);
            ref[i] = double2{v.re, v.im};
        } else {
            const cpx<T> v = blocks[j];
            ref[i] = double2{(double)v.re, (double)v.im};
        }
    }
}

static int grid_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 65535 ? b : 65535);
}

template <typename T>
void launch_ref_to_blocks(const double *ref, void *blocks, const Lattice &L, int m0, int count, cudaStream_t stream,
                          void *lo, int nc) {
    const size_t n = (size_t)count * L.V * nc * kSpin;
    if (n == 0) return;
    ref_to_blocks_kernel<T><<<grid_for(n), 256, 0, stream>>>(reinterpret_cast<const double2 *>(ref),
                                                             reinterpret_cast<cpx<T> *>(blocks), L.V, m0, count,
                                                             reinterpret_cast<unsigned char *>(lo), nc * kSpin);
}

template <typename T>
void launch_blocks_to_ref(const void *blocks, double *ref, const Lattice &L, int m0, int count, cudaStream_t stream,
                          const void *lo, int nc) {
    const size_t n = (size_t)count * L.V * nc * kSpin;
    if (n == 0) return;
    blocks_to_ref_kernel<T><<<grid_for(n), 256, 0, stream>>>(reinterpret_cast<const cpx<T> *>(blocks),
                                                             reinterpret_cast<double2 *>(ref), L.V, m0, count,
                                                             reinterpret_cast<const unsigned char *>(lo), nc * kSpin);
}

// ------------------------------------------------------------ plane waves --
// InitialConditions::SetFreeFermions with GetWilsonDiracSpinor / GetWilsonPhase
// (SetFreeFermions.cpp:3-56, FermionField.cpp:145-328), or for overlap
// fermions GetOverlapDiracSpinor / GetOverlapPhase (FermionField.cpp:331-528):
// the same helicity spinors of the momentum p and mass meff, which for the
// overlap operator are p = M hp / s and meff = M (1 + hp5 / s) with
// hp = sin(2 pi n / N), hp5 = 3 - M - sum cos(2 pi n / N), s = |(hp, hp5)|.
// Mode index
// particle + 2(colour + Nc(spin + 2(px + N0(py + N1 pz)))); particles
// exp(+i p.x) with frequency +w, antiparticles exp(-i p.x) with -w; psimid =
// psi exp(-i w dt / 2).
struct FreeMode { double u[8]; double omega; int colour, k0, k1, k2, particle, bad; };

__device__ FreeMode free_mode(const Lattice &L, int g, double r, double m, int nc, int overlap, double mdw) {
    FreeMode fm;
    const int N[3] = {L.N0, L.N1, L.N2};
    fm.particle = g % 2; g /= 2;
    fm.colour = g % nc; g /= nc;
    const int spin = g % 2; g /= 2;
    int k[3];
    k[0] = g % N[0]; g /= N[0];
    k[1] = g % N[1]; g /= N[1];
    k[2] = g % N[2];
    fm.k0 = k[0]; fm.k1 = k[1]; fm.k2 = k[2];
    double pp[3], meff = m, p2 = 0.0;
    if (overlap) {
        double hp5 = 3.0 - mdw, s2 = 0.0;
        for (int i = 0; i < 3; i++) {
            const int n = fm.particle == 0 ? k[i] : N[i] - k[i];
            pp[i] = sin(2.0 * M_PI * n / (double)N[i]);
            hp5 -= cos(2.0 * M_PI * n / (double)N[i]);
            s2 += pp[i] * pp[i];
        }
        const double sabs = sqrt(s2 + hp5 * hp5);
        for (int i = 0; i < 3; i++) {
            pp[i] = mdw * pp[i] / sabs;
            p2 += pp[i] * pp[i];
        }
        meff = mdw * (1.0 + hp5 / sabs);
    } else {
        for (int i = 0; i < 3; i++) {
            const int n = fm.particle == 0 ? k[i] : N[i] - k[i];
            pp[i] = sin(2.0 * M_PI * n / (double)N[i]);
            const double h = sin(M_PI * n / (double)N[i]);
            meff += 2.0 * r * h * h;
            p2 += pp[i] * pp[i];
        }
    }
    const double pabs = sqrt(p2);
    const double w = sqrt(p2 + meff * meff);
    const double omega = fm.particle == 0 ? w : -w;
    fm.omega = omega;
    // the axis cases test k == 0 or k == N/2 in integer division (FermionField.cpp:188,229):
    // for odd N the index (N-1)/2 takes them too, and its spinor fails the eigen check
    bool edge[3];
    for (int i = 0; i < 3; i++) edge[i] = (k[i] == 0 || k[i] == N[i] / 2);
    cpx<double> phi0, phi1;
    double hel;
    if (edge[0] && edge[1]) {
        phi0 = mk<double>(spin == 0 ? 1.0 : 0.0, 0.0);
        phi1 = mk<double>(spin == 0 ? 0.0 : 1.0, 0.0);
        hel = (spin == 0 ? 1.0 : -1.0) * pp[2] / fabs(pp[2]);
        if (edge[2]) hel = 0.0;
    } else {
        hel = spin == 0 ? 1.0 : -1.0;
        // q = -(pz - hel |p|) / (px - i py)
        const double nr = -(pp[2] - hel * pabs);
        const double den = pp[0] * pp[0] + pp[1] * pp[1];
        const cpx<double> q = mk<double>(nr * pp[0] / den, nr * pp[1] / den);
        const double d = sqrt(1.0 + q.re * q.re + q.im * q.im);
        phi0 = mk<double>(1.0 / d, 0.0);
        phi1 = mk<double>(q.re / d, q.im / d);
    }
    cpx<double> u[4];
    if (edge[0] && edge[1] && edge[2]) {
        const bool upper = (fm.particle == 0) == (meff >= 0.0);
        const cpx<double> zero = mk<double>(0.0, 0.0);
        u[0] = upper ? phi0 : zero;
        u[1] = upper ? phi1 : zero;
        u[2] = upper ? zero : phi0;
        u[3] = upper ? zero : phi1;
    } else {
        const double norm = sqrt(2.0 * omega * (omega - meff) / p2);
        const double lower = hel * (omega - meff) / pabs;
        u[0] = (1.0 / norm) * phi0;
        u[1] = (1.0 / norm) * phi1;
        u[2] = (lower / norm) * phi0;
        u[3] = (lower / norm) * phi1;
    }
    // eigen-residual |w u - H u| and |u|^2 - 1 with H = g0 (meff + p.gamma) (FermionField.cpp:270-312)
    constexpr mono G0 = kGamma0;
    constexpr mono GX0 = mono_mul(kGamma0, kGammaX), GY0 = mono_mul(kGamma0, kGammaY), GZ0 = mono_mul(kGamma0, kGammaZ);
    bool bad = false;
    double n2 = 0.0;
#pragma unroll
    for (int a = 0; a < 4; a++) {
        cpx<double> hu = (G0.ph[a] == 0 ? meff : -meff) * u[G0.perm[a]];
        hu = hu + pp[0] * iphase(GX0.ph[a], u[GX0.perm[a]]) + pp[1] * iphase(GY0.ph[a], u[GY0.perm[a]]) +
             pp[2] * iphase(GZ0.ph[a], u[GZ0.perm[a]]);
        const cpx<double> dlt = omega * u[a] - hu;
        if (sqrt(dlt.re * dlt.re + dlt.im * dlt.im) > 1e-6) bad = true;
        n2 += u[a].re * u[a].re + u[a].im * u[a].im;
    }
    if (fabs(n2 - 1.0) > 1e-6) bad = true;
    fm.bad = bad ? 1 : 0;
    for (int a = 0; a < 4; a++) { fm.u[2 * a] = u[a].re; fm.u[2 * a + 1] = u[a].im; }
    return fm;
}

__global__ void free_modes_kernel(FreeMode *info, int n_modes, int first_mode, Lattice L, double r, double m, int *bad,
                                  int nc, int overlap, double mdw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_modes) return;
    FreeMode fm = free_mode(L, first_mode + i, r, m, nc, overlap, mdw);
    info[i] = fm;
    if (fm.bad) atomicAdd(bad, 1);
}

template <typename T>
__global__ void free_fill_kernel(const FreeMode *__restrict__ info, cpx<T> *psi, cpx<T> *psimid, Lattice L, int n_modes,
                                 int n_mb, double dt, unsigned char *lo_psi, unsigned char *lo_mid, int nc) {
    const int lane = threadIdx.x;
    const int site = blockIdx.x * blockDim.y + threadIdx.y;
    const int mb = blockIdx.y;
    if (site >= L.V) return;
    const int m = mb * kModeBlock + lane;
    int x, y, z;
    site_coords(L, site, x, y, z);
    cpx<double> u[4] = {mk<double>(0, 0), mk<double>(0, 0), mk<double>(0, 0), mk<double>(0, 0)};
    cpx<double> phase = mk<double>(0, 0), half = mk<double>(1, 0);
    int colour = -1;
    if (m < n_modes) {
        const FreeMode fm = info[m];
        for (int a = 0; a < 4; a++) u[a] = mk<double>(fm.u[2 * a], fm.u[2 * a + 1]);
        const double arg = (fm.k0 * x) / (double)L.N0 + (fm.k1 * y) / (double)L.N1 + (fm.k2 * z) / (double)L.N2;
        double sn, cs;
        sincos((fm.particle == 0 ? 2.0 : -2.0) * M_PI * arg, &sn, &cs);
        phase = mk<double>(cs, sn);
        sincos(-0.5 * fm.omega * dt, &sn, &cs);
        half = mk<double>(cs, sn);
        colour = fm.colour;
    }
    for (int c = 0; c < nc; c++)
        for (int a = 0; a < kSpin; a++) {
            cpx<double> v = c == colour ? phase * u[a] : mk<double>(0, 0);
            cpx<double> vm = c == colour ? v * half : mk<double>(0, 0);
            const size_t idx = block_index(L.V, nc * kSpin, m, site, c * kSpin + a);
            if (lo_psi) {  // 40-bit storage
                store40(reinterpret_cast<uint2 *>(psi), lo_psi, idx, v.re, v.im);
                store40(reinterpret_cast<uint2 *>(psimid), lo_mid, idx, vm.re, vm.im);
            } else {
                st(psi + idx, mk<T>((T)v.re, (T)v.im));
                st(psimid + idx, mk<T>((T)vm.re, (T)vm.im));
            }
        }
}

template <typename T>
void launch_free_fermions(void *psi, void *psimid, const Lattice &L, int n_modes, int n_mb, int first_mode,
                          double r_wilson, double m_fermion, double dt, int *bad, cudaStream_t stream, void *lo_psi,
                          void *lo_mid, int nc, bool overlap, double m_dw) {
    FreeMode *info = nullptr;
    cudaMallocAsync(&info, sizeof(FreeMode) * (size_t)n_modes, stream);
    cudaMemsetAsync(bad, 0, sizeof(int), stream);
    free_modes_kernel<<<(n_modes + 127) / 128, 128, 0, stream>>>(info, n_modes, first_mode, L, r_wilson, m_fermion, bad,
                                                                 nc, overlap ? 1 : 0, m_dw);
    dim3 block(kModeBlock, kSitesPerCta);
    dim3 grid((L.V + kSitesPerCta - 1) / kSitesPerCta, n_mb);
    free_fill_kernel<T><<<grid, block, 0, stream>>>(info, reinterpret_cast<cpx<T> *>(psi), reinterpret_cast<cpx<T> *>(psimid),
                                                    L, n_modes, n_mb, dt, reinterpret_cast<unsigned char *>(lo_psi),
                                                    reinterpret_cast<unsigned char *>(lo_mid), nc);
    cudaFreeAsync(info, stream);
}

#define OVL_INSTANTIATE(T)                                                                                          \
    template void launch_charges<T>(const double *, const double *, const void *, const Lattice &, int, int, int,     \
                                    double, double *, double *, cudaStream_t);                                      \
    template void launch_currents<T>(const double *, const double *, const void *, const Lattice &, int, int, int,   \
                                     double, double *, double *, cudaStream_t);                                     \
    template void launch_ref_to_blocks<T>(const double *, void *, const Lattice &, int, int, cudaStream_t, void *,    \
                                          int);                                                                     \
    template void launch_blocks_to_ref<T>(const void *, double *, const Lattice &, int, int, cudaStream_t,          \
                                          const void *, int);                                                       \
    template void launch_free_fermions<T>(void *, void *, const Lattice &, int, int, int, double, double, double,    \
                                          int *, cudaStream_t, void *, void *, int, bool, double);
OVL_INSTANTIATE(double)
OVL_INSTANTIATE(float)

}  // namespace ovl
