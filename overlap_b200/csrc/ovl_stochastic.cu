// Stochastic vacuum modes (no reference counterpart: the reference always uses
// the complete plane-wave basis, FermionField.cpp:145-328).
//
// The vacuum-subtracted mode sums of the currents are traces against
//   S = sum_m w_m |psi_m><psi_m| = V (P+ - P-),
// the difference of the projectors on the positive- and negative-energy
// states of the free Wilson Hamiltonian h = i D (particles carry w = +1,
// antiparticles w = -1; the plane waves have |psi(x)|^2 = 1 per site, hence V).
// With R noise vectors eta_r whose components are independent complex Z2
// numbers ((+-1 +- i)/sqrt 2: E[eta eta^+] = 1),
//   S ~ (V/R) sum_r (P+ eta_r)(P+ eta_r)^+ - (P- eta_r)(P- eta_r)^+,
// unbiased; so modes 2r and 2r+1 of a context are set to sqrt(V/R) P+ eta_r
// and sqrt(V/R) P- eta_r.  The noise is drawn in momentum space, where P+- are 4x4
// spin projectors per momentum: for unit links and a plane wave e^{ipx} u,
//   h(p) = g0 M(p) + sum_mu g0 g_mu sin p_mu,   M(p) = (6r + 2m - 2M)/2 - sum_mu cos p_mu,
// h(p)^2 = omega(p)^2 = M(p)^2 + sum_mu sin^2 p_mu, and P+-(p) = (1 +- h(p)/omega(p))/2
// (the free Wilson spinors of the plane-wave basis are the eigenvectors of
// the same h(p)).  psimid is the state half a step later, e^{-i h dt/2} psi:
// e^{-+ i omega dt/2} on the two parts.  A unitary inverse DFT, done as three
// passes of one-dimensional transforms, takes the vectors to position space.
// With Z2 noise, |eta(p)|^2 is exactly 1 per component, so the vacuum energy
// (1/2V) sum_m w_m <psi_m, h psi_m> = (1/2) Tr |h| is reproduced exactly by
// every sample.
#include <algorithm>

#include "ovl_fp40.cuh"
#include "ovl_internal.h"

namespace ovl {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    // SplitMix64 finaliser (Steele, Lea and Flood, OOPSLA 2014)
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Momentum-space modes of a chunk of mode blocks [mb0, mb0 + nmb): thread per
// (block, momentum, colour, lane).  mid: write the psimid version.
__global__ void stochastic_fill_kernel(cpx<double> *__restrict__ out, Lattice L, int mb0, int nmb, int n_modes,
                                       int first_mode, double amass, double dt, double inv_sqrt_r, uint64_t seed,
                                       int mid, int nc) {
    const size_t n = (size_t)nmb * L.V * nc * kModeBlock;
    const int ncomp = nc * kSpin;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int lane = (int)(t % kModeBlock);
        const int c = (int)((t / kModeBlock) % nc);
        const int q = (int)((t / ((size_t)kModeBlock * nc)) % L.V);
        const int mbl = (int)(t / ((size_t)kModeBlock * nc * L.V));
        const int mode = (mb0 + mbl) * kModeBlock + lane;
        cpx<double> res[kSpin];
        for (int a = 0; a < kSpin; a++) res[a] = mk<double>(0.0, 0.0);
        if (mode < n_modes) {
            const int g = first_mode + mode;  // global index: pair r, sign by parity
            const int r = g >> 1;
            const double sign = (g & 1) ? -1.0 : 1.0;
            int x, y, z;
            site_coords(L, q, x, y, z);
            const double p[3] = {2.0 * M_PI * x / L.N0, 2.0 * M_PI * y / L.N1, 2.0 * M_PI * z / L.N2};
            double s[3], M = 0.5 * amass;
            for (int mu = 0; mu < 3; mu++) {
                double sn, cs;
                sincos(p[mu], &sn, &cs);
                s[mu] = sn;
                M -= cs;
            }
            const double omega = sqrt(M * M + s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
            // noise of (pair, momentum, colour, spin)
            cpx<double> eta[kSpin];
            const uint64_t key = mix64(seed ^ mix64((uint64_t)r * 0x100000001b3ull + (uint64_t)q * 31u + (uint64_t)c));
            const uint64_t bits = mix64(key);
            for (int a = 0; a < kSpin; a++)
                eta[a] = mk<double>(((bits >> (2 * a)) & 1) ? -M_SQRT1_2 : M_SQRT1_2,
                                    ((bits >> (2 * a + 1)) & 1) ? -M_SQRT1_2 : M_SQRT1_2);
            // h eta = g0 M eta + sum_mu s_mu g0 g_mu eta
            constexpr mono G0 = kGamma0;
            constexpr mono G0M[3] = {mono_mul(kGamma0, kGammaX), mono_mul(kGamma0, kGammaY), mono_mul(kGamma0, kGammaZ)};
            cpx<double> h[kSpin];
            for (int a = 0; a < kSpin; a++) {
                cpx<double> v = iphase(G0.ph[a], eta[G0.perm[a]]);
                h[a] = mk<double>(M * v.re, M * v.im);
                for (int mu = 0; mu < 3; mu++) {
                    const cpx<double> w = iphase(G0M[mu].ph[a], eta[G0M[mu].perm[a]]);
                    h[a] = mk<double>(h[a].re + s[mu] * w.re, h[a].im + s[mu] * w.im);
                }
            }
            // (1 +- h/omega)/2 eta sqrt(V/R), times e^{-+ i omega dt/2} for psimid
            const double f = 0.5 * inv_sqrt_r, ho = sign / omega;
            double ph_re = 1.0, ph_im = 0.0;
            if (mid) sincos(-sign * 0.5 * omega * dt, &ph_im, &ph_re);
            for (int a = 0; a < kSpin; a++) {
                const double vr = f * (eta[a].re + ho * h[a].re), vi = f * (eta[a].im + ho * h[a].im);
                res[a] = mk<double>(vr * ph_re - vi * ph_im, vr * ph_im + vi * ph_re);
            }
        }
        for (int a = 0; a < kSpin; a++)
            out[(((size_t)mbl * L.V + q) * ncomp + c * kSpin + a) * kModeBlock + lane] = res[a];
    }
}

// One pass of the unitary inverse DFT along axis `ax` of a chunk in the
// mode-block layout: out(x_ax) = N^-1/2 sum_k in(k) e^{+2 pi i k x_ax / N}.
__global__ void idft_axis_kernel(const cpx<double> *__restrict__ in, cpx<double> *__restrict__ out, Lattice L, int nmb,
                                 int ax, int ncomp) {
    extern __shared__ cpx<double> tw[];  // e^{2 pi i j / N}, j < N
    const int N = ax == 0 ? L.N0 : ax == 1 ? L.N1 : L.N2;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * j / N, &sn, &cs);
        tw[j] = mk<double>(cs, sn);
    }
    __syncthreads();
    const double norm = rsqrt((double)N);
    const int stride = ax == 0 ? 1 : ax == 1 ? L.N0 : L.N0 * L.N1;
    const size_t n = (size_t)nmb * L.V * ncomp * kModeBlock;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int lane = (int)(e % kModeBlock);
        const int comp = (int)((e / kModeBlock) % ncomp);
        const int site = (int)((e / ((size_t)kModeBlock * ncomp)) % L.V);
        const int mb = (int)(e / ((size_t)kModeBlock * ncomp * L.V));
        int x, y, z;
        site_coords(L, site, x, y, z);
        const int xa = ax == 0 ? x : ax == 1 ? y : z;
        const int base = site - xa * stride;
        double re = 0.0, im = 0.0;
        for (int k = 0; k < N; k++) {
            const cpx<double> v = in[(((size_t)mb * L.V + base + k * stride) * ncomp + comp) * kModeBlock + lane];
            const cpx<double> w = tw[(k * xa) % N];
            re += v.re * w.re - v.im * w.im;
            im += v.re * w.im + v.im * w.re;
        }
        out[e] = mk<double>(norm * re, norm * im);
    }
}

// FP64 mode blocks -> the context's storage (kind 0 FP64, 1 FP32, 2 FP40).
__global__ void store_blocks_kernel(const cpx<double> *__restrict__ src, void *dst, unsigned char *lo, size_t off,
                                    size_t n, int kind) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const cpx<double> v = src[e];
        if (kind == 0) reinterpret_cast<cpx<double> *>(dst)[off + e] = v;
        else if (kind == 1) reinterpret_cast<cpx<float> *>(dst)[off + e] = mk<float>((float)v.re, (float)v.im);
        else store40(reinterpret_cast<uint2 *>(dst), lo, off + e, v.re, v.im);
    }
}

static int grid_of(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 65535); }

void launch_stochastic_modes(void *psi, void *psimid, void *psi_lo, void *psimid_lo, int kind, const Lattice &L,
                             int n_mb, int n_modes, int first_mode, double amass, double dt, uint64_t seed, int pairs,
                             double *scratch_a, double *scratch_b, int chunk_mb, cudaStream_t stream,
                             uint64_t *launches, int nc) {
    const int ncomp = nc * kSpin;
    const double inv_sqrt_r = std::sqrt((double)L.V / (double)pairs);  // sqrt(V / R)
    cpx<double> *a = reinterpret_cast<cpx<double> *>(scratch_a), *b = reinterpret_cast<cpx<double> *>(scratch_b);
    const int maxN = std::max(L.N0, std::max(L.N1, L.N2));
    uint64_t nl = 0;
    for (int f = 0; f < 2; f++) {
        void *dst = f == 0 ? psi : psimid;
        unsigned char *lo = reinterpret_cast<unsigned char *>(f == 0 ? psi_lo : psimid_lo);
        for (int mb0 = 0; mb0 < n_mb; mb0 += chunk_mb) {
            const int nmb = std::min(chunk_mb, n_mb - mb0);
            const size_t nfill = (size_t)nmb * L.V * nc * kModeBlock;
            const size_t nel = (size_t)nmb * L.V * ncomp * kModeBlock;
            stochastic_fill_kernel<<<grid_of(nfill), 256, 0, stream>>>(a, L, mb0, nmb, n_modes, first_mode, amass, dt,
                                                                    inv_sqrt_r, seed, f, nc);
            idft_axis_kernel<<<grid_of(nel), 256, sizeof(cpx<double>) * maxN, stream>>>(a, b, L, nmb, 0, ncomp);
            idft_axis_kernel<<<grid_of(nel), 256, sizeof(cpx<double>) * maxN, stream>>>(b, a, L, nmb, 1, ncomp);
            idft_axis_kernel<<<grid_of(nel), 256, sizeof(cpx<double>) * maxN, stream>>>(a, b, L, nmb, 2, ncomp);
            store_blocks_kernel<<<grid_of(nel), 256, 0, stream>>>(b, dst, lo, (size_t)mb0 * L.V * ncomp * kModeBlock, nel,
                                                                  kind);
            nl += 5;
        }
    }
    if (launches) *launches += nl;
}

}  // namespace ovl
