// Quasi-particle gauge fields on the device: InitialConditions::SetQuasiParticles
// (INITIALCONDITIONS/SetQuasiParticles.cpp:28-157) for unit lattice spacing in
// the Minkowski metric, two or three colours.
//
// Per lattice momentum k (p_mu = -i (1 - exp(-2 pi i k_mu / N_mu)),
// LATTICE/Momenta.cpp:4-8) and colour component a:
//   A_mu(k, a) = sqrt(f(p) V) (c1 xi1_mu + c2 xi2_mu),
//   E_mu(k, a) = sqrt(f(p) V) i omega (c1 xi1_mu + c2 xi2_mu),
// with the transverse polarisation vectors xi1, xi2 of
// MISC/MinkowskiWaveVectors.cpp:7-44 (base vector (1/sqrt3, 1/sqrt2, 1/sqrt6)),
// omega = |p|, the occupancy f(p) = n0 / sqrt(|p|^2/Qs^2 + 0.1) below Qs and 0
// above (SingleParticleDistribution, :27-40; a mode on |p| = Qs is not
// occupied, decided with a 1e-12 margin), and complex Gaussians c1, c2 of
// unit variance.  The unnormalised backward transform to position space
// (FFTW_BACKWARD in the reference) runs as three passes of one-dimensional
// transforms; then A(x) = 2 Re A / V, E(x) = 2 Re E / V and
// U_mu(x) = exp(-i A^a_mu(x) t^a) (SetCoordinateSpaceVariables, :112-151).
//
// The reference draws c1, c2 from its GSL generator in loop order.  Here each
// (k, a) draws its own from a counter-based generator, so the fields do not
// depend on the thread order and a host restatement reproduces them exactly:
//   n = (kx + N0 (ky + N1 kz)) * ncomp + a,  key = mix64(seed ^ mix64(n)),
//   u_j = ((mix64(key + j) >> 11) + 1) 2^-53 in (0, 1], j = 0..3,
//   (g0, g1), (g2, g3) by Box-Muller from (u0, u1), (u2, u3):
//     r = sqrt(-2 ln u_even), g = r cos(2 pi u_odd), r sin(2 pi u_odd),
//   c1 = (g0 + i g1) / sqrt 2,  c2 = (g2 + i g3) / sqrt 2,
// with mix64 the SplitMix64 finaliser (Steele, Lea and Flood, OOPSLA 2014).
#include <cmath>

#include "ovl_device.cuh"
#include "ovl_internal.h"
#include "ovl_su3.cuh"

namespace ovl {

namespace {

// A mode exactly on |p| = Qs is not occupied (the strict test of
// SingleParticleDistribution); the margin keeps rounding from deciding modes
// on that boundary (|p|^2 = 4 sin^2(pi/6) = 1 for k/N = 1/6, say).
constexpr double kEdge = 1.0 - 1e-12;

__device__ __forceinline__ uint64_t qp_mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double unit_interval(uint64_t bits) {
    return (double)((bits >> 11) + 1) * 0x1.0p-53;  // (0, 1]
}

__device__ __forceinline__ cpx<double> cmul(cpx<double> a, cpx<double> b) { return a * b; }

// Momentum-space fields of one (k, a): A and E, [mu][k][a] complex.
__global__ void qp_fill_kernel(cpx<double> *__restrict__ A, cpx<double> *__restrict__ E, Lattice L, int ncomp,
                               double n0, double qs, uint64_t seed) {
    const size_t n = (size_t)L.V * ncomp;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int a = (int)(t % ncomp);
        const int k = (int)(t / ncomp);
        int kk[3];
        site_coords(L, k, kk[0], kk[1], kk[2]);
        const int NN[3] = {L.N0, L.N1, L.N2};
        cpx<double> cdp[3];
        double p2 = 0.0, psq = 0.0;
        for (int m = 0; m < 3; m++) {
            double s, c;
            sincos(-2.0 * M_PI * kk[m] / (double)NN[m], &s, &c);
            cdp[m] = mk<double>(-s, -(1.0 - c));  // -i (1 - e^{-i theta})
            const double ab2 = cdp[m].re * cdp[m].re + cdp[m].im * cdp[m].im;
            p2 += ab2;
            const double pv = (cdp[m].re > 0.0 ? 1.0 : (cdp[m].re < 0.0 ? -1.0 : 0.0)) * sqrt(ab2);
            psq += pv * pv;
        }
        const double omega = sqrt(p2);
        const double occ = psq < kEdge * qs * qs ? n0 / sqrt(psq / (qs * qs) + 0.1) : 0.0;
        // transverse polarisation vectors (zero at p = 0)
        cpx<double> xi1[3] = {mk<double>(0.0, 0.0), mk<double>(0.0, 0.0), mk<double>(0.0, 0.0)};
        cpx<double> xi2[3] = {mk<double>(0.0, 0.0), mk<double>(0.0, 0.0), mk<double>(0.0, 0.0)};
        if (p2 > 0.0) {
            const double base[3] = {1.0 / sqrt(3.0), 1.0 / sqrt(2.0), 1.0 / (sqrt(2.0) * sqrt(3.0))};
            const double bsq = base[0] * base[0] + base[1] * base[1] + base[2] * base[2];
            const cpx<double> bdp = base[0] * cdp[0] + base[1] * cdp[1] + base[2] * cdp[2];
            const double nrm = sqrt(fabs(bsq - (bdp.re * bdp.re + bdp.im * bdp.im) / p2));
            const double den = nrm * sqrt(2.0 * omega);
            for (int m = 0; m < 3; m++) {
                const cpx<double> q = cmul(bdp, conj(cdp[m]));
                xi1[m] = mk<double>((base[m] - q.re / p2) / den, (-q.im / p2) / den);
            }
            for (int m = 0; m < 3; m++) {
                const cpx<double> v = cmul(cdp[(m + 1) % 3], conj(xi1[(m + 2) % 3])) -
                                      cmul(cdp[(m + 2) % 3], conj(xi1[(m + 1) % 3]));
                xi2[m] = mk<double>(v.re / omega, v.im / omega);
            }
        }
        // complex Gaussians c1, c2 of (k, a)
        const uint64_t key = qp_mix64(seed ^ qp_mix64((uint64_t)t));
        double g[4];
        for (int j = 0; j < 4; j += 2) {
            const double u0 = unit_interval(qp_mix64(key + j)), u1 = unit_interval(qp_mix64(key + j + 1));
            const double r = sqrt(-2.0 * log(u0));
            double s, c;
            sincos(2.0 * M_PI * u1, &s, &c);
            g[j] = r * c;
            g[j + 1] = r * s;
        }
        const cpx<double> c1 = mk<double>(g[0] * M_SQRT1_2, g[1] * M_SQRT1_2);
        const cpx<double> c2 = mk<double>(g[2] * M_SQRT1_2, g[3] * M_SQRT1_2);
        const double amp = sqrt(occ) * sqrt((double)L.V);
        for (int m = 0; m < 3; m++) {
            const cpx<double> mode = cmul(c1, xi1[m]) + cmul(c2, xi2[m]);
            A[(size_t)m * n + t] = mk<double>(amp * mode.re, amp * mode.im);
            E[(size_t)m * n + t] = mk<double>(-amp * omega * mode.im, amp * omega * mode.re);  // i omega
        }
    }
}

// One pass of the unnormalised backward transform, out(x) = sum_k in(k)
// e^{+2 pi i k x / N}, along axis `axis` of [field][site][a] arrays (fields
// of V * ncomp complex numbers; site = x + N0 (y + N1 z)).
__global__ void qp_dft_kernel(const cpx<double> *__restrict__ in, cpx<double> *__restrict__ out, Lattice L, int ncomp,
                              int fields, int axis) {
    const size_t per = (size_t)L.V * ncomp, n = per * fields;
    const int Nax = axis == 0 ? L.N0 : (axis == 1 ? L.N1 : L.N2);
    const int stride = axis == 0 ? 1 : (axis == 1 ? L.N0 : L.N0 * L.N1);
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int a = (int)(t % ncomp);
        const size_t f = t / per;
        const int site = (int)((t / ncomp) % L.V);
        int c[3];
        site_coords(L, site, c[0], c[1], c[2]);
        const int x = c[axis];
        const int row0 = site - x * stride;  // the site with coordinate 0 on this axis
        const cpx<double> *src = in + f * per;
        double re = 0.0, im = 0.0;
        for (int k = 0; k < Nax; k++) {
            const cpx<double> v = src[(size_t)(row0 + k * stride) * ncomp + a];
            double s, cs;
            sincospi(2.0 * (double)((long long)k * x % Nax) / Nax, &s, &cs);
            re += v.re * cs - v.im * s;
            im += v.re * s + v.im * cs;
        }
        out[t] = mk<double>(re, im);
    }
}

// Position-space fields: A = 2 Re A / V -> U = exp(-i A^a t^a); E = 2 Re E / V.
__global__ void qp_links_kernel(const cpx<double> *__restrict__ A, const cpx<double> *__restrict__ Ef, double *U,
                                double *E, Lattice L, int nc) {
    const int ncomp = nc * nc - 1;
    const size_t per = (size_t)L.V * ncomp;
    const int n_links = 3 * L.V;
    const double s = 2.0 / L.V;
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < n_links; l += gridDim.x * blockDim.x) {
        const int site = l / 3, mu = l % 3;
        double al[8];
        for (int a = 0; a < ncomp; a++) {
            al[a] = s * A[(size_t)mu * per + (size_t)site * ncomp + a].re;
            E[(size_t)ncomp * l + a] = s * Ef[(size_t)mu * per + (size_t)site * ncomp + a].re;
        }
        if (nc == 2) {
            store_link(U, site, mu, qexp(-1.0, al[0], al[1], al[2]));
        } else {
            store_su3(U, site, mu, su3_exp(-1.0, al));
        }
    }
}

}  // namespace

size_t quasi_particle_scratch_bytes(const Lattice &L, int nc) {
    return sizeof(cpx<double>) * 12 * (size_t)L.V * (nc * nc - 1);  // A and E (x3 directions), and a copy
}

void launch_quasi_particles(double *U, double *E, void *scratch, const Lattice &L, int nc, double n0, double qs,
                            uint64_t seed, int sm_count, cudaStream_t stream) {
    const int ncomp = nc * nc - 1;
    const size_t per = (size_t)L.V * ncomp;
    cpx<double> *buf = reinterpret_cast<cpx<double> *>(scratch);
    cpx<double> *AE = buf, *tmp = buf + 6 * per;  // A (3 fields) then E (3 fields); the transform's second buffer
    const int blocks = std::max(1, std::min((int)((per + 255) / 256), 16 * sm_count));
    qp_fill_kernel<<<blocks, 256, 0, stream>>>(AE, AE + 3 * per, L, ncomp, n0, qs, seed);
    const int tb = std::max(1, std::min((int)((6 * per + 255) / 256), 16 * sm_count));
    qp_dft_kernel<<<tb, 256, 0, stream>>>(AE, tmp, L, ncomp, 6, 0);
    qp_dft_kernel<<<tb, 256, 0, stream>>>(tmp, AE, L, ncomp, 6, 1);
    qp_dft_kernel<<<tb, 256, 0, stream>>>(AE, tmp, L, ncomp, 6, 2);
    const int lb = std::max(1, std::min((3 * L.V + 127) / 128, 16 * sm_count));
    qp_links_kernel<<<lb, 128, 0, stream>>>(tmp, tmp + 3 * per, U, E, L, nc);
}

}  // namespace ovl
