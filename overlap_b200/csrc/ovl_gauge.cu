// Gauge-field kernels (all FP64): link update, staple force, the improved
// E.B of the Chern-Simons rate, and the bulk observables (energy, Gauss law,
// unitarity).  One thread per site or link; these fields are 3V links and are
// touched once or twice per leapfrog step, far from the fermion kernels' cost.
// Reductions are two-stage with a fixed summation order, so results do not
// depend on scheduling.

#include "ovl_device.cuh"
#include "ovl_internal.h"
#include "ovl_su3.cuh"

namespace ovl {

constexpr int kReduceThreads = 256;

// Fixed-order block sum of NV values per thread; thread 0 returns the totals.
template <int NV, bool MAX_LAST>
__device__ void block_reduce(double (&v)[NV], double *sh) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double t = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            double u = __shfl_down_sync(0xffffffffu, t, o);
            t = (MAX_LAST && k == NV - 1) ? fmax(t, u) : t + u;
        }
        v[k] = t;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int k = 0; k < NV; k++) sh[warp * NV + k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int k = 0; k < NV; k++) {
            double t = sh[k];
            for (int w = 1; w < nw; w++) t = (MAX_LAST && k == NV - 1) ? fmax(t, sh[w * NV + k]) : t + sh[w * NV + k];
            v[k] = t;
        }
    }
}

// ------------------------------------------------------------ link update --
// U <- exp(i cU E^a t^a) U with cU = -dt (Dynamics.cpp:97-138, Minkowski, a = 1).
// U32 (optional): FP32 copy of the updated links for the FP32 hopping kernels.
// reunit: project the updated link back onto SU(2), U / |U| (MaxTraceProjection,
// SUNc/SU2/GroupOperations.cpp:261-281); the reference never does this during
// the evolution (it only measures the violation), so it is off by default.
__global__ void update_links_kernel(double *U, const double *__restrict__ E, int n_links, double cU, float4 *U32,
                                    int reunit) {
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_links) return;
    const double *e = E + 3 * l;
    quat g = qexp(cU, e[0], e[1], e[2]);
    const int site = l / 3, mu = l % 3;
    quat u = qmul(g, load_link(U, site, mu));
    if (reunit) {
        const double nrm = sqrt(u.v0 * u.v0 + u.v1 * u.v1 + u.v2 * u.v2 + u.s * u.s);
        u = {u.v0 / nrm, u.v1 / nrm, u.v2 / nrm, u.s / nrm};
    }
    store_link(U, site, mu, u);
    if (U32) U32[l] = float4{(float)u.v0, (float)u.v1, (float)u.v2, (float)u.s};
}

void launch_update_links(double *U, const double *E, const Lattice &L, double dt_step, cudaStream_t stream,
                         float *U32, bool reunit) {
    const int n = 3 * L.V;
    update_links_kernel<<<(n + 255) / 256, 256, 0, stream>>>(U, E, n, -dt_step, reinterpret_cast<float4 *>(U32),
                                                             reunit ? 1 : 0);
}

// ------------------------------------------------------- Wilson loops ------
__device__ inline quat path_step(const double *__restrict__ U, const Lattice &L, int c[3], int mu, int dir, quat acc) {
    if (dir > 0) {
        quat u = load_link(U, site_index(L, c[0], c[1], c[2]), mu);
        c[mu] += 1;
        return qmul(acc, u);
    }
    c[mu] -= 1;
    return qmul(acc, qdag(load_link(U, site_index(L, c[0], c[1], c[2]), mu)));
}

// Counter-clockwise lmu x lnu loop in the (mu, nu) plane with (x, y, z) at its
// corner in quadrant (smu, snu), holonomy based at that corner.
__device__ quat loop(const double *__restrict__ U, const Lattice &L, int x, int y, int z, int mu, int nu, int smu,
                     int snu, int lmu, int lnu) {
    const int dmu[4] = {mu, nu, mu, nu}, ddir[4] = {+1, +1, -1, -1}, dlen[4] = {lmu, lnu, lmu, lnu};
    const int start = (smu > 0 && snu > 0) ? 0 : (smu < 0 && snu > 0) ? 1 : (smu < 0 && snu < 0) ? 2 : 3;
    int c[3] = {x, y, z};
    quat acc = {0.0, 0.0, 0.0, 1.0};
    for (int k = 0; k < 4; k++) {
        const int j = (start + k) & 3;
        for (int n = 0; n < dlen[j]; n++) acc = path_step(U, L, c, dmu[j], ddir[j], acc);
    }
    return acc;
}

// ------------------------------------------------------------ staple force --
// E^a_mu(x) += -2 dt sum_{nu != mu} [Re tr(i t^a U_{mu,nu}) + Re tr(i t^a U_{mu,-nu})],
// both staples written to start with U_mu(x) (Dynamics.cpp:145-197).
// Re tr(i t^a q) = -q_a.
__global__ void update_efield_kernel(const double *__restrict__ U, double *E, Lattice L, double gamma) {
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 3 * L.V) return;
    const int site = l / 3, mu = l % 3;
    int x, y, z;
    site_coords(L, site, x, y, z);
    double f[3] = {0.0, 0.0, 0.0};
    for (int nu = 0; nu < 3; nu++) {
        if (nu == mu) continue;
        int c[3] = {x, y, z};
        quat up = {0.0, 0.0, 0.0, 1.0};
        up = path_step(U, L, c, mu, +1, up);
        up = path_step(U, L, c, nu, +1, up);
        up = path_step(U, L, c, mu, -1, up);
        up = path_step(U, L, c, nu, -1, up);
        int d[3] = {x, y, z};
        quat dn = {0.0, 0.0, 0.0, 1.0};
        dn = path_step(U, L, d, mu, +1, dn);
        dn = path_step(U, L, d, nu, -1, dn);
        dn = path_step(U, L, d, mu, -1, dn);
        dn = path_step(U, L, d, nu, +1, dn);
        for (int a = 0; a < 3; a++) f[a] += -qcomp(up, a) - qcomp(dn, a);
    }
    for (int a = 0; a < 3; a++) E[3 * l + a] += gamma * f[a];
}

void launch_update_efield(const double *U, double *E, double * /*unused*/, const Lattice &L, double dt_step,
                          cudaStream_t stream) {
    const int n = 3 * L.V;
    update_efield_kernel<<<(n + 127) / 128, 128, 0, stream>>>(U, E, L, -2.0 * dt_step);
}

// ----------------------------------------------------------------- NCsDot --
// Improved E_mu at x: -1/12, 7/12, 7/12, -1/12 of E_mu at x+mu, x, x-mu, x-2mu
// transported to x (ChernSimonsOperators.cpp:379-401).
__device__ void improved_e(const double *__restrict__ U, const double *__restrict__ E, const Lattice &L, int x, int y,
                           int z, int mu, double out[3]) {
    int c[3] = {x, y, z};
    const int s0 = site_index(L, c[0], c[1], c[2]);
    c[mu] += 1;
    const int sp = site_index(L, c[0], c[1], c[2]);
    c[mu] -= 2;
    const int sm = site_index(L, c[0], c[1], c[2]);
    c[mu] -= 1;
    const int smm = site_index(L, c[0], c[1], c[2]);
    const quat um = load_link(U, sm, mu);
    adj3 Rp = adjoint(load_link(U, s0, mu));
    adj3 Rm = adjoint(qdag(um));
    adj3 Rmm = adjoint(qmul(qdag(um), qdag(load_link(U, smm, mu))));
    const double *ep = E + 3 * (mu + 3 * sp), *e0 = E + 3 * (mu + 3 * s0);
    const double *em = E + 3 * (mu + 3 * sm), *emm = E + 3 * (mu + 3 * smm);
    for (int a = 0; a < 3; a++) {
        double t = (7.0 / 12.0) * e0[a];
        for (int b = 0; b < 3; b++)
            t += -(1.0 / 12.0) * Rp.r[a][b] * ep[b] + (7.0 / 12.0) * Rm.r[a][b] * em[b] -
                 (1.0 / 12.0) * Rmm.r[a][b] * emm[b];
        out[a] = t;
    }
}

// Improved B for the (mu, nu) plane: 5/12 of the four plaquettes and -1/24 of
// the eight 2x1 rectangles with x at a corner, all counter-clockwise and based
// at x; B^a = 2 Re tr(i t^a avg) (ChernSimonsOperators.cpp:283-421).
__device__ void improved_b(const double *__restrict__ U, const Lattice &L, int x, int y, int z, int mu, int nu,
                           double out[3]) {
    double avg[4] = {0.0, 0.0, 0.0, 0.0};
    const int sg[4][2] = {{+1, +1}, {-1, +1}, {-1, -1}, {+1, -1}};
    for (int q = 0; q < 4; q++) {
        quat box = loop(U, L, x, y, z, mu, nu, sg[q][0], sg[q][1], 1, 1);
        quat r1 = loop(U, L, x, y, z, mu, nu, sg[q][0], sg[q][1], 2, 1);
        quat r2 = loop(U, L, x, y, z, mu, nu, sg[q][0], sg[q][1], 1, 2);
        avg[0] += (5.0 / 12.0) * box.v0 - (1.0 / 24.0) * (r1.v0 + r2.v0);
        avg[1] += (5.0 / 12.0) * box.v1 - (1.0 / 24.0) * (r1.v1 + r2.v1);
        avg[2] += (5.0 / 12.0) * box.v2 - (1.0 / 24.0) * (r1.v2 + r2.v2);
    }
    for (int a = 0; a < 3; a++) out[a] = -2.0 * avg[a];
}

__global__ void __launch_bounds__(kReduceThreads) ncsdot_kernel(const double *__restrict__ U, const double *__restrict__ E,
                                                                 Lattice L, double *partial) {
    __shared__ double sh[32];
    CompSum sum;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.V; s += gridDim.x * blockDim.x) {
        int x, y, z;
        site_coords(L, s, x, y, z);
        const int plane[3][2] = {{1, 2}, {2, 0}, {0, 1}};  // B_x from yz, B_y from zx, B_z from xy
        for (int mu = 0; mu < 3; mu++) {
            double e[3], b[3];
            improved_e(U, E, L, x, y, z, mu, e);
            improved_b(U, L, x, y, z, plane[mu][0], plane[mu][1], b);
            sum.add(e[0] * b[0] + e[1] * b[1] + e[2] * b[2]);
        }
    }
    double v[1] = {sum.value()};
    block_reduce<1, false>(v, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

template <int NV, bool MAX_LAST>
__global__ void finish_kernel(const double *__restrict__ partial, int n, double *out, double scale) {
    __shared__ double sh[32 * NV];
    double v[NV];
    CompSum t[NV];
    double mx = -1e300;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int k = 0; k < NV; k++) {
            const double p = partial[(size_t)i * NV + k];
            if (MAX_LAST && k == NV - 1) mx = fmax(mx, p);
            else t[k].add(p);
        }
    for (int k = 0; k < NV; k++) v[k] = (MAX_LAST && k == NV - 1) ? mx : t[k].value();
    block_reduce<NV, MAX_LAST>(v, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < NV; k++) out[k] = (MAX_LAST && k == NV - 1) ? v[k] : scale * v[k];
}

static int reduce_blocks(int V) {
    int b = (V + kReduceThreads - 1) / kReduceThreads;
    return b < 1024 ? b : 1024;
}

size_t ncsdot_partial_doubles(const Lattice &L) { return (size_t)reduce_blocks(L.V); }

void launch_ncsdot(const double *U, const double *E, const Lattice &L, double *partial, double *out, cudaStream_t stream) {
    const int nb = reduce_blocks(L.V);
    ncsdot_kernel<<<nb, kReduceThreads, 0, stream>>>(U, E, L, partial);
    // NCsDot = E.B / (8 pi^2) (ChernSimonsDerivative.cpp:48)
    finish_kernel<1, false><<<1, kReduceThreads, 0, stream>>>(partial, nb, out, 0.125 / (M_PI * M_PI));
}

// One partial sum per block of kReduceThreads sites, for callers that provide
// their own partial-sum storage of `blocks` doubles.
int ncsdot_blocks_exact(const Lattice &L) { return (L.V + kReduceThreads - 1) / kReduceThreads; }

void launch_ncsdot_into(const double *U, const double *E, const Lattice &L, int blocks, double *partial, double *out,
                        cudaStream_t stream) {
    ncsdot_kernel<<<blocks, kReduceThreads, 0, stream>>>(U, E, L, partial);
    finish_kernel<1, false><<<1, kReduceThreads, 0, stream>>>(partial, blocks, out, 0.125 / (M_PI * M_PI));
}

// ----------------------------------------------------- geodesic interpolation --
// GeodesicInterpolation (SUNc/AdvancedOperations.cpp:432-443) on every link:
// E_mid = -i log(U_new U_old^+) (MatrixILog with C = -1, SU2/AlgebraOperations.cpp:59-74),
// U_mid = exp(-i c E_mid) U_old; E_mid carries the Minkowski factor cE = 1
// (CoolingMethod.cpp:37-66).
__global__ void geodesic_kernel(const double *__restrict__ Uold, const double *__restrict__ Unew, double c,
                                double *Umid, double *Emid, int n_links) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_links) return;
    const int site = l / 3, mu = l % 3;
    const quat uo = load_link(Uold, site, mu);
    const quat b = qmul(load_link(Unew, site, mu), qdag(uo));
    const double d = sqrt(b.v0 * b.v0 + b.v1 * b.v1 + b.v2 * b.v2);
    double e0 = 0.0, e1 = 0.0, e2 = 0.0;
    if (d != 0.0) {
        const double arg = atan2(d, b.s);
        const double M = 2.0 * arg / (-1.0 * d);
        e0 = M * b.v0;
        e1 = M * b.v1;
        e2 = M * b.v2;
    }
    Emid[3 * l + 0] = e0;
    Emid[3 * l + 1] = e1;
    Emid[3 * l + 2] = e2;
    store_link(Umid, site, mu, qmul(qexp(-c, e0, e1, e2), uo));
}

void launch_geodesic(const double *Uold, const double *Unew, double c, double *Umid, double *Emid, const Lattice &L,
                     cudaStream_t stream) {
    const int n = 3 * L.V;
    geodesic_kernel<<<(n + 255) / 256, 256, 0, stream>>>(Uold, Unew, c, Umid, Emid, n);
}

// ----------------------------------------------------- handmade sphaleron --
// InitialConditions::HandmadeSphaleron::Setup (INITIALCONDITIONS/HandmadeSphaleron.cpp:114-170):
// G(x) in SU(2) from the site's lattice coordinates -- arctangent map onto the
// torus (LocalizedLatticeMap, :7-18), tan((t - pi) / 2) onto R^3 with the point
// at infinity where an angle is 0 or 2 pi (TorusProjection, :22-31), inverse
// stereographic projection onto S^3 (:35-60) --; the links start at 1 and the
// field E = -i log(G(x) G(x+mu)^+) / t_sph (GeodesicInterpolation from the unit
// links, MatrixILog with C = -1, :73-101) carries them to G(x) G(x+mu)^+ in the
// time t_sph.  One thread per link; the two G's it needs are recomputed.
__device__ __forceinline__ double torus_angle(int i, int n, double r) {
    const double b = 1.0 / r, h = n / 2.0;
    return 2.0 * M_PI * (atan(b * (i - h)) - atan(b * (-h))) / (atan(b * h) - atan(-b * h));
}

__device__ __forceinline__ quat sphaleron_g(const Lattice &L, int x, int y, int z, double r) {
    const double tx = torus_angle(x, L.N0, r), ty = torus_angle(y, L.N1, r), tz = torus_angle(z, L.N2, r);
    const double tp = 2.0 * M_PI;
    if (tx == 0.0 || tx == tp || ty == 0.0 || ty == tp || tz == 0.0 || tz == tp) return quat{0.0, 0.0, 0.0, 1.0};
    const double a = tan(0.5 * (tx - M_PI)), b = tan(0.5 * (ty - M_PI)), c = tan(0.5 * (tz - M_PI));
    const double q = a * a + b * b + c * c, u = (q - 1.0) / (q + 1.0);
    return quat{(1.0 - u) * a, (1.0 - u) * b, (1.0 - u) * c, u};
}

__global__ void sphaleron_kernel(double *U, double *E, double *Ufinal, Lattice L, double r, double inv_t,
                                 int n_links) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_links) return;
    const int site = l / 3, mu = l % 3;
    int x, y, z;
    site_coords(L, site, x, y, z);
    const quat g = sphaleron_g(L, x, y, z, r);
    const quat gn = sphaleron_g(L, mu == 0 ? (x + 1) % L.N0 : x, mu == 1 ? (y + 1) % L.N1 : y,
                                mu == 2 ? (z + 1) % L.N2 : z, r);
    const quat b = qmul(g, qdag(gn));
    const double d = sqrt(b.v0 * b.v0 + b.v1 * b.v1 + b.v2 * b.v2);
    const double m = d != 0.0 ? 2.0 * atan2(d, b.s) / (-1.0 * d) : 0.0;
    E[3 * l + 0] = (m * b.v0) * inv_t;
    E[3 * l + 1] = (m * b.v1) * inv_t;
    E[3 * l + 2] = (m * b.v2) * inv_t;
    store_link(U, site, mu, quat{0.0, 0.0, 0.0, 1.0});
    if (Ufinal) store_link(Ufinal, site, mu, b);
}

void launch_sphaleron(double *U, double *E, double *Ufinal, const Lattice &L, double r, double t,
                      cudaStream_t stream) {
    const int n = 3 * L.V;
    sphaleron_kernel<<<(n + 255) / 256, 256, 0, stream>>>(U, E, Ufinal, L, r, 1.0 / t, n);
}

// ------------------------------------------------------------------- bulk --
// Per-thread sums: E^2 per direction (3), B^2 per direction (3), Gauss
// violation squares, unitarity squares, unitarity max, Gauss max (last, max-reduced).
constexpr int kBulkVals = 10;

__global__ void __launch_bounds__(kReduceThreads) bulk_kernel(const double *__restrict__ U, const double *__restrict__ E,
                                                               Lattice L, double *partial) {
    __shared__ double sh[32 * kBulkVals];
    double v[kBulkVals];
    for (int k = 0; k < kBulkVals; k++) v[k] = 0.0;
    double umax = 0.0, gmax = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.V; s += gridDim.x * blockDim.x) {
        int x, y, z;
        site_coords(L, s, x, y, z);
        for (int mu = 0; mu < 3; mu++)
            for (int a = 0; a < 3; a++) {
                double e = E[a + 3 * (mu + 3 * s)];
                v[mu] += e * e;
            }
        // B^2_k = 4 Re tr(1 - U_plaq) of the plaquette orthogonal to k (BulkObservables.cpp:72-77)
        const int plane[3][2] = {{1, 2}, {2, 0}, {0, 1}};
        for (int k = 0; k < 3; k++) {
            quat pl = loop(U, L, x, y, z, plane[k][0], plane[k][1], +1, +1, 1, 1);
            v[3 + k] += 4.0 * 2.0 * (1.0 - pl.s);
        }
        // G^a = sum_mu E_mu(x) - (U^+ E U)(x - mu)
        double g[3] = {0.0, 0.0, 0.0};
        for (int mu = 0; mu < 3; mu++) {
            int c[3] = {x, y, z};
            c[mu] -= 1;
            const int sm = site_index(L, c[0], c[1], c[2]);
            adj3 R = adjoint(qdag(load_link(U, sm, mu)));
            for (int a = 0; a < 3; a++) {
                double t = E[a + 3 * (mu + 3 * s)];
                for (int b = 0; b < 3; b++) t -= R.r[a][b] * E[b + 3 * (mu + 3 * sm)];
                g[a] += t;
            }
        }
        for (int a = 0; a < 3; a++) {
            gmax = fmax(gmax, g[a]);  // signed maximum, as GaussLawViolation.cpp:44
            v[6] += g[a] * g[a];
        }
        for (int mu = 0; mu < 3; mu++) {
            quat u = load_link(U, s, mu);
            double dev = fabs(u.v0 * u.v0 + u.v1 * u.v1 + u.v2 * u.v2 + u.s * u.s - 1.0);
            umax = fmax(umax, dev);
            v[7] += dev * dev;
        }
    }
    v[8] = umax;
    v[9] = gmax;
    // max-reduce slot 8 by hand; block_reduce max-reduces only the last slot
    double vm[1] = {v[8]};
    v[8] = 0.0;
    block_reduce<kBulkVals, true>(v, sh);
    __syncthreads();
    double t = vm[0];
    for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_down_sync(0xffffffffu, t, o));
    __shared__ double shm[32];
    if ((threadIdx.x & 31) == 0) shm[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) t = fmax(t, shm[w]);
        for (int k = 0; k < kBulkVals; k++) partial[(size_t)blockIdx.x * (kBulkVals + 1) + k] = v[k];
        partial[(size_t)blockIdx.x * (kBulkVals + 1) + kBulkVals] = t;
    }
}

__global__ void bulk_finish_kernel(const double *__restrict__ partial, int n, Lattice L, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    CompSum cs[8];
    double gmax = 0.0, umax = 0.0;
    for (int i = 0; i < n; i++) {
        const double *p = partial + (size_t)i * (kBulkVals + 1);
        for (int k = 0; k < 8; k++) cs[k].add(p[k]);
        gmax = fmax(gmax, p[9]);
        umax = fmax(umax, p[10]);
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
    out[6] = gmax;
    out[7] = sqrt(s[6] / (3.0 * V));
    out[8] = umax;
    out[9] = sqrt(s[7] / (3.0 * V));
}

// ------------------------------------------------------ Gauss restoration --
// GaussLawRestoration (GAUSSLAWFIXING/GaussRestore.cpp:13-168).  The violation
// G^a(x) = sum_mu E_mu(x) - (U^+ E U)_mu(x - mu) per site into G, with the sum of
// squares and the signed maximum (starting from 0, as :46-49) per block.
__global__ void __launch_bounds__(kReduceThreads) gauss_violation_kernel(const double *__restrict__ U,
                                                                         const double *__restrict__ E, Lattice L,
                                                                         double *__restrict__ G, double *partial) {
    __shared__ double sh[32 * 2];
    double v[2] = {0.0, 0.0};
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.V; s += gridDim.x * blockDim.x) {
        int x, y, z;
        site_coords(L, s, x, y, z);
        double g[3] = {0.0, 0.0, 0.0};
        for (int mu = 0; mu < 3; mu++) {
            int c[3] = {x, y, z};
            c[mu] -= 1;
            const int sm = site_index(L, c[0], c[1], c[2]);
            adj3 R = adjoint(qdag(load_link(U, sm, mu)));
            for (int a = 0; a < 3; a++) {
                double t = E[a + 3 * (mu + 3 * s)];
                for (int b = 0; b < 3; b++) t -= R.r[a][b] * E[b + 3 * (mu + 3 * sm)];
                g[a] += t;
            }
        }
        for (int a = 0; a < 3; a++) {
            G[a + 3 * s] = g[a];
            v[0] += g[a] * g[a];
            v[1] = fmax(v[1], g[a]);
        }
    }
    block_reduce<2, true>(v, sh);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = v[0];
        partial[2 * blockIdx.x + 1] = v[1];
    }
}

// E_mu(x) -= gamma (G(x) - U_mu(x) G(x + mu) U_mu(x)^+)   (GaussRestore.cpp:72-118)
__global__ void gauss_update_kernel(const double *__restrict__ U, const double *__restrict__ G, double *__restrict__ E,
                                    Lattice L, double gamma) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * L.V) return;
    const int s = t / 3, mu = t % 3;
    int x, y, z;
    site_coords(L, s, x, y, z);
    int c[3] = {x, y, z};
    c[mu] += 1;
    const int sp = site_index(L, c[0], c[1], c[2]);
    const adj3 R = adjoint(load_link(U, s, mu));
    for (int a = 0; a < 3; a++) {
        double up = 0.0;
        for (int b = 0; b < 3; b++) up += R.r[a][b] * G[b + 3 * sp];
        E[a + 3 * (mu + 3 * s)] -= gamma * (G[a + 3 * s] - up);
    }
}

size_t gauss_partial_doubles(const Lattice &L) { return (size_t)reduce_blocks(L.V) * 2; }

// out[0] = sum of G^2, out[1] = signed maximum.
void launch_gauss_violation(const double *U, const double *E, const Lattice &L, double *G, double *partial,
                            double *out, cudaStream_t stream) {
    const int nb = reduce_blocks(L.V);
    gauss_violation_kernel<<<nb, kReduceThreads, 0, stream>>>(U, E, L, G, partial);
    finish_kernel<2, true><<<1, 256, 0, stream>>>(partial, nb, out, 1.0);
}

void launch_gauss_update(const double *U, const double *G, double *E, const Lattice &L, double gamma,
                         cudaStream_t stream) {
    const int n = 3 * L.V;
    gauss_update_kernel<<<(n + 127) / 128, 128, 0, stream>>>(U, G, E, L, gamma);
}

size_t bulk_partial_doubles(const Lattice &L) { return (size_t)reduce_blocks(L.V) * (kBulkVals + 1); }

void launch_bulk(const double *U, const double *E, const Lattice &L, double *partial, double *out, cudaStream_t stream) {
    const int nb = reduce_blocks(L.V);
    bulk_kernel<<<nb, kReduceThreads, 0, stream>>>(U, E, L, partial);
    bulk_finish_kernel<<<1, 32, 0, stream>>>(partial, nb, L, out);
}

// ------------------------------------------------------------- cooling ----
// Blocking (LATTICE/GaugeLinks.cpp:126-153): the link of the lattice with
// twice the spacing is the product of the two fine links it spans,
// U'_mu(x) = U_mu(2x) U_mu(2x + mu).  Lout = L halved in every direction.
template <int NC>
__global__ void block_links_kernel(const double *__restrict__ U, Lattice L, double *__restrict__ Uout, Lattice Lout) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 3 * Lout.V) return;
    const int site = l / 3, mu = l % 3;
    int x, y, z;
    site_coords(Lout, site, x, y, z);
    int c[3] = {2 * x, 2 * y, 2 * z};
    const int s0 = site_index(L, c[0], c[1], c[2]);
    c[mu] += 1;
    const int s1 = site_index(L, c[0], c[1], c[2]);
    if (NC == 2) store_link(Uout, site, mu, qmul(load_link(U, s0, mu), load_link(U, s1, mu)));
    else store_su3(Uout, site, mu, m3_mul(load_su3(U, s0, mu), load_su3(U, s1, mu)));
}

void launch_block_links(const double *U, const Lattice &L, double *Uout, const Lattice &Lout, int nc,
                        cudaStream_t stream) {
    const int n = 3 * Lout.V;
    if (nc == 3) block_links_kernel<3><<<(n + 127) / 128, 128, 0, stream>>>(U, L, Uout, Lout);
    else block_links_kernel<2><<<(n + 127) / 128, 128, 0, stream>>>(U, L, Uout, Lout);
}

// The structure constants f(a, b, c) exactly as the vacuum estimator reads
// them.  Two colours: (a-b)(a-c)(c-b)/2, the Levi-Civita symbol on 0..2
// (SU2/AlgebraOperations.cpp:21-25).  Three colours: the reference's table
// (SU3/AlgebraOperations.cpp:28-76) is written for generator labels 1..8 and
// the estimator calls it with components 0..7, so the entries it reaches are
// those whose three labels are all at most 7 -- f123 = 1, f147 = f246 = f257 =
// f345 = 1/2, f156 = f367 = -1/2 -- applied to components with those numbers;
// the sign is that of (a-b)(a-c)(c-b).
__device__ __forceinline__ double vacuum_f(int nc, int a, int b, int c) {
    const int prod = (a - b) * (a - c) * (c - b);
    if (prod == 0) return 0.0;
    const double sgn = prod > 0 ? 1.0 : -1.0;
    if (nc == 2) return 0.5 * prod;
    const int lo = min(a, min(b, c)), hi = max(a, max(b, c)), mid = a + b + c - lo - hi;
    const int key = 100 * lo + 10 * mid + hi;
    switch (key) {
        case 123: return sgn;
        case 147: case 246: case 257: case 345: return 0.5 * sgn;
        case 156: case 367: return -0.5 * sgn;
        default: return 0.0;
    }
}

// 2 Re tr(i t^a U) of one link: ReTrIGenU(2, U) (SU2/GroupOperations.cpp:86-92,
// SU3/GroupOperations.cpp:120-130).
template <int NC>
__device__ __forceinline__ void link_algebra(const double *__restrict__ U, int site, int mu, double *A) {
    if (NC == 2) {
        const quat q = load_link(U, site, mu);
        A[0] = -2.0 * q.v0;
        A[1] = -2.0 * q.v1;
        A[2] = -2.0 * q.v2;
    } else {
        su3_retr_ita(load_su3(U, site, mu), A);
        for (int a = 0; a < 8; a++) A[a] *= 2.0;
    }
}

// ChernSimonsNumber::VacuumEstimator::NCS (TOPOLOGY/VacuumEstimator.cpp:7-85):
// with A_mu(x) = (ReTrIGenU(2, U_mu(x)) + ReTrIGenU(2, U_mu(x - mu))) / 2,
// sum over sites of f(a,b,c) A_x^a A_y^b A_z^c / (16 pi^2).
template <int NC>
__global__ void __launch_bounds__(kReduceThreads) vacuum_ncs_kernel(const double *__restrict__ U, Lattice L,
                                                                     double *partial) {
    constexpr int NA = NC * NC - 1;
    __shared__ double sh[32];
    CompSum sum;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.V; s += gridDim.x * blockDim.x) {
        int x, y, z;
        site_coords(L, s, x, y, z);
        double A[3][NA];
        for (int mu = 0; mu < 3; mu++) {
            double ap[NA], am[NA];
            int c[3] = {x, y, z};
            c[mu] -= 1;
            link_algebra<NC>(U, s, mu, ap);
            link_algebra<NC>(U, site_index(L, c[0], c[1], c[2]), mu, am);
            for (int a = 0; a < NA; a++) A[mu][a] = 0.5 * (ap[a] + am[a]);
        }
        double local = 0.0;
        for (int a = 0; a < NA; a++)
            for (int b = 0; b < NA; b++)
                for (int c = 0; c < NA; c++) {
                    const double f = vacuum_f(NC, a, b, c);
                    if (f != 0.0) local += f * A[0][a] * A[1][b] * A[2][c];
                }
        sum.add(local);
    }
    double v[1] = {sum.value()};
    block_reduce<1, false>(v, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

void launch_vacuum_ncs(const double *U, const Lattice &L, int nc, double *partial, double *out, cudaStream_t stream) {
    const int nb = reduce_blocks(L.V);
    if (nc == 3) vacuum_ncs_kernel<3><<<nb, kReduceThreads, 0, stream>>>(U, L, partial);
    else vacuum_ncs_kernel<2><<<nb, kReduceThreads, 0, stream>>>(U, L, partial);
    finish_kernel<1, false><<<1, kReduceThreads, 0, stream>>>(partial, nb, out, 1.0 / (16.0 * M_PI * M_PI));
}

}  // namespace ovl
