// Extreme eigenvalues of h_W^2 for the overlap operator's spectral bounds:
// OverlapOperations::RitzSolver with one eigenvalue
// (FERMIONS/OVERLAP/OPERATOR/RitzSolver.cpp:91-292), called twice per bound
// computation by Dynamics::Fermions::ComputeRitzEigenvalues
// (FERMIONS/OVERLAP/OverlapUpdate.cpp:61-97): sign = +1 gives the smallest
// eigenvalue, sign = -1 the largest (negated).  The iteration is a
// conjugate-gradient minimisation of the Rayleigh quotient of sign * A,
// A = -D^2 = h_W^2: per step a rotation of x in the plane of (x, p) chosen from
// 2x2 Rayleigh-Ritz, and a new search direction p = g + beta (p - x <x, p>).
//
// Both problems run together, one per blockIdx.y, on vectors in a compact
// layout [problem][site][colour * 4 + spin] (double2): one thread per site;
// NCOMP = 4 Nc components per site (two or three colours).
// Each step is a fixed sequence of kernels; every dot product is reduced per
// CTA into a partial buffer and the next kernel adds the partials in a fixed
// order (every CTA computes bit-identical scalars, so all take the same
// decisions).  Scalars that outlive a kernel sit in RitzScalars; each field is
// written (by CTA 0) in exactly one kernel of a step and read only by later
// kernels.  The partial buffers alternate between two slots so that no kernel
// reads the slot it writes.  A problem that has stopped skips all work.
#include <algorithm>
#include <cmath>

#include "ovl_internal.h"
#include "ovl_stencil.cuh"
#include "ovl_su3.cuh"

namespace ovl {

constexpr int kRitzThreads = 128;
constexpr int kRitzParts = 4;  // doubles per CTA partial

struct RitzScalars {
    double xy_re, xy_im;    // Rayleigh quotient <x, y> (restart, residual)
    double oxy_re, oxy_im;  // its value before the rotation (rotate)
    double pnorm;           // |p| before normalisation (normp)
    double gnormim;         // |g|^2 of the previous step (normp)
    double gnorm;           // |g|^2 of this step (direction)
    int ittot;              // steps taken (rotate)
    int done;               // stopped (direction; host at start)
};

struct RitzArgs {
    int nblocks;            // CTAs per problem
    double sign[2];         // problem 0: +1 (lambda_min), problem 1: -1 (-lambda_max)
    double delitr;          // NormRatio
    int max_iter;           // MaximumIterations
};

__device__ __forceinline__ double2 ld2(const double2 *p) { return __ldg(p); }

template <typename T>
__device__ __forceinline__ void load_compact(const double2 *__restrict__ v, int site, Spinor<T> &s) {
    const double2 *p = v + (size_t)site * kComp;
#pragma unroll
    for (int c = 0; c < kColours; c++)
#pragma unroll
        for (int a = 0; a < kSpin; a++) {
            const double2 t = ld2(p + c * kSpin + a);
            s.c[c][a] = mk<T>(t.x, t.y);
        }
}

// Block-wide sum of up to kRitzParts values in a fixed order; thread 0 writes
// them to part[k].
__device__ __forceinline__ void block_partials(double (&v)[kRitzParts], int nv, double *part) {
    __shared__ double sh[kRitzThreads / 32][kRitzParts];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < nv; k++) {
        double t = v[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) sh[warp][k] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < nv; k++) {
            double t = 0.0;
            for (int w = 0; w < kRitzThreads / 32; w++) t += sh[w][k];
            part[k] = t;
        }
    }
}

// Sums the nblocks partials of a problem (k = 0..nv-1) in a fixed order; every
// thread of the CTA gets the same values.
__device__ __forceinline__ void reduce_partials(const double *__restrict__ part, int nblocks, int nv,
                                                double (&out)[kRitzParts]) {
    __shared__ double sh[kRitzParts];
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        for (int k = 0; k < nv; k++) {
            double t = 0.0;
            for (int b = lane; b < nblocks; b += 32) t += part[(size_t)b * kRitzParts + k];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) sh[k] = t;
        }
    }
    __syncthreads();
    for (int k = 0; k < nv; k++) out[k] = sh[k];
    __syncthreads();
}

// Whether a problem has stopped, read once per CTA (thread 0) and shared, so
// that the whole CTA takes the same branch even while CTA 0 of the direction
// kernel sets the flag.
__device__ __forceinline__ bool ritz_stopped(const RitzScalars *st, int prob) {
    __shared__ int flag;
    if (threadIdx.x == 0) flag = *reinterpret_cast<const volatile int *>(&st[prob].done);
    __syncthreads();
    return flag != 0;
}

__device__ __forceinline__ double *part_of(double *base, int slot, int prob, int nblocks) {
    return base + ((size_t)slot * 2 + prob) * nblocks * kRitzParts;
}

// <a, b> = sum conj(a) b over the NCOMP components of one site
template <int NCOMP>
__device__ __forceinline__ void site_dot(const double2 *a, const double2 *b, double &re, double &im) {
#pragma unroll
    for (int k = 0; k < NCOMP; k++) {
        const double2 u = a[k], w = b[k];
        re += u.x * w.x + u.y * w.y;
        im += u.x * w.y - u.y * w.x;
    }
}

// x = start for both problems; partial |x|^2 -> slot 0
template <int NCOMP>
__global__ void __launch_bounds__(kRitzThreads)
    ritz_start_kernel(const double2 *__restrict__ start, double2 *x, int V, RitzArgs a, double *part) {
    const int prob = blockIdx.y, site = blockIdx.x * kRitzThreads + threadIdx.x;
    double v[kRitzParts] = {0.0, 0.0, 0.0, 0.0};
    if (site < V) {
        double2 *xs = x + ((size_t)prob * V + site) * NCOMP;
#pragma unroll
        for (int k = 0; k < NCOMP; k++) {
            const double2 s = start[(size_t)site * NCOMP + k];
            xs[k] = s;
            v[0] += s.x * s.x + s.y * s.y;
        }
    }
    block_partials(v, 1, part_of(part, 0, prob, a.nblocks) + (size_t)blockIdx.x * kRitzParts);
}

// x /= |x| (slot 0)
template <int NCOMP>
__global__ void __launch_bounds__(kRitzThreads)
    ritz_scale_x_kernel(double2 *x, int V, RitzArgs a, double *part) {
    const int prob = blockIdx.y, site = blockIdx.x * kRitzThreads + threadIdx.x;
    double r[kRitzParts];
    reduce_partials(part_of(part, 0, prob, a.nblocks), a.nblocks, 1, r);
    const double s = 1.0 / sqrt(r[0]);
    if (site < V) {
        double2 *xs = x + ((size_t)prob * V + site) * NCOMP;
#pragma unroll
        for (int k = 0; k < NCOMP; k++) xs[k] = make_double2(xs[k].x * s, xs[k].y * s);
    }
}

// SECOND = false: dst = D src.  SECOND = true: dst = -sign D src (= sign A v
// when src = D v) and partials <da, dst> (k = 0, 1) and <db, dst> (k = 2, 3,
// when db is set) -> slot 0.  NC colours: the two-colour stencil of
// ovl_stencil.cuh or the three-colour one of ovl_su3.cuh on the compact layout.
template <int NC, bool U1, bool SECOND, class LK>
__global__ void __launch_bounds__(kRitzThreads)
    ritz_apply_kernel(LK lk, const double2 *__restrict__ src, double2 *__restrict__ dst,
                      const double2 *__restrict__ da, const double2 *__restrict__ db, Lattice L, double amass,
                      const RitzScalars *__restrict__ st, RitzArgs a, double *part) {
    constexpr int NCOMP = 4 * NC;
    const int prob = blockIdx.y, site = blockIdx.x * kRitzThreads + threadIdx.x;
    if (ritz_stopped(st, prob)) return;
    const int V = L.V;
    const size_t off = (size_t)prob * V;
    double v[kRitzParts] = {0.0, 0.0, 0.0, 0.0};
    if (site < V) {
        const double2 *s = src + off * NCOMP;
        const Nbrs n = neighbours(L, site);
        const double scale = SECOND ? -a.sign[prob] : 1.0;
        double2 o[NCOMP];
        if constexpr (NC == 2) {
            Spinor<double> acc, f;
            load_compact(s, site, f);
#pragma unroll
            for (int c = 0; c < kColours; c++)
#pragma unroll
                for (int s2 = 0; s2 < kSpin; s2++) acc.c[c][s2] = amass * f.c[c][s2];
            load_compact(s, n.xp, f);
            hop<double, 0, true>(acc, f, lk.template get<double>(site, 0));
            load_compact(s, n.xm, f);
            hop<double, 0, false>(acc, f, lk.template get<double>(n.xm, 0));
            load_compact(s, n.yp, f);
            hop<double, 1, true>(acc, f, lk.template get<double>(site, 1));
            load_compact(s, n.ym, f);
            hop<double, 1, false>(acc, f, lk.template get<double>(n.ym, 1));
            load_compact(s, n.zp, f);
            hop<double, 2, true>(acc, f, lk.template get<double>(site, 2));
            load_compact(s, n.zm, f);
            hop<double, 2, false>(acc, f, lk.template get<double>(n.zm, 2));
#pragma unroll
            for (int c = 0; c < kColours; c++)
#pragma unroll
                for (int s2 = 0; s2 < kSpin; s2++) {
                    const cpx<double> r = finish_component(acc.c[c][s2], s2);
                    o[c * kSpin + s2] = make_double2(scale * r.re, scale * r.im);
                }
        } else {
            const cpx<double> *f = reinterpret_cast<const cpx<double> *>(s);
            Spinor3<double> acc;
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int s2 = 0; s2 < kSpin; s2++) acc.c[c][s2] = amass * ld(f + (size_t)site * NCOMP + c * kSpin + s2);
            hop3<double, 0, true, false, 1>(acc, f + (size_t)n.xp * NCOMP, lk.template get<double>(site, 0));
            hop3<double, 0, false, false, 1>(acc, f + (size_t)n.xm * NCOMP, lk.template get<double>(n.xm, 0));
            hop3<double, 1, true, false, 1>(acc, f + (size_t)n.yp * NCOMP, lk.template get<double>(site, 1));
            hop3<double, 1, false, false, 1>(acc, f + (size_t)n.ym * NCOMP, lk.template get<double>(n.ym, 1));
            hop3<double, 2, true, false, 1>(acc, f + (size_t)n.zp * NCOMP, lk.template get<double>(site, 2));
            hop3<double, 2, false, false, 1>(acc, f + (size_t)n.zm * NCOMP, lk.template get<double>(n.zm, 2));
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int s2 = 0; s2 < kSpin; s2++) {
                    const cpx<double> r = finish_component(acc.c[c][s2], s2);
                    o[c * kSpin + s2] = make_double2(scale * r.re, scale * r.im);
                }
        }
        double2 *d = dst + (off + site) * NCOMP;
#pragma unroll
        for (int k = 0; k < NCOMP; k++) d[k] = o[k];
        if (SECOND) {
            site_dot<NCOMP>(da + (off + site) * NCOMP, o, v[0], v[1]);
            if (db) site_dot<NCOMP>(db + (off + site) * NCOMP, o, v[2], v[3]);
        }
    }
    if (SECOND) block_partials(v, 4, part_of(part, 0, prob, a.nblocks) + (size_t)blockIdx.x * kRitzParts);
}

// Restart (RitzSolver.cpp:138-166): xy = <x, y>; g = p = y - xy x; |g|^2 -> slot 1.
template <int NCOMP>
__global__ void __launch_bounds__(kRitzThreads)
    ritz_restart_kernel(const double2 *__restrict__ x, const double2 *__restrict__ y, double2 *__restrict__ g,
                        double2 *__restrict__ praw, int V, RitzScalars *st, RitzArgs a, double *part) {
    const int prob = blockIdx.y, site = blockIdx.x * kRitzThreads + threadIdx.x;
    if (ritz_stopped(st, prob)) return;
    double r[kRitzParts];
    reduce_partials(part_of(part, 0, prob, a.nblocks), a.nblocks, 2, r);
    const double xr = r[0], xi = r[1];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st[prob].xy_re = xr;
        st[prob].xy_im = xi;
    }
    double v[kRitzParts] = {0.0, 0.0, 0.0, 0.0};
    if (site < V) {
        const size_t o = ((size_t)prob * V + site) * NCOMP;
#pragma unroll
        for (int k = 0; k < NCOMP; k++) {
            const double2 xv = x[o + k], yv = y[o + k];
            const double2 gv = make_double2(yv.x - (xr * xv.x - xi * xv.y), yv.y - (xr * xv.y + xi * xv.x));
            g[o + k] = gv;
            praw[o + k] = gv;
            v[0] += gv.x * gv.x + gv.y * gv.y;
        }
    }
    block_partials(v, 1, part_of(part, 1, prob, a.nblocks) + (size_t)blockIdx.x * kRitzParts);
}

// p = praw / |praw| (slot 1); pnorm; gnormim = |praw|^2 on a restart (p = g
// there), else the gnorm of this step.
template <int NCOMP>
__global__ void __launch_bounds__(kRitzThreads)
    ritz_normp_kernel(const double2 *__restrict__ praw, double2 *__restrict__ p, int V, int restart, RitzScalars *st,
                      RitzArgs a, const double *part) {
    const int prob = blockIdx.y, site = blockIdx.x * kRitzThreads + threadIdx.x;
    if (ritz_stopped(st, prob)) return;
    double r[kRitzParts];
    reduce_partials(part_of(const_cast<double *>(part), 1, prob, a.nblocks), a.nblocks, 1, r);
    const double pn = sqrt(r[0]);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st[prob].pnorm = pn;
        st[prob].gnormim = restart ? r[0] : st[prob].gnorm;
    }
    if (site < V) {
        const size_t o = ((size_t)prob * V + site) * NCOMP;
#pragma unroll
        for (int k = 0; k < NCOMP; k++) p[o + k] = make_double2(praw[o + k].x / pn, praw[o + k].y / pn);
    }
}

// The rotation of x in the (x, p) plane (RitzSolver.cpp:176-222), from slot 0:
// pz = Re <p, z>, xz = Re <x, z>.  Then <x, x>, <x, y> -> slot 1.
template <int NCOMP>
__global__ void __launch_bounds__(kRitzThreads)
    ritz_rotate_kernel(double2 *x, double2 *y, const double2 *__restrict__ p, const double2 *__restrict__ z, int V,
                       RitzScalars *st, RitzArgs a, double *part) {
    const int prob = blockIdx.y, site = blockIdx.x * kRitzThreads + threadIdx.x;
    if (ritz_stopped(st, prob)) return;
    double r[kRitzParts];
    reduce_partials(part_of(part, 0, prob, a.nblocks), a.nblocks, 4, r);
    const double pz = r[0], ccc = r[2];
    const double xy_re = st[prob].xy_re, xy_im = st[prob].xy_im;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st[prob].oxy_re = xy_re;
        st[prob].oxy_im = xy_im;
        st[prob].ittot += 1;
    }
    const double amb = xy_re - pz;  // Re(xy - Re <p, z>)
    const double cox = 2.0 * ccc / amb;
    const double sig1 = -copysign(1.0, amb);
    const double sig2 = copysign(1.0, cox) * sig1;
    const double c2 = cox * cox;
    double ct, sn;
    if (c2 <= 1.0e-3) {
        // the reference's series for the rotation, constants as there (:197-200)
        const double sqp = 1.0 - 0.125 * c2 + 0.0859375 * c2 * c2 - 0.0673828125 * c2 * c2 * c2 +
                           0.0562439 * c2 * c2 * c2 * c2 + 0.0487 * c2 * c2 * c2 * c2 * c2;
        const double sqm = 0.5 * sig1 * sig2 * cox *
                           (1.0 - 0.375 * c2 + 0.2421875 * c2 * c2 - 0.182617875 * c2 * c2 * c2 +
                            0.1482849 * c2 * c2 * c2 * c2 - 0.12575 * c2 * c2 * c2 * c2 * c2 +
                            0.1097 * c2 * c2 * c2 * c2 * c2 * c2);
        if (sig1 < 0.0) {
            ct = sqm;
            sn = sig2 * sqp;
        } else {
            ct = sqp;
            sn = sig2 * sqm;
        }
    } else {
        const double sox = sig1 / sqrt(1.0 + c2);
        ct = sqrt((1.0 + sox) * 0.5);
        sn = sqrt((1.0 - sox) * 0.5) * sig2;
    }
    double v[kRitzParts] = {0.0, 0.0, 0.0, 0.0};
    if (site < V) {
        const size_t o = ((size_t)prob * V + site) * NCOMP;
        double2 xn[NCOMP], yn[NCOMP];
#pragma unroll
        for (int k = 0; k < NCOMP; k++) {
            const double2 xv = x[o + k], pv = p[o + k], yv = y[o + k], zv = z[o + k];
            xn[k] = make_double2(xv.x * ct + pv.x * sn, xv.y * ct + pv.y * sn);
            yn[k] = make_double2(yv.x * ct + zv.x * sn, yv.y * ct + zv.y * sn);
            x[o + k] = xn[k];
            y[o + k] = yn[k];
        }
        double im0 = 0.0;
        site_dot<NCOMP>(xn, xn, v[0], im0);
        site_dot<NCOMP>(xn, yn, v[1], v[2]);
    }
    block_partials(v, 3, part_of(part, 1, prob, a.nblocks) + (size_t)blockIdx.x * kRitzParts);
}

// x normalised, xy = <x, y> / |x|, g = y - xy x (RitzSolver.cpp:224-243), from
// slot 1.  Then |g|^2, <x, p> -> slot 0.
template <int NCOMP>
__global__ void __launch_bounds__(kRitzThreads)
    ritz_residual_kernel(double2 *x, const double2 *__restrict__ y, double2 *__restrict__ g,
                         const double2 *__restrict__ p, int V, RitzScalars *st, RitzArgs a, double *part) {
    const int prob = blockIdx.y, site = blockIdx.x * kRitzThreads + threadIdx.x;
    if (ritz_stopped(st, prob)) return;
    double r[kRitzParts];
    reduce_partials(part_of(part, 1, prob, a.nblocks), a.nblocks, 3, r);
    const double xnorm = 1.0 / sqrt(r[0]);
    const double xr = r[1] * xnorm, xi = r[2] * xnorm;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st[prob].xy_re = xr;
        st[prob].xy_im = xi;
    }
    double v[kRitzParts] = {0.0, 0.0, 0.0, 0.0};
    if (site < V) {
        const size_t o = ((size_t)prob * V + site) * NCOMP;
        double2 xn[NCOMP], gn[NCOMP];
#pragma unroll
        for (int k = 0; k < NCOMP; k++) {
            const double2 xv = x[o + k], yv = y[o + k];
            xn[k] = make_double2(xv.x * xnorm, xv.y * xnorm);
            gn[k] = make_double2(yv.x - (xr * xn[k].x - xi * xn[k].y), yv.y - (xr * xn[k].y + xi * xn[k].x));
            x[o + k] = xn[k];
            g[o + k] = gn[k];
        }
        double im0 = 0.0;
        site_dot<NCOMP>(gn, gn, v[0], im0);
        site_dot<NCOMP>(xn, p + o, v[1], v[2]);
    }
    block_partials(v, 3, part_of(part, 0, prob, a.nblocks) + (size_t)blockIdx.x * kRitzParts);
}

// Stopping tests and the new search direction (RitzSolver.cpp:245-284), from
// slot 0: gnorm = |g|^2, xp = <x, p>.  praw = g + beta (p - x xp); |praw|^2 -> slot 1.
template <int NCOMP>
__global__ void __launch_bounds__(kRitzThreads)
    ritz_direction_kernel(const double2 *__restrict__ x, const double2 *__restrict__ g, const double2 *__restrict__ p,
                          double2 *__restrict__ praw, int V, RitzScalars *st, RitzArgs a, double *part) {
    const int prob = blockIdx.y, site = blockIdx.x * kRitzThreads + threadIdx.x;
    if (ritz_stopped(st, prob)) return;
    double r[kRitzParts];
    reduce_partials(part_of(part, 0, prob, a.nblocks), a.nblocks, 3, r);
    const double gnorm = r[0], xpr = r[1], xpi = r[2];
    // fields not written by this kernel (gnorm and done are: CTA 0 below)
    const double xy_re = st[prob].xy_re, oxy_re = st[prob].oxy_re;
    const double gnormim = st[prob].gnormim, pnorm = st[prob].pnorm;
    const int ittot = st[prob].ittot;
    bool stop = xy_re > oxy_re || gnorm < a.delitr * a.sign[prob] * xy_re;
    const double beta = gnorm / gnormim * pnorm;
    double v[kRitzParts] = {0.0, 0.0, 0.0, 0.0};
    if (!stop && site < V) {
        const size_t o = ((size_t)prob * V + site) * NCOMP;
#pragma unroll
        for (int k = 0; k < NCOMP; k++) {
            const double2 xv = x[o + k], gv = g[o + k], pv = p[o + k];
            const double2 xxp = make_double2(xv.x * xpr - xv.y * xpi, xv.x * xpi + xv.y * xpr);
            const double2 pn = make_double2(gv.x + beta * (pv.x - xxp.x), gv.y + beta * (pv.y - xxp.y));
            praw[o + k] = pn;
            v[0] += pn.x * pn.x + pn.y * pn.y;
        }
    }
    if (!stop && ittot >= a.max_iter) stop = true;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st[prob].gnorm = gnorm;
        if (stop) st[prob].done = 1;
    }
    block_partials(v, 1, part_of(part, 1, prob, a.nblocks) + (size_t)blockIdx.x * kRitzParts);
}

// Start vector with the reference's distribution (Re, Im uniform in [0, 1),
// OverlapUpdate.cpp:69-84) from a counter-based generator: SplitMix64
// (Steele, Lea and Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014) of (seed, call, index); the top 53 bits give the uniform.
__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void ritz_random_start_kernel(double2 *start, size_t n, uint64_t seed, uint64_t call) {
    const uint64_t key = splitmix64(seed ^ splitmix64(call));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t a = splitmix64(key + 2 * i), b = splitmix64(key + 2 * i + 1);
        start[i] = make_double2((double)(a >> 11) * 0x1.0p-53, (double)(b >> 11) * 0x1.0p-53);
    }
}

// ---------------------------------------------------------------- host side --

// The iteration between two reads of the stop flags (kRitzPoll steps, with or
// without the restart that opens a cycle of nrestart steps) captured once as
// CUDA graphs and replayed; recaptured when an argument they bake in changes.
constexpr int kRitzPoll = 25;

struct RitzGraphs {
    cudaGraphExec_t restart = nullptr, plain = nullptr;
    const double *U = nullptr, *u1 = nullptr;
    int N[3] = {0, 0, 0};
    double amass = 0.0, delitr = 0.0;
    int max_iter = 0;
    bool failed = false;  // capture not possible on this stream: step the loop instead
    void release() {
        if (restart) cudaGraphExecDestroy(restart);
        if (plain) cudaGraphExecDestroy(plain);
        restart = plain = nullptr;
    }
};

struct RitzWork {
    double2 *x = nullptr, *y = nullptr, *z = nullptr, *t = nullptr, *p = nullptr, *praw = nullptr, *g = nullptr;
    double2 *start = nullptr;
    double *part = nullptr;
    RitzScalars *st = nullptr;
    RitzScalars *host = nullptr;  // pinned
    int V = 0;
    int nc = 2;  // colours: vectors of 4 nc components per site
    RitzGraphs graphs;
};

size_t ritz_work_bytes(int V, int nc) {
    const int nblocks = (V + kRitzThreads - 1) / kRitzThreads;
    return sizeof(double2) * 4 * nc * (size_t)V * (7 * 2 + 1) + sizeof(double) * 4 * nblocks * kRitzParts +
           2 * sizeof(RitzScalars);
}

void *ritz_create(int V, int nc) {
    RitzWork *w = new RitzWork;
    w->V = V;
    w->nc = nc;
    const size_t vec = sizeof(double2) * 4 * nc * (size_t)V * 2;
    const int nblocks = (V + kRitzThreads - 1) / kRitzThreads;
    double2 **bufs[] = {&w->x, &w->y, &w->z, &w->t, &w->p, &w->praw, &w->g};
    bool ok = true;
    for (double2 **b : bufs) ok = ok && cudaMalloc(b, vec) == cudaSuccess;
    ok = ok && cudaMalloc(&w->start, vec / 2) == cudaSuccess;
    ok = ok && cudaMalloc(&w->part, sizeof(double) * 4 * nblocks * kRitzParts) == cudaSuccess;
    ok = ok && cudaMalloc(&w->st, 2 * sizeof(RitzScalars)) == cudaSuccess;
    ok = ok && cudaMallocHost(&w->host, 2 * sizeof(RitzScalars)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        ritz_destroy(w);
        return nullptr;
    }
    return w;
}

void ritz_destroy(void *work) {
    RitzWork *w = static_cast<RitzWork *>(work);
    if (!w) return;
    void *bufs[] = {w->x, w->y, w->z, w->t, w->p, w->praw, w->g, w->start, w->part, w->st};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (w->host) cudaFreeHost(w->host);
    w->graphs.release();
    delete w;
}

double2 *ritz_start_buffer(void *work) { return static_cast<RitzWork *>(work)->start; }

void launch_ritz_random_start(void *work, uint64_t seed, uint64_t call, cudaStream_t stream) {
    RitzWork &w = *static_cast<RitzWork *>(work);
    const size_t n = (size_t)w.V * 4 * w.nc;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 1024);
    ritz_random_start_kernel<<<blocks, 256, 0, stream>>>(w.start, n, seed, call);
}

template <int NC, bool U1>
static void launch_apply(const RitzWork &w, const double *U, const double *u1, const Lattice &L, double amass,
                         const double2 *src, double2 *dst, const double2 *da, const double2 *db, bool second,
                         const RitzArgs &a, dim3 grid, cudaStream_t stream) {
    if constexpr (NC == 2) {
        LinksF64<U1> lk{U, reinterpret_cast<const double2 *>(u1), L.N0 * L.N1};
        if (second)
            ritz_apply_kernel<2, U1, true><<<grid, kRitzThreads, 0, stream>>>(lk, src, dst, da, db, L, amass, w.st, a,
                                                                             w.part);
        else
            ritz_apply_kernel<2, U1, false><<<grid, kRitzThreads, 0, stream>>>(lk, src, dst, da, db, L, amass, w.st, a,
                                                                              w.part);
    } else {
        Links3<false, U1> lk{U, u1, L.N0 * L.N1};
        if (second)
            ritz_apply_kernel<3, U1, true><<<grid, kRitzThreads, 0, stream>>>(lk, src, dst, da, db, L, amass, w.st, a,
                                                                             w.part);
        else
            ritz_apply_kernel<3, U1, false><<<grid, kRitzThreads, 0, stream>>>(lk, src, dst, da, db, L, amass, w.st, a,
                                                                              w.part);
    }
}

template <int NC>
static cudaError_t ritz_run_nc(RitzWork &w, const double *U, const double *u1, const Lattice &L, double amass,
                               int max_iter, int nrestart, double delitr, double out[2], int iters[2],
                               cudaStream_t stream, uint64_t *launches) {
    constexpr int NCOMP = 4 * NC;
    const int V = L.V;
    RitzArgs a;
    a.nblocks = (V + kRitzThreads - 1) / kRitzThreads;
    a.sign[0] = 1.0;
    a.sign[1] = -1.0;
    a.delitr = delitr;
    a.max_iter = max_iter;
    const dim3 grid(a.nblocks, 2);
    uint64_t nl = 0;
    cudaError_t e = cudaMemsetAsync(w.st, 0, 2 * sizeof(RitzScalars), stream);
    if (e != cudaSuccess) return e;
    auto apply = [&](const double2 *src, double2 *dst, const double2 *da, const double2 *db, bool second) {
        if (u1) launch_apply<NC, true>(w, U, u1, L, amass, src, dst, da, db, second, a, grid, stream);
        else launch_apply<NC, false>(w, U, u1, L, amass, src, dst, da, db, second, a, grid, stream);
        nl++;
    };
    ritz_start_kernel<NCOMP><<<grid, kRitzThreads, 0, stream>>>(w.start, w.x, V, a, w.part);
    ritz_scale_x_kernel<NCOMP><<<grid, kRitzThreads, 0, stream>>>(w.x, V, a, w.part);
    nl += 2;
    // restart: y = sign A x, xy, g = p = y - xy x
    auto restart_seq = [&]() {
        apply(w.x, w.t, nullptr, nullptr, false);
        apply(w.t, w.y, w.x, nullptr, true);
        ritz_restart_kernel<NCOMP><<<grid, kRitzThreads, 0, stream>>>(w.x, w.y, w.g, w.praw, V, w.st, a, w.part);
        ritz_normp_kernel<NCOMP><<<grid, kRitzThreads, 0, stream>>>(w.praw, w.p, V, 1, w.st, a, w.part);
        nl += 2;
    };
    auto step_seq = [&]() {
        apply(w.p, w.t, nullptr, nullptr, false);
        apply(w.t, w.z, w.p, w.x, true);
        ritz_rotate_kernel<NCOMP><<<grid, kRitzThreads, 0, stream>>>(w.x, w.y, w.p, w.z, V, w.st, a, w.part);
        ritz_residual_kernel<NCOMP><<<grid, kRitzThreads, 0, stream>>>(w.x, w.y, w.g, w.p, V, w.st, a, w.part);
        ritz_direction_kernel<NCOMP><<<grid, kRitzThreads, 0, stream>>>(w.x, w.g, w.p, w.praw, V, w.st, a, w.part);
        ritz_normp_kernel<NCOMP><<<grid, kRitzThreads, 0, stream>>>(w.praw, w.p, V, 0, w.st, a, w.part);
        nl += 4;
    };
    auto poll = [&](bool &finished, int step) -> cudaError_t {
        cudaError_t r;
        if ((r = cudaGetLastError()) != cudaSuccess) return r;
        if ((r = cudaMemcpyAsync(w.host, w.st, 2 * sizeof(RitzScalars), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess)
            return r;
        if ((r = cudaStreamSynchronize(stream)) != cudaSuccess) return r;
        finished = (w.host[0].done && w.host[1].done) || step >= max_iter;
        return cudaSuccess;
    };
    // The graphs replace the loop below when the restart cycle and the step
    // limit are whole numbers of poll intervals: the same kernels in the same
    // order, so the same results.
    RitzGraphs &gr = w.graphs;
    bool graphs = !gr.failed && nrestart % kRitzPoll == 0 && max_iter % kRitzPoll == 0;
    if (graphs && !(gr.restart && gr.U == U && gr.u1 == u1 && gr.N[0] == L.N0 && gr.N[1] == L.N1 && gr.N[2] == L.N2 &&
                    gr.amass == amass && gr.delitr == delitr && gr.max_iter == max_iter)) {
        gr.release();
        auto capture = [&](bool with_restart, cudaGraphExec_t &exec) {
            if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
            const uint64_t nl0 = nl;
            if (with_restart) restart_seq();
            for (int i = 0; i < kRitzPoll; i++) step_seq();
            nl = nl0;  // counted when replayed
            cudaGraph_t g = nullptr;
            if (cudaStreamEndCapture(stream, &g) != cudaSuccess || !g) return false;
            const bool ok = cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
            cudaGraphDestroy(g);
            return ok;
        };
        if (capture(true, gr.restart) && capture(false, gr.plain)) {
            gr.U = U;
            gr.u1 = u1;
            gr.N[0] = L.N0;
            gr.N[1] = L.N1;
            gr.N[2] = L.N2;
            gr.amass = amass;
            gr.delitr = delitr;
            gr.max_iter = max_iter;
        } else {
            cudaGetLastError();
            gr.release();
            gr.failed = true;
            graphs = false;
        }
    }
    int step = 0;
    bool finished = false;
    if (graphs) {
        // one graph per poll interval, the restart one opening each cycle
        while (!finished) {
            const bool restart = step % nrestart == 0;
            if ((e = cudaGraphLaunch(restart ? gr.restart : gr.plain, stream)) != cudaSuccess) return e;
            nl += (restart ? 4 : 0) + 6 * kRitzPoll;
            step += kRitzPoll;
            if ((e = poll(finished, step)) != cudaSuccess) return e;
        }
    } else {
        // Host loop: restarts every nrestart steps; the done flags are read back
        // every kRitzPoll steps (both problems step in lockstep until they stop).
        while (!finished) {
            restart_seq();
            for (int itt = 1; itt <= nrestart; itt++) {
                step_seq();
                step++;
                if (step % kRitzPoll == 0 || itt == nrestart || step >= max_iter) {
                    if ((e = poll(finished, step)) != cudaSuccess) return e;
                    if (finished) break;
                }
            }
        }
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(w.host, w.st, 2 * sizeof(RitzScalars), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    for (int k = 0; k < 2; k++) {
        out[k] = w.host[k].xy_re;
        if (iters) iters[k] = w.host[k].ittot;
    }
    if (launches) *launches += nl;
    return cudaSuccess;
}

// Runs both Ritz problems from the start vector already in the start buffer
// (compact [V][4 nc] double2; links of the work space's colour count).  out:
// {lambda_min, -lambda_max as returned by the sign = -1 problem}; iters: steps
// per problem.  Returns a CUDA error or cudaSuccess; *launches counts kernels.
cudaError_t ritz_run(void *work, const double *U, const double *u1, const Lattice &L, double amass, int max_iter,
                     int nrestart, double delitr, double out[2], int iters[2], cudaStream_t stream,
                     uint64_t *launches) {
    RitzWork &w = *static_cast<RitzWork *>(work);
    if (w.nc == 3)
        return ritz_run_nc<3>(w, U, u1, L, amass, max_iter, nrestart, delitr, out, iters, stream, launches);
    return ritz_run_nc<2>(w, U, u1, L, amass, max_iter, nrestart, delitr, out, iters, stream, launches);
}

}  // namespace ovl
