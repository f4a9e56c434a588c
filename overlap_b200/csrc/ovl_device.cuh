// Device building blocks shared by the overlap_b200 kernels: complex numbers,
// SU(2) links stored as quaternions, Dirac matrices as monomial matrices and
// the lattice / mode-block indexing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ovl {

// ------------------------------------------------------------------ layout --
// Modes live in blocks of kModeBlock modes.  Within a block the field is
// [site][component][mode-in-block], component = colour*4 + spin, so a warp
// reading one component of one site for its 32 modes touches one contiguous
// 32-element run (512 B in FP64, 256 B in FP32).
constexpr int kModeBlock = 32;
constexpr int kSpin = 4;
constexpr int kColours = 2;
constexpr int kComp = kColours * kSpin;  // complex components per mode and site

struct Lattice {
    int N0, N1, N2;
    int V;
};

__host__ __device__ inline size_t field_index(int V, int mb, int site, int comp, int lane) {
    return (((size_t)mb * V + site) * kComp + comp) * kModeBlock + lane;
}

__device__ inline void site_coords(const Lattice &L, int s, int &x, int &y, int &z) {
    x = s % L.N0;
    int yz = s / L.N0;
    y = yz % L.N1;
    z = yz / L.N1;
}

__device__ inline int site_index(const Lattice &L, int x, int y, int z) {
    x = (x % L.N0 + L.N0) % L.N0;
    y = (y % L.N1 + L.N1) % L.N1;
    z = (z % L.N2 + L.N2) % L.N2;
    return x + L.N0 * (y + L.N1 * z);
}

// ------------------------------------------------------ compensated sums --
// Neumaier's compensated summation (Z. angew. Math. Mech. 54, 1974): the
// running sum s and the accumulated rounding c, so that a long sum of FP64
// terms loses no more than a few units of the last place of the result.  The
// global sums of the axial charge, the energy and E.B accumulate in it.
struct CompSum {
    double s = 0.0, c = 0.0;
    __host__ __device__ void add(double x) {
        const double t = s + x;
        c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    __host__ __device__ double value() const { return s + c; }
};

// ----------------------------------------------------------------- complex --
// The GPU's global nanosecond timer (bounds for waits on other CTAs).
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// A load with acquire semantics at GPU scope (pairs with a fence + atomic release).
__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// *p += v with release semantics at GPU scope: the writes this thread has
// made or observed (through a CTA barrier, cumulativity) are visible to a
// thread that reads the count with ld_acquire.
__device__ __forceinline__ void red_release_add(int *p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounds of a wait on other CTAs: elapsed time, and a poll count as a second
// bound (>= 2 s with the 100 ns sleeps between polls).
constexpr long long kWaitNs = 1000000000LL;
constexpr long long kWaitPolls = 20000000;

// One thread waits until *counter >= target.  It gives up when the wait runs
// past either bound, or at once when *err is set (another CTA gave up); giving
// up sets *err.  Returns whether the count was reached.
__device__ __forceinline__ bool wait_count(const int *counter, int target, int *err) {
    long long polls = 0;
    const unsigned long long t0 = global_ns();
    while (ld_acquire(counter) < target) {
        if (++polls > kWaitPolls || (long long)(global_ns() - t0) > kWaitNs || *(volatile int *)err) {
            atomicExch(err, 1);
            return false;
        }
        __nanosleep(100);
    }
    return true;
}

// Phase j of 2n of a two-phase pipeline over n groups -> (group g, phase h) in
// the order (0,0), (1,0), (0,1), (2,0), (1,1), ..., (n-1,0), (n-2,1), (n-1,1):
// a group's second phase runs two phases after its first.
__device__ __forceinline__ void pipe_phase(int j, int n, int &g, int &h) {
    if (j == 2 * n - 1) { g = n - 1; h = 1; }
    else if (j == 0) { g = 0; h = 0; }
    else if (j & 1) { g = (j + 1) / 2; h = 0; }
    else { g = j / 2 - 1; h = 1; }
}

template <typename T> struct cpx { T re, im; };
template <typename T> struct vec2_of;
template <> struct vec2_of<double> { using type = double2; };
template <> struct vec2_of<float> { using type = float2; };

template <typename T> __device__ __forceinline__ cpx<T> mk(T re, T im) { return {re, im}; }
template <typename T> __device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> __device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T> __device__ __forceinline__ cpx<T> operator*(cpx<T> a, cpx<T> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T> __device__ __forceinline__ cpx<T> operator*(T s, cpx<T> a) { return {s * a.re, s * a.im}; }
template <typename T> __device__ __forceinline__ cpx<T> conj(cpx<T> a) { return {a.re, -a.im}; }
template <typename T> __device__ __forceinline__ cpx<T> times_i(cpx<T> a) { return {-a.im, a.re}; }
template <typename T> __device__ __forceinline__ cpx<T> times_mi(cpx<T> a) { return {a.im, -a.re}; }
// conj(a) * b
template <typename T> __device__ __forceinline__ cpx<T> cdot(cpx<T> a, cpx<T> b) {
    return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}

template <typename T> __device__ __forceinline__ cpx<T> ld(const cpx<T> *p) {
    using V2 = typename vec2_of<T>::type;
    V2 v = __ldg(reinterpret_cast<const V2 *>(p));
    return {v.x, v.y};
}
template <typename T> __device__ __forceinline__ void st(cpx<T> *p, cpx<T> a) {
    using V2 = typename vec2_of<T>::type;
    *reinterpret_cast<V2 *>(p) = V2{a.re, a.im};
}

// ------------------------------------------------------------------- SU(2) --
// q = (v0, v1, v2, s) is s + i v_k sigma_k, the reference's 4-real format.
struct quat { double v0, v1, v2, s; };

__device__ __forceinline__ quat load_link(const double *__restrict__ U, int site, int mu) {
    const double2 *p = reinterpret_cast<const double2 *>(U) + 2 * (3 * site + mu);
    const double2 a = __ldg(p), b = __ldg(p + 1);
    return {a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ void store_link(double *U, int site, int mu, quat q) {
    reinterpret_cast<double4 *>(U)[3 * site + mu] = double4{q.v0, q.v1, q.v2, q.s};
}
__device__ __forceinline__ quat qdag(quat a) { return {-a.v0, -a.v1, -a.v2, a.s}; }
__device__ __forceinline__ quat qmul(quat a, quat b) {
    quat c;
    c.s = a.s * b.s - (a.v0 * b.v0 + a.v1 * b.v1 + a.v2 * b.v2);
    c.v0 = a.s * b.v0 + b.s * a.v0 - (a.v1 * b.v2 - a.v2 * b.v1);
    c.v1 = a.s * b.v1 + b.s * a.v1 - (a.v2 * b.v0 - a.v0 * b.v2);
    c.v2 = a.s * b.v2 + b.s * a.v2 - (a.v0 * b.v1 - a.v1 * b.v0);
    return c;
}
__device__ __forceinline__ double qcomp(const quat &q, int a) { return a == 0 ? q.v0 : (a == 1 ? q.v1 : q.v2); }

// Colour matrix of a link, M = [[s + i v2, v1 + i v0], [-v1 + i v0, s - i v2]].
template <typename T> struct cmat2 { cpx<T> m00, m01, m10, m11; };

template <typename T> __device__ __forceinline__ cmat2<T> link_matrix(quat q) {
    return {mk<T>((T)q.s, (T)q.v2), mk<T>((T)q.v1, (T)q.v0), mk<T>((T)-q.v1, (T)q.v0), mk<T>((T)q.s, (T)-q.v2)};
}
// Link of direction mu at `site`, dressed by the U(1) background phase of the
// (x, y) plane when one is set: u1 holds QED::U, index mu + 2 (x + N0 y) for
// mu = 0, 1 (QED/QED.cpp:6-23); the z links carry no U(1) phase.
template <typename T>
__device__ __forceinline__ cmat2<T> dressed_link(const double *__restrict__ U, const double2 *__restrict__ u1,
                                                 int site, int mu, int n01) {
    cmat2<T> M = link_matrix<T>(load_link(U, site, mu));
    if (u1 != nullptr && mu < 2) {
        const double2 ph = __ldg(u1 + 2 * (site % n01) + mu);
        const cpx<T> p = mk<T>((T)ph.x, (T)ph.y);
        M.m00 = p * M.m00;
        M.m01 = p * M.m01;
        M.m10 = p * M.m10;
        M.m11 = p * M.m11;
    }
    return M;
}

// M h
// a h0 + b h1 (CONJ: conj(a) h0 + conj(b) h1) as two chains of fused
// multiply-adds, one per real and imaginary part: 2 multiplies and 6 fused
// multiply-adds instead of 4 + 4 and 2 adds (the signs of the im * im terms
// are operand negations).
template <typename T, bool CONJ>
__device__ __forceinline__ cpx<T> row2(const cpx<T> &a, const cpx<T> &b, const cpx<T> &h0, const cpx<T> &h1) {
    const T s = CONJ ? (T)1 : (T)-1;  // sign of a.im * h.im in the real part
    return {fma(a.re, h0.re, fma(s * a.im, h0.im, fma(b.re, h1.re, s * b.im * h1.im))),
            fma(a.re, h0.im, fma(-s * a.im, h0.re, fma(b.re, h1.im, -s * b.im * h1.re)))};
}
template <typename T> __device__ __forceinline__ void mul(const cmat2<T> &M, cpx<T> h0, cpx<T> h1, cpx<T> &k0, cpx<T> &k1) {
    k0 = row2<T, false>(M.m00, M.m01, h0, h1);
    k1 = row2<T, false>(M.m10, M.m11, h0, h1);
}
// M^+ h
template <typename T> __device__ __forceinline__ void mul_dag(const cmat2<T> &M, cpx<T> h0, cpx<T> h1, cpx<T> &k0, cpx<T> &k1) {
    k0 = row2<T, true>(M.m00, M.m10, h0, h1);
    k1 = row2<T, true>(M.m01, M.m11, h0, h1);
}

// exp(i c alpha^a sigma^a / 2)
__device__ inline quat qexp(double c, double a0, double a1, double a2) {
    double d = sqrt((c * a0) * (c * a0) + (c * a1) * (c * a1) + (c * a2) * (c * a2));
    if (d == 0.0) return {0.0, 0.0, 0.0, 1.0};
    double sn, cs;
    sincos(0.5 * d, &sn, &cs);
    double f = c * sn / d;
    return {f * a0, f * a1, f * a2, cs};
}

// Adjoint representation R_ab = 2 tr(t^a q t^b q^+), written out for a quaternion.
struct adj3 { double r[3][3]; };
__device__ inline adj3 adjoint(quat q) {
    adj3 R;
    const double a = q.v0, b = q.v1, c = q.v2, d = q.s;
    R.r[0][0] = a * a + d * d - b * b - c * c;
    R.r[0][1] = 2.0 * (a * b + c * d);
    R.r[0][2] = 2.0 * (a * c - b * d);
    R.r[1][0] = 2.0 * (a * b - c * d);
    R.r[1][1] = b * b + d * d - a * a - c * c;
    R.r[1][2] = 2.0 * (b * c + a * d);
    R.r[2][0] = 2.0 * (a * c + b * d);
    R.r[2][1] = 2.0 * (b * c - a * d);
    R.r[2][2] = c * c + d * d - a * a - b * b;
    return R;
}

// --------------------------------------------------------------- Dirac rep --
// Every matrix of the Dirac algebra in the Dirac representation
// (DiracAlgebra.cpp:5-12) has one nonzero per row: (G psi)_a = i^ph[a] psi_perm[a].
struct mono { int perm[4]; int ph[4]; };

__host__ __device__ constexpr mono mono_mul(mono A, mono B) {
    mono C{};
    for (int a = 0; a < 4; a++) {
        C.perm[a] = B.perm[A.perm[a]];
        C.ph[a] = (A.ph[a] + B.ph[A.perm[a]]) & 3;
    }
    return C;
}
constexpr mono kGamma0{{0, 1, 2, 3}, {0, 0, 2, 2}};
constexpr mono kGammaX{{3, 2, 1, 0}, {0, 0, 2, 2}};
constexpr mono kGammaY{{3, 2, 1, 0}, {3, 1, 1, 3}};
constexpr mono kGammaZ{{2, 3, 0, 1}, {0, 2, 2, 0}};
constexpr mono kGamma5{{2, 3, 0, 1}, {0, 0, 0, 0}};

template <typename T> __device__ __forceinline__ cpx<T> iphase(int ph, cpx<T> a) {
    switch (ph & 3) {
        case 0: return a;
        case 1: return times_i(a);
        case 2: return mk<T>(-a.re, -a.im);
        default: return times_mi(a);
    }
}

// sum_a conj(f_a) (G h)_a for one colour
template <typename T>
__device__ __forceinline__ cpx<T> bilinear(const mono &G, const cpx<T> *f, const cpx<T> *h) {
    cpx<T> t = mk<T>(0, 0);
#pragma unroll
    for (int a = 0; a < 4; a++) t = t + cdot(f[a], iphase(G.ph[a], h[G.perm[a]]));
    return t;
}

}  // namespace ovl
