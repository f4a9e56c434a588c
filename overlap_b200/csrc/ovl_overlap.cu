// Overlap evolution operator -i h_ov on the mode batch (FP64 parity form).
//
// Reference: OverlapOperator::Compute (FERMIONS/OVERLAP/OPERATOR/OverlapOperator.cpp:25-65)
// -> OverlapU (OverlapU.cpp:152-208) -> Zolotrr (OverlapU.cpp:5-149):
//   chi = sum_k b_k (h_W^2 + d_k)^-1 phi        (multi-shift CG, 25 shifts)
//   out = M [ -i g0 (1 + m/2) phi + (1 - m/2) D chi ],   D = -i h_W,  h_W^2 = -D^2.
// The reference runs the multi-shift CG once per mode; here every mode of the
// batch runs it in lockstep.  Each mode keeps its own CG scalars and stops on
// its own test (rnorm > cgerr * bnorm, at most nitcgm iterations, OverlapU.cpp:56,113)
// through a per-mode `active` mask, so every mode takes exactly the iterations
// the reference would.  The scalar recurrences keep the reference's order of
// operations (OverlapU.cpp:71-110).  Dot products are per mode, two-stage with
// a fixed order.

#include <algorithm>
#include <vector>

#include "ovl_device.cuh"
#include "ovl_internal.h"

namespace ovl {

// Elementwise loop over one field: element e = ((mb*V + site)*kComp + comp)*32 + lane.
#define OVL_FIELD_LOOP(n)                                                                                    \
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (n); e += (size_t)gridDim.x * blockDim.x)

__device__ __forceinline__ int mode_of(size_t e, int V) {
    const int lane = (int)(e % kModeBlock);
    const size_t mb = e / ((size_t)V * kComp * kModeBlock);
    return (int)mb * kModeBlock + lane;
}

static int elem_grid(size_t n, int sm_count) {
    size_t b = (n + 255) / 256;
    size_t cap = (size_t)sm_count * 16;
    return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

// ------------------------------------------------------------ dot products --
// part[chunk][mode] = sum over the chunk's sites and all components of Re(conj(a) b)
// (or |a|^2 when b == a).  Grid: (n_mb, kDotChunks), one warp per CTA.
__global__ void dot_partial_kernel(const cpx<double> *__restrict__ a, const cpx<double> *__restrict__ b, int V,
                                   double *__restrict__ part, int modes_padded) {
    const int lane = threadIdx.x, mb = blockIdx.x, chunk = blockIdx.y;
    const int s0 = (int)((long long)V * chunk / kDotChunks), s1 = (int)((long long)V * (chunk + 1) / kDotChunks);
    double t = 0.0;
    for (int s = s0; s < s1; s++)
        for (int c = 0; c < kComp; c++) {
            const size_t i = field_index(V, mb, s, c, lane);
            const cpx<double> x = ld(a + i), y = ld(b + i);
            t += x.re * y.re + x.im * y.im;
        }
    part[(size_t)chunk * modes_padded + mb * kModeBlock + lane] = t;
}

__global__ void dot_finish_kernel(const double *__restrict__ part, int modes_padded, double *__restrict__ out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= modes_padded) return;
    double t = 0.0;
    for (int c = 0; c < kDotChunks; c++) t += part[(size_t)c * modes_padded + m];
    out[m] = t;
}

// ---------------------------------------------------------- vector kernels --
// r = phi, p_k = phi, x_k = 0
__global__ void mscg_init_vectors_kernel(const cpx<double> *__restrict__ phi, cpx<double> *r, cpx<double> *p,
                                         cpx<double> *x, size_t n, int npoles) {
    OVL_FIELD_LOOP(n) {
        const cpx<double> v = ld(phi + e);
        st(r + e, v);
        for (int k = 0; k < npoles; k++) {
            st(p + (size_t)k * n + e, v);
            st(x + (size_t)k * n + e, mk<double>(0.0, 0.0));
        }
    }
}

// q = -q + d0 p0   (q holds D(D p0) on entry; h_W^2 p0 = -D^2 p0, WilsonUU, RitzSolver.cpp:49-89)
__global__ void shifted_square_kernel(cpx<double> *q, const cpx<double> *__restrict__ p0, size_t n, double d0) {
    OVL_FIELD_LOOP(n) {
        const cpx<double> a = ld(q + e), b = ld(p0 + e);
        st(q + e, mk<double>(-a.re + b.re * d0, -a.im + b.im * d0));
    }
}

// r -= beta0 q for active modes
__global__ void residual_kernel(cpx<double> *r, const cpx<double> *__restrict__ q, const double *__restrict__ beta0,
                                const int *__restrict__ active, size_t n, int V) {
    OVL_FIELD_LOOP(n) {
        const int m = mode_of(e, V);
        if (!active[m]) continue;
        const double b = beta0[m];
        const cpx<double> a = ld(r + e), y = ld(q + e);
        st(r + e, mk<double>(a.re - b * y.re, a.im - b * y.im));
    }
}

// x_k += beta_k p_k ; p_k = p_k alpha_k + r g_k   for active modes (OverlapU.cpp:95-108)
__global__ void shift_update_kernel(cpx<double> *x, cpx<double> *p, const cpx<double> *__restrict__ r,
                                    const double *__restrict__ beta, const double *__restrict__ alpha,
                                    const double *__restrict__ g, const int *__restrict__ active, size_t n, int V,
                                    int npoles, int modes_padded) {
    OVL_FIELD_LOOP(n) {
        const int m = mode_of(e, V);
        if (!active[m]) continue;
        const cpx<double> rv = ld(r + e);
        for (int k = 0; k < npoles; k++) {
            const size_t i = (size_t)k * n + e;
            const size_t s = (size_t)k * modes_padded + m;
            const cpx<double> pv = ld(p + i), xv = ld(x + i);
            const double bk = beta[s], ak = alpha[s], gk = g[s];
            st(x + i, mk<double>(xv.re + bk * pv.re, xv.im + bk * pv.im));
            st(p + i, mk<double>(pv.re * ak + rv.re * gk, pv.im * ak + rv.im * gk));
        }
    }
}

// chi = sum_k b_k x_k (OverlapU.cpp:129-133)
__global__ void combine_shifts_kernel(cpx<double> *chi, const cpx<double> *__restrict__ x, const double *__restrict__ bz,
                                      size_t n, int npoles) {
    OVL_FIELD_LOOP(n) {
        cpx<double> t = mk<double>(0.0, 0.0);
        for (int k = 0; k < npoles; k++) {
            const cpx<double> v = ld(x + (size_t)k * n + e);
            t = mk<double>(t.re + v.re * bz[k], t.im + v.im * bz[k]);
        }
        st(chi + e, t);
    }
}

// out = M [ -i g0 (1 + m/2) phi + (1 - m/2) Dchi ]  (OverlapU.cpp:188-202); dst = out or dst += dt out
__global__ void overlap_finish_kernel(const cpx<double> *__restrict__ phi, const cpx<double> *__restrict__ dchi,
                                      cpx<double> *dst, size_t n, double mdw, double mf, double dt, int accumulate) {
    OVL_FIELD_LOOP(n) {
        const int spin = (int)((e / kModeBlock) % kComp) % kSpin;
        const cpx<double> f = ld(phi + e), d = ld(dchi + e);
        const double cp = 1.0 + 0.5 * mf, cm = 1.0 - 0.5 * mf;
        // -i g0: spins 0,1 -> -i, spins 2,3 -> +i
        const cpx<double> a = spin < 2 ? mk<double>(cp * f.im, -cp * f.re) : mk<double>(-cp * f.im, cp * f.re);
        const cpx<double> o = mk<double>(mdw * (a.re + cm * d.re), mdw * (a.im + cm * d.im));
        if (accumulate) {
            const cpx<double> v = ld(dst + e);
            st(dst + e, mk<double>(v.re + dt * o.re, v.im + dt * o.im));
        } else {
            st(dst + e, o);
        }
    }
}

// ---------------------------------------------------------- scalar kernels --
struct CgScalars {
    double *rnorm, *bnorm, *betam, *pap, *rr;
    double *alpha, *beta, *z, *g;  // [npoles][modes_padded]
    int *active, *next, *iters;    // active this iteration / after it
    int *count;                    // number of modes active after the update
};

// rnorm = |phi|^2, bnorm = sqrt(rnorm), betam = 1, alpha_0 = 0, z_k = g_k = 1 (OverlapU.cpp:39-54)
__global__ void cg_init_scalars_kernel(CgScalars s, const double *__restrict__ norm2, int n_modes, int modes_padded,
                                       int npoles, double cgerr) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= modes_padded) return;
    const double rn = norm2[m];
    s.rnorm[m] = rn;
    s.bnorm[m] = sqrt(rn);
    s.betam[m] = 1.0;
    for (int k = 0; k < npoles; k++) {
        s.alpha[(size_t)k * modes_padded + m] = 0.0;
        s.z[(size_t)k * modes_padded + m] = 1.0;
        s.g[(size_t)k * modes_padded + m] = 1.0;
        s.beta[(size_t)k * modes_padded + m] = 0.0;
    }
    s.iters[m] = 0;
    const int act = (m < n_modes) && (rn > cgerr * sqrt(rn));
    s.active[m] = act;
    s.next[m] = act;
    if (act) atomicAdd(s.count, 1);
}

// beta_0 = rnorm / <p0, q>; for k >= 1: z_k, beta_k from the previous alpha_0,
// z_k, betam (OverlapU.cpp:71-88)
__global__ void cg_scalars_beta_kernel(CgScalars s, const double *__restrict__ dz, int modes_padded, int npoles) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= modes_padded || !s.active[m]) return;
    const double b0 = s.rnorm[m] / s.pap[m];
    s.beta[m] = b0;
    const double a0 = s.alpha[m], bm = s.betam[m];
    for (int k = 1; k < npoles; k++) {
        const size_t i = (size_t)k * modes_padded + m;
        const double dr = b0 * a0 * (1.0 - s.z[i]) + bm * (1.0 + (dz[k] - dz[0]) * b0);
        s.z[i] = bm / dr;
        s.beta[i] = b0 * s.z[i];
    }
}

// alpha_0 = |r|^2 / rnorm, rnorm = |r|^2; per shift alpha_k and g_k as the
// shift loop of OverlapU.cpp:95-106 computes them (alpha_0 is rewritten at
// k = 0 before the other shifts read it); betam = beta_0; iteration count and
// the stopping test (OverlapU.cpp:56, 110-117).
__global__ void cg_scalars_alpha_kernel(CgScalars s, int modes_padded, int npoles, double cgerr, int max_iter) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= modes_padded) return;
    if (!s.active[m]) {
        s.next[m] = 0;
        return;
    }
    const double rr = s.rr[m];
    double a0 = rr / s.rnorm[m];
    s.rnorm[m] = rr;
    const double b0 = s.beta[m];
    for (int k = 0; k < npoles; k++) {
        const size_t i = (size_t)k * modes_padded + m;
        const double ak = a0 * s.z[i] * s.beta[i] / b0;
        if (k == 0) a0 = ak;
        s.alpha[i] = ak;
        s.g[i] = s.g[i] * s.z[i];
    }
    s.betam[m] = b0;
    const int it = s.iters[m] + 1;
    s.iters[m] = it;
    const int act = (it < max_iter) && (rr > cgerr * s.bnorm[m]);
    s.next[m] = act;
    if (act) atomicAdd(s.count, 1);
}

// --------------------------------------------------------- overlap currents --
// Fermions::Observables::ComputeCurrents, overlap (FERMIONS/OVERLAP/OverlapCurrents.cpp:35-212):
// local bilinears only, with O = -i h_ov psi:
//   jV^mu = Re[psi^+ g0 g_mu psi + psi^+ (-i/2) g0 g_mu g0 O]
//   jA^mu = Re[psi^+ g0 g_mu g5 psi + psi^+ (-i/2) g0 g_mu g5 g0 O]      (g_0 for mu = 0)
// weighted by the vacuum sign and summed over colours and modes; per site the
// output slots are those of the Wilson currents (jV, jA; the rest zero).
// Modes of precision T and NC colours; the bilinears in FP64.
template <typename T, int NC>
__global__ void __launch_bounds__(kModeBlock *kSitesPerCta)
    overlap_currents_kernel(const cpx<T> *__restrict__ psi, const cpx<T> *__restrict__ opsi, Lattice L,
                            int n_mb, int n_modes, int first_mode, int groups, double *__restrict__ partial) {
    constexpr mono GV[4] = {mono_mul(kGamma0, kGamma0), mono_mul(kGamma0, kGammaX), mono_mul(kGamma0, kGammaY),
                            mono_mul(kGamma0, kGammaZ)};
    constexpr mono GA[4] = {mono_mul(GV[0], kGamma5), mono_mul(GV[1], kGamma5), mono_mul(GV[2], kGamma5),
                            mono_mul(GV[3], kGamma5)};
    constexpr mono GV2[4] = {mono_mul(GV[0], kGamma0), mono_mul(GV[1], kGamma0), mono_mul(GV[2], kGamma0),
                             mono_mul(GV[3], kGamma0)};
    constexpr mono GA2[4] = {mono_mul(GA[0], kGamma0), mono_mul(GA[1], kGamma0), mono_mul(GA[2], kGamma0),
                             mono_mul(GA[3], kGamma0)};
    const int lane = threadIdx.x;
    const int site = blockIdx.x * kSitesPerCta + threadIdx.y;
    const int g = blockIdx.y;
    if (site >= L.V) return;
    CompSum sum[8];
    for (int mb = g; mb < n_mb; mb += groups) {
        const int mode = mb * kModeBlock + lane;
        const double w = mode >= n_modes ? 0.0 : (((first_mode + mode) & 1) == 0 ? 1.0 : -1.0);
        cpx<double> f[NC][kSpin], o[NC][kSpin];
        const size_t base = (((size_t)mb * L.V + site) * (NC * kSpin)) * kModeBlock + lane;
#pragma unroll
        for (int c = 0; c < NC; c++)
#pragma unroll
            for (int a = 0; a < kSpin; a++) {
                const cpx<T> x = ld(psi + base + (c * kSpin + a) * kModeBlock);
                const cpx<T> y = ld(opsi + base + (c * kSpin + a) * kModeBlock);
                f[c][a] = mk<double>((double)x.re, (double)x.im);
                o[c][a] = mk<double>((double)y.re, (double)y.im);
            }
#pragma unroll
        for (int mu = 0; mu < 4; mu++) {
            cpx<double> v1 = mk<double>(0, 0), v2 = mk<double>(0, 0), a1 = mk<double>(0, 0), a2 = mk<double>(0, 0);
#pragma unroll
            for (int c = 0; c < NC; c++) {
                v1 = v1 + bilinear<double>(GV[mu], f[c], f[c]);
                v2 = v2 + bilinear<double>(GV2[mu], f[c], o[c]);
                a1 = a1 + bilinear<double>(GA[mu], f[c], f[c]);
                a2 = a2 + bilinear<double>(GA2[mu], f[c], o[c]);
            }
            // Re(z1 + (-i/2) z2) = Re z1 + Im z2 / 2
            sum[mu].add(w * (v1.re + 0.5 * v2.im));
            sum[4 + mu].add(w * (a1.re + 0.5 * a2.im));
        }
    }
    double acc[8];
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] = sum[k].value();
#pragma unroll
    for (int k = 0; k < 8; k++) {
        double t = acc[k];
        for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
        acc[k] = t;
    }
    if (lane == 0) {
        double *p = partial + ((size_t)g * L.V + site) * kCurrentsPerSite;
        for (int k = 0; k < kCurrentsPerSite; k++) p[k] = k < 8 ? acc[k] : 0.0;
    }
}

template <typename T, int NC>
static void overlap_currents_t(const void *psi, const void *opsi, const Lattice &L, int n_mb, int n_modes,
                               int first_mode, int groups, double *partial, cudaStream_t stream) {
    dim3 block(kModeBlock, kSitesPerCta);
    dim3 grid((L.V + kSitesPerCta - 1) / kSitesPerCta, groups);
    overlap_currents_kernel<T, NC><<<grid, block, 0, stream>>>(reinterpret_cast<const cpx<T> *>(psi),
                                                               reinterpret_cast<const cpx<T> *>(opsi), L, n_mb, n_modes,
                                                               first_mode, groups, partial);
}

void launch_overlap_currents(const void *psi, const void *opsi, const Lattice &L, int n_mb, int n_modes,
                             int first_mode, double *partial, double *per_site, cudaStream_t stream, bool fp32, int nc) {
    const int groups = currents_groups(n_mb);
    if (nc == 3) {
        if (fp32) overlap_currents_t<float, 3>(psi, opsi, L, n_mb, n_modes, first_mode, groups, partial, stream);
        else overlap_currents_t<double, 3>(psi, opsi, L, n_mb, n_modes, first_mode, groups, partial, stream);
    } else {
        if (fp32) overlap_currents_t<float, 2>(psi, opsi, L, n_mb, n_modes, first_mode, groups, partial, stream);
        else overlap_currents_t<double, 2>(psi, opsi, L, n_mb, n_modes, first_mode, groups, partial, stream);
    }
    launch_currents_finish(partial, groups, L, per_site, stream);
}

// ------------------------------------------------------------------ driver --
void overlap_apply(OverlapWork &w, const double *U, const double *u1, const void *src, void *dst, const Lattice &L, int n_mb,
                   int n_modes, const OverlapCoeffs &co, double amass, double mdw, double mf, double dt,
                   bool accumulate, int sm_count, cudaStream_t stream, OverlapStats *stats) {
    const size_t n = (size_t)n_mb * L.V * kComp * kModeBlock;
    const int mp = n_mb * kModeBlock;
    const int np = co.npoles;
    const int grid = elem_grid(n, sm_count);
    const int sg = (mp + 127) / 128;
    const cpx<double> *phi = reinterpret_cast<const cpx<double> *>(src);
    cpx<double> *r = reinterpret_cast<cpx<double> *>(w.r), *q = reinterpret_cast<cpx<double> *>(w.q);
    cpx<double> *t = reinterpret_cast<cpx<double> *>(w.t);
    cpx<double> *x = reinterpret_cast<cpx<double> *>(w.x), *p = reinterpret_cast<cpx<double> *>(w.p);
    CgScalars s{w.rnorm, w.bnorm, w.betam, w.pap, w.rr, w.alpha, w.beta, w.z, w.g, w.active, w.next, w.iters, w.count};
    cudaMemcpyAsync(w.dz, co.d, sizeof(double) * np, cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(w.bz, co.b, sizeof(double) * np, cudaMemcpyHostToDevice, stream);

    mscg_init_vectors_kernel<<<grid, 256, 0, stream>>>(phi, r, p, x, n, np);
    dim3 dgrid(n_mb, kDotChunks);
    dot_partial_kernel<<<dgrid, kModeBlock, 0, stream>>>(phi, phi, L.V, w.part, mp);
    dot_finish_kernel<<<sg, 128, 0, stream>>>(w.part, mp, w.rr);
    cudaMemsetAsync(w.count, 0, sizeof(int), stream);
    cg_init_scalars_kernel<<<sg, 128, 0, stream>>>(s, w.rr, n_modes, mp, np, co.cg_tol);
    int launches = 5;
    int active = 0;
    cudaMemcpyAsync(w.host_count, w.count, sizeof(int), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    active = *w.host_count;
    int iterations = 0;
    while (active > 0) {
        // q = h_W^2 p0 + d0 p0 = -D(D p0) + d0 p0
        launch_wilson<double>(U, u1, p, w.t, L, 0, n_mb, amass, 0.0, false, stream);
        launch_wilson<double>(U, u1, w.t, w.q, L, 0, n_mb, amass, 0.0, false, stream);
        shifted_square_kernel<<<grid, 256, 0, stream>>>(q, p, n, co.d[0]);
        dot_partial_kernel<<<dgrid, kModeBlock, 0, stream>>>(p, q, L.V, w.part, mp);
        dot_finish_kernel<<<sg, 128, 0, stream>>>(w.part, mp, w.pap);
        cg_scalars_beta_kernel<<<sg, 128, 0, stream>>>(s, w.dz, mp, np);
        residual_kernel<<<grid, 256, 0, stream>>>(r, q, w.beta, s.active, n, L.V);
        dot_partial_kernel<<<dgrid, kModeBlock, 0, stream>>>(r, r, L.V, w.part, mp);
        dot_finish_kernel<<<sg, 128, 0, stream>>>(w.part, mp, w.rr);
        cudaMemsetAsync(w.count, 0, sizeof(int), stream);
        cg_scalars_alpha_kernel<<<sg, 128, 0, stream>>>(s, mp, np, co.cg_tol, co.cg_max_iter);
        shift_update_kernel<<<grid, 256, 0, stream>>>(x, p, r, w.beta, w.alpha, w.g, s.active, n, L.V, np, mp);
        launches += 11;
        std::swap(s.active, s.next);
        cudaMemcpyAsync(w.host_count, w.count, sizeof(int), cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
        active = *w.host_count;
        iterations++;
        if (iterations > co.cg_max_iter + 1) break;  // every mode stops by then
    }
    combine_shifts_kernel<<<grid, 256, 0, stream>>>(q, x, w.bz, n, np);
    launch_wilson<double>(U, u1, q, w.t, L, 0, n_mb, amass, 0.0, false, stream);
    overlap_finish_kernel<<<grid, 256, 0, stream>>>(phi, t, reinterpret_cast<cpx<double> *>(dst), n, mdw, mf, dt,
                                                    accumulate ? 1 : 0);
    launches += 3;
    if (stats) {
        stats->launches += launches;
        stats->iterations = iterations;
        int mx = 0;
        std::vector<int> it(mp);
        cudaMemcpyAsync(it.data(), w.iters, sizeof(int) * mp, cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
        int capped = 0;
        for (int m = 0; m < n_modes; m++) {
            mx = std::max(mx, it[m]);
            if (it[m] >= co.cg_max_iter) capped++;
        }
        stats->max_mode_iterations = mx;
        stats->not_converged = capped;
    }
}

}  // namespace ovl
