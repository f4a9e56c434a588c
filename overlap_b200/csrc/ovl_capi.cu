// C ABI of overlap_b200 (include/ovl.h): context lifetime, host <-> device
// transfers in the reference's layouts, and the leapfrog driver.

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "ovl.h"
#include "ovl_device.cuh"
#include "ovl_internal.h"

using ovl::Lattice;

struct ovl_ctx {
    ovl_params p{};
    int nc = 2;                   // colours: 2 (quaternion links) or 3 (3x3 complex links)
    int comp = 8;                 // complex components per mode and site (4 nc)
    int link_doubles = 4;         // doubles per link
    int e_comp = 3;               // E components per link (nc^2 - 1)
    Lattice L{};
    int n_mb = 0;                 // mode blocks of 32
    size_t field_complex = 0;     // complex numbers per mode field
    size_t elem_bytes = 0;        // bytes per complex number
    void *psi = nullptr, *psimid = nullptr;
    double *U = nullptr, *E = nullptr;
    void *deriv = nullptr;        // plain form: derivative buffer
    int deriv_mb = 0;             // mode blocks per derivative chunk
    double *per_site = nullptr;   // currents per site
    double *partial = nullptr;    // reduction scratch
    size_t partial_doubles = 0;
    double *dev_small = nullptr;  // small device results
    double *host_small = nullptr; // pinned mirror
    int *dev_int = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int tsteps = 0;
    int sm_count = 148;
    uint64_t launches = 0;
    std::string err;
    // overlap fermions
    ovl::OverlapWork ow;
    std::vector<double> bounds;   // (lambda_min, lambda_max) per overlap application
    size_t bound_next = 0;
    double coeff_lo = -1.0, coeff_hi = -1.0;
    ovl::OverlapCoeffs coeffs{};
    ovl::OverlapStats ostats;
    ovl::ChebyshevWork cw;
    std::vector<double> cheb;     // Chebyshev coefficients c_0..c_K
    void *aux_src = nullptr, *aux_dst = nullptr;  // ovl_apply / overlap currents
    // U(1) background phases of the hopping term (ovl_set_u1)
    double *u1 = nullptr;
    bool u1_on = false;
    // FP32 copies of links and phases for the FP32 hopping kernels; kernel variant
    float *U32 = nullptr, *u1_32 = nullptr;
    int hop_variant = -1;  // -1: autotune before the first step
    int mode_group = -1;   // mode blocks per group of the grouped fused step (0: whole batch)
    double *U_b = nullptr; // links at the half step (grouped fused step)
    void *psi_lo = nullptr, *psimid_lo = nullptr;      // FP40 extension bytes of the mode fields
    void *aux_src_lo = nullptr, *aux_dst_lo = nullptr; // and of the operator buffers (autotuner)
    float *U32_b = nullptr;
    // Chern-Simons number along the cooling path (ovl_ncs_update)
    double *u_old = nullptr, *u_mid = nullptr, *e_mid = nullptr;
    bool have_u_old = false;
    double ncs_total = 0.0;
    // Ritz solver for the overlap spectral bounds (ovl_ritz_bounds, ritz_auto)
    void *ritz = nullptr;
    uint64_t ritz_calls = 0;
    double ritz_last[2] = {0.0, 0.0};
    // charges summed inside the last half step (ovl_step_observe)
    double *obs_partial = nullptr, *obs_scratch = nullptr;
    // pipelined grouped step (FP32, hop variant 3): per-group counters, ticket,
    // error word; pipe_ran: a pipelined step was enqueued since the last check
    int *pipe = nullptr;
    bool pipe_ran = false;
    // per-kernel timing (ovl_profile_enable): event pairs per kind
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof[OVL_PROF_KINDS];
    std::vector<cudaEvent_t> event_pool;
};

namespace {

std::string g_err;  // errors without a context (creation)

int fail(ovl_ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf; else g_err = buf;
    return code;
}

int cuda_fail(ovl_ctx *c, cudaError_t e, const char *what) {
    return fail(c, OVL_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define OVL_CUDA(c, call)                                         \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail((c), e_, #call);  \
    } while (0)

// Brackets a launch with events when profiling is on.
struct ProfScope {
    ovl_ctx *c;
    int kind;
    cudaEvent_t start = nullptr;
    cudaEvent_t take() {
        if (c->event_pool.empty()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            return e;
        }
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    ProfScope(ovl_ctx *ctx, int k) : c(ctx), kind(k) {
        if (c->profiling && (start = take())) cudaEventRecord(start, c->stream);
    }
    ~ProfScope() {
        if (!start) return;
        cudaEvent_t stop = take();
        if (!stop) { c->event_pool.push_back(start); return; }
        cudaEventRecord(stop, c->stream);
        c->prof[kind].emplace_back(start, stop);
    }
};

// Checks for launch errors after a batch of `n` kernel launches.
int launched(ovl_ctx *c, int n, const char *what) {
    c->launches += (uint64_t)n;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, what);
    return OVL_OK;
}

bool all_finite(const double *a, size_t n) {
    for (size_t i = 0; i < n; i++)
        if (!std::isfinite(a[i])) return false;
    return true;
}

int set_device(ovl_ctx *c) {
    OVL_CUDA(c, cudaSetDevice(c->p.device));
    return OVL_OK;
}

bool fp32(const ovl_ctx *c) { return c->p.precision == OVL_PREC_FP32; }
// 40-bit storage: high words in the field, extension bytes in a parallel array
bool fp40(const ovl_ctx *c) { return c->p.precision == OVL_PREC_FP40; }

double amass(const ovl_params &p) { return 6.0 * p.r_wilson + 2.0 * p.m_fermion - 2.0 * p.m_dw; }

bool overlap(const ovl_ctx *c) { return c->p.fermion == OVL_FERMION_OVERLAP; }

bool su3(const ovl_ctx *c) { return c->nc == 3; }

ovl::Su3Links su3_links(const ovl_ctx *c) {
    ovl::Su3Links lk;
    lk.U = c->U;
    lk.u1 = c->u1_on ? c->u1 : nullptr;
    lk.U32 = c->U32;
    lk.u1_32 = c->u1_on ? c->u1_32 : nullptr;
    lk.variant = c->hop_variant < 0 ? 0 : c->hop_variant;
    return lk;
}

// The link update of either colour count (Dynamics.cpp:97-138).
void launch_links(ovl_ctx *c, double *U, float *U32, double dt_step) {
    if (su3(c)) ovl::su3_launch_update_links(U, c->E, c->L, dt_step, U32, c->p.reunitarize != 0, c->stream);
    else ovl::launch_update_links(U, c->E, c->L, dt_step, c->stream, U32, c->p.reunitarize != 0);
}

// Upper bound on h_W^2 for any gauge field: ||h_W|| <= |6r + 2m - 2M| / 2 + 3
// (the hopping term is a sum of three operators of norm one).
double wilson_norm_bound2(const ovl_params &p) {
    const double b = 0.5 * std::fabs(amass(p)) + 3.0;
    return b * b;
}

// Zolotarev coefficients for the next overlap application; `consume` advances
// the bounds schedule (OverlapUpdate.cpp:105,119 recompute the bounds before
// every half step).
// ComputeRitzEigenvalues (OverlapUpdate.cpp:61-97): MinEValue = 0.95 lambda_min,
// MaxEValue = 1.05 lambda_max, with MaximumIterations 2000, NumberOfRestarts 100,
// NormRatio 1e-16 (:53-58).
int ritz_bounds(ovl_ctx *c, const double *start, double out[2], double raw[2], int iters[2]) {
    if (!c->ritz && !(c->ritz = ovl::ritz_create(c->L.V, c->nc))) return fail(c, OVL_E_OOM, "Ritz solver: work space");
    const size_t n = (size_t)c->L.V * 4 * c->nc;
    if (start)
        OVL_CUDA(c, cudaMemcpyAsync(ovl::ritz_start_buffer(c->ritz), start, sizeof(double2) * n, cudaMemcpyHostToDevice,
                                    c->stream));
    else
        ovl::launch_ritz_random_start(c->ritz, c->p.ritz_seed, c->ritz_calls++, c->stream);
    double r[2];
    int it[2];
    uint64_t nl = start ? 0 : 1;
    cudaError_t e;
    {
        ProfScope ps(c, OVL_PROF_OBS);
        e = ovl::ritz_run(c->ritz, c->U, c->u1_on ? c->u1 : nullptr, c->L, amass(c->p), 2000, 100, 1e-16, r, it,
                          c->stream, &nl);
    }
    c->launches += nl;
    if (e != cudaSuccess) return cuda_fail(c, e, "Ritz solver");
    const double lmin = r[0], lmax = -r[1];
    if (!(lmin > 0.0) || !(lmax > lmin) || !std::isfinite(lmax))
        return fail(c, OVL_E_STATE, "Ritz solver: bounds (%g, %g) are not 0 < min < max", lmin, lmax);
    out[0] = 0.95 * lmin;
    out[1] = 1.05 * lmax;
    c->ritz_last[0] = out[0];
    c->ritz_last[1] = out[1];
    if (raw) { raw[0] = lmin; raw[1] = lmax; }
    if (iters) { iters[0] = it[0]; iters[1] = it[1]; }
    return OVL_OK;
}


// (lambda_min, lambda_max) for the next overlap application: the next pair of
// the schedule set by ovl_set_spectral_bounds, or, with no schedule and
// ritz_auto, fresh Ritz bounds (OverlapUpdate.cpp:105,119 compute them before
// every half step).  `consume` advances the schedule.
int take_bounds(ovl_ctx *c, bool consume, double &lo, double &hi) {
    // the Chebyshev series without a schedule or Ritz bounds: on [eps, 1] of
    // h^2 / (the bound on h_W^2 that holds for every gauge field)
    if (c->bounds.empty() && c->p.sign_method == OVL_SIGN_CHEBYSHEV && !c->p.ritz_auto) {
        hi = wilson_norm_bound2(c->p);
        lo = c->p.cheb_eps * hi;
        return OVL_OK;
    }
    if (c->bounds.empty()) {
        if (!c->p.ritz_auto) return fail(c, OVL_E_STATE, "overlap: no spectral bounds set (ovl_set_spectral_bounds)");
        double b[2];
        int rc = ritz_bounds(c, nullptr, b, nullptr, nullptr);
        if (rc) return rc;
        lo = b[0];
        hi = b[1];
        return OVL_OK;
    }
    const size_t pairs = c->bounds.size() / 2;
    size_t i = pairs == 1 ? 0 : c->bound_next;
    if (i >= pairs) return fail(c, OVL_E_STATE, "overlap: spectral-bounds schedule exhausted after %zu applications", pairs);
    lo = c->bounds[2 * i];
    hi = c->bounds[2 * i + 1];
    if (consume && pairs > 1) c->bound_next++;
    return OVL_OK;
}

int next_coeffs(ovl_ctx *c, bool consume) {
    double lo, hi;
    int rc = take_bounds(c, consume, lo, hi);
    if (rc) return rc;
    if (lo != c->coeff_lo || hi != c->coeff_hi) {
        c->coeffs.npoles = c->p.zolo_poles;
        ovl::zolotarev(lo, hi, c->p.zolo_tol, c->p.zolo_poles, c->coeffs.b, c->coeffs.d);
        c->coeffs.cg_tol = c->p.cg_tol;
        c->coeffs.cg_max_iter = c->p.cg_max_iter;
        c->coeff_lo = lo;
        c->coeff_hi = hi;
    }
    return OVL_OK;
}

ovl::HopConfig hop_config(const ovl_ctx *c);
int su3_autotune(ovl_ctx *c, double ms_out[ovl::kHopVariants]);

int run_overlap(ovl_ctx *c, const void *src, void *dst, int n_mb, int n_modes, bool accumulate, bool consume) {
    if (c->p.sign_method == OVL_SIGN_CHEBYSHEV) {
        double lo, hi;
        int rc = take_bounds(c, consume, lo, hi);
        if (rc) return rc;
        if (su3(c) && c->hop_variant < 0 && (rc = su3_autotune(c, nullptr))) return rc;
        ProfScope ps(c, OVL_PROF_HOP);
        uint64_t nl = 0;
        if (su3(c) && fp32(c))
            ovl::su3_chebyshev_apply<float>(c->cw, su3_links(c), src, dst, c->L, n_mb, c->cheb.data(), c->p.cheb_degree,
                                            c->p.cheb_eps, hi, amass(c->p), c->p.m_dw, c->p.m_fermion, c->p.dt,
                                            accumulate, c->sm_count, c->stream, &nl);
        else if (su3(c))
            ovl::su3_chebyshev_apply<double>(c->cw, su3_links(c), src, dst, c->L, n_mb, c->cheb.data(),
                                             c->p.cheb_degree, c->p.cheb_eps, hi, amass(c->p), c->p.m_dw,
                                             c->p.m_fermion, c->p.dt, accumulate, c->sm_count, c->stream, &nl);
        else if (fp32(c))
            ovl::chebyshev_apply<float>(c->cw, hop_config(c), src, dst, c->L, n_mb, c->cheb.data(),
                                        c->p.cheb_degree, c->p.cheb_eps, hi, amass(c->p), c->p.m_dw, c->p.m_fermion,
                                        c->p.dt, accumulate, c->sm_count, c->stream, &nl);
        else
            ovl::chebyshev_apply<double>(c->cw, hop_config(c), src, dst, c->L, n_mb, c->cheb.data(),
                                         c->p.cheb_degree, c->p.cheb_eps, hi, amass(c->p), c->p.m_dw, c->p.m_fermion,
                                         c->p.dt, accumulate, c->sm_count, c->stream, &nl);
        c->ostats.iterations = c->ostats.max_mode_iterations = c->p.cheb_degree;
        c->ostats.not_converged = lo < c->p.cheb_eps * hi ? 1 : 0;
        return launched(c, (int)nl, "overlap operator (Chebyshev)");
    }
    int rc = next_coeffs(c, consume);
    if (rc) return rc;
    ProfScope ps(c, OVL_PROF_HOP);
    c->ostats.launches = 0;
    ovl::overlap_apply(c->ow, c->U, c->u1_on ? c->u1 : nullptr, src, dst, c->L, n_mb, n_modes, c->coeffs, amass(c->p), c->p.m_dw, c->p.m_fermion,
                       c->p.dt, accumulate, c->sm_count, c->stream, &c->ostats);
    return launched(c, (int)c->ostats.launches, "overlap operator");
}

ovl::HopConfig hop_config(const ovl_ctx *c) {
    ovl::HopConfig h;
    h.U = c->U;
    h.u1 = c->u1_on ? c->u1 : nullptr;
    if (c->p.precision == OVL_PREC_FP32) {
        h.U32 = c->U32;
        h.u1_32 = c->u1_on ? c->u1_32 : nullptr;
    }
    h.variant = c->hop_variant < 0 ? 0 : c->hop_variant;
    return h;
}

// Whether a host buffer is page-locked.  A copy from pageable memory has been
// staged when cudaMemcpyAsync returns, so the caller may reuse the buffer at
// once; a copy from page-locked memory may still be reading it, so the upload
// then waits for the copy before returning.
bool page_locked(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;  // unknown: wait, the safe choice
    }
    return a.type == cudaMemoryTypeHost;
}

void refresh_links32(ovl_ctx *c) {
    if (c->U32) {
        if (su3(c)) ovl::su3_launch_links_to_f32(c->U, c->U32, c->L, c->stream);
        else ovl::launch_links_to_f32(c->U, c->U32, (size_t)12 * c->L.V, c->stream);
        c->launches++;
    }
}

// One leapfrog step's hop work in the fused form, group by group:
// dst1 += dt D(src1) with links h1, then dst2 += dt D(src2) with links h2, for
// each group of `group` mode blocks (group <= 0 or >= n_mb: the whole batch).
// The extension bytes of a mode field or operator buffer in 40-bit storage.
void *lo_of(const ovl_ctx *c, const void *field) {
    if (field == c->psi) return c->psi_lo;
    if (field == c->psimid) return c->psimid_lo;
    if (field == c->aux_src) return c->aux_src_lo;
    if (field == c->aux_dst) return c->aux_dst_lo;
    return nullptr;
}

// The pipelined form of grouped_pass: FP32 with hop variant 3 and the FP32
// link copies, when the second half step reads the first one's output.
// (Its tickets are 32-bit: 2 x groups x 16-site tiles, below 2^31 for any
// fields that fit in device memory; checked all the same.)
bool pipelined(const ovl_ctx *c, const ovl::HopConfig &h1, const ovl::HopConfig &h2, const void *dst1,
               const void *src2) {
    const long long items = 2LL * c->n_mb * ((c->L.V + 15) / 16);  // at most, groups of one block
    return fp32(c) && c->pipe && h1.variant == ovl::kPackedVariant && h1.U32 && h2.U32 && dst1 == src2 &&
           items < (1LL << 31) - 1;
}

void grouped_pass(ovl_ctx *c, const ovl::HopConfig &h1, const ovl::HopConfig &h2, const void *src1, void *dst1,
                  const void *src2, void *dst2, int group, double *obs = nullptr) {
    const int G = (group <= 0 || group >= c->n_mb) ? c->n_mb : group;
    if (pipelined(c, h1, h2, dst1, src2)) {
        ovl::launch_wilson_pipeline(h1, h2, src1, dst1, dst2, c->L, c->n_mb, G, amass(c->p), c->p.dt, c->pipe,
                                    c->sm_count, c->p.n_modes, c->p.first_mode, obs, c->stream);
        c->launches += 1;
        c->pipe_ran = true;
        return;
    }
    for (int g0 = 0; g0 < c->n_mb; g0 += G) {
        const int nmb = std::min(G, c->n_mb - g0);
        if (fp40(c)) {
            ovl::launch_wilson40(h1, src1, lo_of(c, src1), dst1, lo_of(c, dst1), c->L, g0, nmb, amass(c->p), c->p.dt,
                                 true, c->stream);
            ovl::launch_wilson40(h2, src2, lo_of(c, src2), dst2, lo_of(c, dst2), c->L, g0, nmb, amass(c->p), c->p.dt,
                                 true, c->stream);
        } else if (fp32(c)) {
            ovl::launch_wilson_tuned<float>(h1, src1, dst1, c->L, g0, nmb, amass(c->p), c->p.dt, true, c->stream);
            ovl::launch_wilson_tuned<float>(h2, src2, dst2, c->L, g0, nmb, amass(c->p), c->p.dt, true, c->stream);
        } else {
            ovl::launch_wilson_tuned<double>(h1, src1, dst1, c->L, g0, nmb, amass(c->p), c->p.dt, true, c->stream);
            ovl::launch_wilson_tuned<double>(h2, src2, dst2, c->L, g0, nmb, amass(c->p), c->p.dt, true, c->stream);
        }
        c->launches += 2;
    }
}

// Times candidates 0..n-1 of one launch (run(k) enqueues candidate k on
// `stream` and returns the kernels it launched) and writes each one's time per
// launch into ms[k].  First a burst: one warm-up and three timed launches per
// candidate.  Where the fastest burst takes kSustainMinMs or more, the GPU
// reaches its power cap within a run of such launches, and then the clock a
// kernel holds depends on its own power draw: each candidate is timed again
// over windows of about kSustainWindowMs of back-to-back launches (the second
// half of each window timed), in kSustainRounds rounds whose order alternates
// 0..n-1, n-1..0 (a drift of the clock over the tuning cancels), and ms[k] is
// the median of its rounds (one window caught by a clock excursion does not
// decide).  Returns false if an event could not be created.
constexpr double kSustainMinMs = 1.0, kSustainWindowMs = 120.0;
constexpr int kSustainRounds = 6;

template <class F>
bool time_candidates(cudaStream_t stream, int n, F run, double *ms, uint64_t &launches) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return false;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return false;
    }
    auto timed = [&](int k, int warm, int reps) {
        for (int r = 0; r < warm; r++) launches += run(k);
        cudaEventRecord(e0, stream);
        for (int r = 0; r < reps; r++) launches += run(k);
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        return (double)t / reps;
    };
    double best = 1e300;
    for (int k = 0; k < n; k++) {
        ms[k] = timed(k, 1, 3);
        best = std::min(best, ms[k]);
    }
    if (best >= kSustainMinMs) {
        std::vector<std::vector<double>> w(n);
        for (int round = 0; round < kSustainRounds; round++)
            for (int i = 0; i < n; i++) {
                const int k = round % 2 == 0 ? i : n - 1 - i;
                const int half = std::max(4, (int)(0.5 * kSustainWindowMs / std::max(ms[k], 1e-3)));
                w[k].push_back(timed(k, half, half));
            }
        for (int k = 0; k < n; k++) {
            std::sort(w[k].begin(), w[k].end());
            ms[k] = 0.5 * (w[k][(kSustainRounds - 1) / 2] + w[k][kSustainRounds / 2]);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return true;
}

// Candidate group sizes (mode blocks) of the grouped fused step; 0 = whole batch.
constexpr int kGroupCandidates[] = {0, 1, 2, 4, 8};

// Times the grouped step pattern (psimid -> aux_dst -> aux_src: the state is
// not touched) for each candidate group size and keeps the fastest.
int autotune_groups(ovl_ctx *c) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return fail(c, OVL_E_CUDA, "autotune: events");
    const size_t bytes = c->field_complex * c->elem_bytes;
    cudaMemsetAsync(c->aux_src, 0, bytes, c->stream);
    cudaMemsetAsync(c->aux_dst, 0, bytes, c->stream);
    if (fp40(c)) {
        cudaMemsetAsync(c->aux_src_lo, 0, c->field_complex * 2, c->stream);
        cudaMemsetAsync(c->aux_dst_lo, 0, c->field_complex * 2, c->stream);
    }
    const ovl::HopConfig h = hop_config(c);
    double best = 1e300;
    int pick = 0;
    for (int G : kGroupCandidates) {
        if (G >= c->n_mb) continue;
        float total = 0.0f;
        for (int rep = 0; rep < 4; rep++) {
            cudaEventRecord(e0, c->stream);
            grouped_pass(c, h, h, c->psimid, c->aux_dst, c->aux_dst, c->aux_src, G);
            cudaEventRecord(e1, c->stream);
            cudaEventSynchronize(e1);
            float t = 0.0f;
            cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0) total += t;
        }
        if (total < best) { best = total; pick = G; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->mode_group = pick;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? OVL_OK : cuda_fail(c, e, "autotune (groups)");
}

// Times each hop-kernel variant on the live fields (psi -> operator buffer,
// the context's state is not touched) and keeps the fastest.
static_assert(ovl::kHopVariants == OVL_HOP_VARIANTS, "hop variant count of the header");

int autotune(ovl_ctx *c, double ms_out[ovl::kHopVariants]) {
    ovl::HopConfig h = hop_config(c);
    // the packed kernel is FP32 only
    const int nv = fp40(c) ? ovl::kFp40Variants : (fp32(c) ? ovl::kHopVariants : ovl::kPackedVariant);
    if (fp40(c)) cudaMemsetAsync(c->aux_dst_lo, 0, c->field_complex * 2, c->stream);
    double ms[ovl::kHopVariants] = {0.0, 0.0, 0.0, 0.0};
    uint64_t nl = 0;
    auto run = [&](int v) {
        h.variant = v;
        if (fp40(c))
            ovl::launch_wilson40(h, c->psi, c->psi_lo, c->aux_dst, c->aux_dst_lo, c->L, 0, c->n_mb, amass(c->p),
                                 c->p.dt, true, c->stream);
        else if (fp32(c)) ovl::launch_wilson_tuned<float>(h, c->psi, c->aux_dst, c->L, 0, c->n_mb, amass(c->p), c->p.dt, true, c->stream);
        else ovl::launch_wilson_tuned<double>(h, c->psi, c->aux_dst, c->L, 0, c->n_mb, amass(c->p), c->p.dt, true, c->stream);
        return 1;
    };
    if (!time_candidates(c->stream, nv, run, ms, nl)) return fail(c, OVL_E_CUDA, "autotune: events");
    int pick = 0;
    for (int v = 1; v < nv; v++)
        if (ms[v] < ms[pick]) pick = v;
    if (ms_out)
        for (int v = 0; v < ovl::kHopVariants; v++) ms_out[v] = ms[v];
    c->hop_variant = pick;
    int rc = launched(c, (int)nl, "autotune");
    if (!rc && c->mode_group < 0) rc = autotune_groups(c);
    return rc;
}

// Three colours, FP32: the scalar stencil (variant 0) against the packed-pair
// stencil (variant 3), timed on the operator buffer as the context uses the
// stencil (the fused half step for Wilson contexts; for overlap contexts a
// Chebyshev series of degree 3, whose D passes and final combination differ
// between the variants); the state is not touched.
int su3_autotune(ovl_ctx *c, double ms_out[ovl::kHopVariants]) {
    if (ms_out)
        for (int v = 0; v < ovl::kHopVariants; v++) ms_out[v] = 0.0;
    if (!fp32(c)) {
        c->hop_variant = 0;
        return OVL_OK;
    }
    const int cand[2] = {0, ovl::kPackedVariant};
    double ms[2] = {0.0, 0.0};
    uint64_t nl = 0;
    ovl::Su3Links lk = su3_links(c);
    const bool cheb = overlap(c) && c->p.sign_method == OVL_SIGN_CHEBYSHEV;
    if (cheb) {
        cudaMemsetAsync(c->cw.b1, 0, c->field_complex * c->elem_bytes, c->stream);
        cudaMemsetAsync(c->cw.b2, 0, c->field_complex * c->elem_bytes, c->stream);
    }
    const double lmax = std::pow(0.5 * std::fabs(amass(c->p)) + 3.0, 2);
    auto run = [&](int k) -> uint64_t {
        lk.variant = cand[k];
        if (cheb) {  // a Chebyshev series of degree 3 (four terms and the combination), psi -> aux_dst
            uint64_t n = 0;
            ovl::su3_chebyshev_apply<float>(c->cw, lk, c->psi, c->aux_dst, c->L, c->n_mb, c->cheb.data(),
                                            std::min(3, c->p.cheb_degree), c->p.cheb_eps, lmax, amass(c->p), c->p.m_dw,
                                            c->p.m_fermion, c->p.dt, false, c->sm_count, c->stream, &n);
            return n;
        }
        const bool acc = !overlap(c);
        ovl::su3_launch_hop<float>(lk, c->psi, c->aux_dst, c->L, 0, c->n_mb, amass(c->p), acc ? c->p.dt : 0.0, acc,
                                   c->stream);
        return 1;
    };
    if (!time_candidates(c->stream, 2, run, ms, nl)) return fail(c, OVL_E_CUDA, "autotune: events");
    c->hop_variant = ms[1] < ms[0] ? cand[1] : cand[0];
    if (ms_out) {
        ms_out[0] = ms[0];
        ms_out[ovl::kPackedVariant] = ms[1];
    }
    return launched(c, (int)nl, "autotune (three colours)");
}

// The three-colour half step: fused (dst += dt D src in one pass) or plain
// (D src into the derivative buffer chunk by chunk, then the axpy).
int su3_half_step(ovl_ctx *c, const void *src, void *dst) {
    if (c->hop_variant < 0) {
        int rc = su3_autotune(c, nullptr);
        if (rc) return rc;
    }
    const ovl::Su3Links lk = su3_links(c);
    const Lattice &L = c->L;
    if (c->p.form == OVL_FORM_FUSED) {
        ProfScope ps(c, OVL_PROF_HOP);
        if (fp32(c)) ovl::su3_launch_hop<float>(lk, src, dst, L, 0, c->n_mb, amass(c->p), c->p.dt, true, c->stream);
        else ovl::su3_launch_hop<double>(lk, src, dst, L, 0, c->n_mb, amass(c->p), c->p.dt, true, c->stream);
        return launched(c, 1, "wilson (fused, three colours)");
    }
    const size_t block_complex = (size_t)L.V * c->comp * ovl::kModeBlock;
    int n = 0;
    for (int mb = 0; mb < c->n_mb; mb += c->deriv_mb) {
        const int nmb = std::min(c->deriv_mb, c->n_mb - mb);
        char *d = static_cast<char *>(dst) + block_complex * c->elem_bytes * (size_t)mb;
        {
            ProfScope ps(c, OVL_PROF_HOP);
            if (fp32(c)) ovl::su3_launch_hop<float>(lk, src, c->deriv, L, mb, nmb, amass(c->p), 0.0, false, c->stream);
            else ovl::su3_launch_hop<double>(lk, src, c->deriv, L, mb, nmb, amass(c->p), 0.0, false, c->stream);
        }
        {
            ProfScope ps(c, OVL_PROF_AXPY);
            if (fp32(c)) ovl::launch_axpy<float>(d, c->deriv, block_complex * nmb, c->p.dt, c->sm_count, c->stream);
            else ovl::launch_axpy<double>(d, c->deriv, block_complex * nmb, c->p.dt, c->sm_count, c->stream);
        }
        n += 2;
    }
    return launched(c, n, "wilson (plain, three colours)");
}

// psi_dst += dt * D psi_src over all modes (one Update.cpp half step).
int half_step(ovl_ctx *c, const void *src, void *dst) {
    const Lattice &L = c->L;
    if (overlap(c)) return run_overlap(c, src, dst, c->n_mb, c->p.n_modes, true, true);
    if (su3(c)) return su3_half_step(c, src, dst);
    if (c->hop_variant < 0) {
        int rc = autotune(c, nullptr);
        if (rc) return rc;
    }
    const ovl::HopConfig hc = hop_config(c);
    if (c->p.form == OVL_FORM_FUSED) {
        ProfScope ps(c, OVL_PROF_HOP);
        if (fp40(c))
            ovl::launch_wilson40(hc, src, lo_of(c, src), dst, lo_of(c, dst), L, 0, c->n_mb, amass(c->p), c->p.dt, true,
                                 c->stream);
        else if (fp32(c)) ovl::launch_wilson_tuned<float>(hc, src, dst, L, 0, c->n_mb, amass(c->p), c->p.dt, true, c->stream);
        else ovl::launch_wilson_tuned<double>(hc, src, dst, L, 0, c->n_mb, amass(c->p), c->p.dt, true, c->stream);
        return launched(c, 1, "wilson (fused)");
    }
    const size_t block_complex = (size_t)L.V * ovl::kComp * ovl::kModeBlock;
    int n = 0;
    for (int mb = 0; mb < c->n_mb; mb += c->deriv_mb) {
        const int nmb = std::min(c->deriv_mb, c->n_mb - mb);
        char *d = static_cast<char *>(dst) + block_complex * c->elem_bytes * (size_t)mb;
        {
            ProfScope ps(c, OVL_PROF_HOP);
            if (fp32(c)) ovl::launch_wilson_tuned<float>(hc, src, c->deriv, L, mb, nmb, amass(c->p), c->p.dt, false, c->stream);
            else ovl::launch_wilson_tuned<double>(hc, src, c->deriv, L, mb, nmb, amass(c->p), c->p.dt, false, c->stream);
        }
        {
            ProfScope ps(c, OVL_PROF_AXPY);
            if (fp32(c)) ovl::launch_axpy<float>(d, c->deriv, block_complex * nmb, c->p.dt, c->sm_count, c->stream);
            else ovl::launch_axpy<double>(d, c->deriv, block_complex * nmb, c->p.dt, c->sm_count, c->stream);
        }
        n += 2;
    }
    return launched(c, n, "wilson (plain)");
}

int run_currents(ovl_ctx *c) {
    if (overlap(c)) {
        // ComputeCurrents recomputes the bounds and applies h_ov to every mode
        // (OverlapCurrents.cpp:106-117)
        int rc = run_overlap(c, c->psi, c->aux_dst, c->n_mb, c->p.n_modes, false, true);
        if (rc) return rc;
        ProfScope ps(c, OVL_PROF_OBS);
        ovl::launch_overlap_currents(c->psi, c->aux_dst, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->partial,
                                     c->per_site, c->stream, fp32(c), c->nc);
        return launched(c, 2, "overlap currents");
    }
    if (su3(c)) {
        ProfScope ps(c, OVL_PROF_OBS);
        if (fp32(c))
            ovl::su3_launch_currents<float>(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->L, c->n_mb, c->p.n_modes,
                                            c->p.first_mode, c->p.r_wilson, c->partial, c->per_site, c->stream);
        else
            ovl::su3_launch_currents<double>(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->L, c->n_mb, c->p.n_modes,
                                             c->p.first_mode, c->p.r_wilson, c->partial, c->per_site, c->stream);
        return launched(c, 2, "currents (three colours)");
    }
    ProfScope ps(c, OVL_PROF_OBS);
    if (fp40(c))
        ovl::launch_currents40(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->psi_lo, c->L, c->n_mb, c->p.n_modes,
                               c->p.first_mode, c->p.r_wilson, c->partial, c->per_site, c->stream);
    else if (fp32(c))
        ovl::launch_currents<float>(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->p.r_wilson,
                                    c->partial, c->per_site, c->stream);
    else
        ovl::launch_currents<double>(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->p.r_wilson,
                                     c->partial, c->per_site, c->stream);
    return launched(c, 2, "currents");
}

}  // namespace

extern "C" {

int ovl_abi_version(void) { return OVL_ABI_VERSION; }

int ovl_params_init(ovl_params *p) {
    if (!p) return OVL_E_ARG;
    std::memset(p, 0, sizeof *p);
    p->N[0] = p->N[1] = p->N[2] = 8;
    p->n_colours = 2;
    p->n_modes = 4 * 2 * 8 * 8 * 8;
    p->first_mode = 0;
    p->fermion = OVL_FERMION_WILSON;
    p->precision = OVL_PREC_FP64;
    p->form = OVL_FORM_PLAIN;
    p->r_wilson = 1.0;
    p->m_fermion = 0.0;
    p->m_dw = 1.4;
    p->dt = 0.02;
    p->qs = 1.0;
    p->t_sphaleron = 6.0;
    p->device = 0;
    p->plain_chunk_modes = 0;
    p->stream = 0;
    p->zolo_poles = 25;
    p->zolo_tol = 1e-12;
    p->cg_max_iter = 1000;
    p->cg_tol = 1e-16;
    p->hop_variant = -1;
    p->reunitarize = 0;
    p->gauge_force = 0;
    p->backreaction = 0.0;
    p->ritz_auto = 0;
    p->ritz_seed = 0;
    p->mode_group = 0;
    p->sign_method = OVL_SIGN_ZOLOTAREV;
    p->cheb_degree = 96;
    p->cheb_eps = 0.01;
    return OVL_OK;
}

int ovl_create(const ovl_params *p, ovl_ctx **out) {
    if (!p || !out) return fail(nullptr, OVL_E_ARG, "ovl_create: null argument");
    *out = nullptr;
    for (int i = 0; i < 3; i++)
        if (p->N[i] < 3 || p->N[i] > 1024) return fail(nullptr, OVL_E_ARG, "ovl_create: N[%d]=%d outside [3, 1024]", i, p->N[i]);
    if (p->n_colours != 2 && p->n_colours != 3)
        return fail(nullptr, OVL_E_UNSUPPORTED, "ovl_create: n_colours=%d (2 or 3)", p->n_colours);
    if (p->n_colours == 3) {
        if (p->fermion == OVL_FERMION_OVERLAP && p->sign_method != OVL_SIGN_CHEBYSHEV)
            return fail(nullptr, OVL_E_UNSUPPORTED, "ovl_create: three-colour overlap fermions use the Chebyshev sign function");
        if (p->precision == OVL_PREC_FP40)
            return fail(nullptr, OVL_E_UNSUPPORTED, "ovl_create: FP40 storage is built for two colours");
    }
    if (p->fermion != OVL_FERMION_WILSON && p->fermion != OVL_FERMION_OVERLAP)
        return fail(nullptr, OVL_E_ARG, "ovl_create: fermion kind %d", p->fermion);
    if (p->fermion == OVL_FERMION_OVERLAP && p->sign_method != OVL_SIGN_ZOLOTAREV && p->sign_method != OVL_SIGN_CHEBYSHEV)
        return fail(nullptr, OVL_E_ARG, "ovl_create: sign_method=%d", p->sign_method);
    if (p->fermion == OVL_FERMION_OVERLAP && p->sign_method == OVL_SIGN_ZOLOTAREV && p->precision != OVL_PREC_FP64)
        return fail(nullptr, OVL_E_UNSUPPORTED, "ovl_create: the Zolotarev overlap operator is built in FP64 only");
    if (p->fermion == OVL_FERMION_OVERLAP && p->sign_method == OVL_SIGN_CHEBYSHEV &&
        (p->cheb_degree < 1 || p->cheb_degree > ovl::kMaxChebDegree || !(p->cheb_eps > 0.0) || !(p->cheb_eps < 1.0)))
        return fail(nullptr, OVL_E_ARG, "ovl_create: cheb_degree=%d (1..%d), cheb_eps=%g (0..1)", p->cheb_degree,
                    ovl::kMaxChebDegree, p->cheb_eps);
    if (p->fermion == OVL_FERMION_OVERLAP && (p->zolo_poles < 1 || p->zolo_poles > ovl::kMaxPoles || p->cg_max_iter < 1))
        return fail(nullptr, OVL_E_ARG, "ovl_create: zolo_poles=%d (1..%d), cg_max_iter=%d", p->zolo_poles, ovl::kMaxPoles,
                    p->cg_max_iter);
    if (p->backreaction != 0.0 && p->fermion != OVL_FERMION_WILSON)
        return fail(nullptr, OVL_E_UNSUPPORTED, "ovl_create: fermion back-reaction is built for Wilson fermions only");
    if (!std::isfinite(p->backreaction)) return fail(nullptr, OVL_E_ARG, "ovl_create: backreaction must be finite");
    if (p->precision != OVL_PREC_FP64 && p->precision != OVL_PREC_FP32 && p->precision != OVL_PREC_FP40)
        return fail(nullptr, OVL_E_ARG, "ovl_create: bad precision");
    if (p->precision == OVL_PREC_FP40 && (p->fermion != OVL_FERMION_WILSON || p->form != OVL_FORM_FUSED))
        return fail(nullptr, OVL_E_UNSUPPORTED, "ovl_create: FP40 storage is built for the fused Wilson form");
    if (p->form != OVL_FORM_PLAIN && p->form != OVL_FORM_FUSED) return fail(nullptr, OVL_E_ARG, "ovl_create: bad form");
    if (p->n_modes <= 0 || p->first_mode < 0) return fail(nullptr, OVL_E_ARG, "ovl_create: n_modes=%d first_mode=%d", p->n_modes, p->first_mode);
    // mode blocks run along grid.y of the stencil launches (at most 65535)
    if ((p->n_modes + ovl::kModeBlock - 1) / ovl::kModeBlock > 65535)
        return fail(nullptr, OVL_E_ARG, "ovl_create: n_modes=%d above %d", p->n_modes, 65535 * ovl::kModeBlock);
    if (!(p->dt > 0.0) || !std::isfinite(p->dt)) return fail(nullptr, OVL_E_ARG, "ovl_create: dt must be positive");
    if (p->mode_group < -1) return fail(nullptr, OVL_E_ARG, "ovl_create: mode_group=%d", p->mode_group);
    if (p->hop_variant < -1 || p->hop_variant >= ovl::kHopVariants)
        return fail(nullptr, OVL_E_ARG, "ovl_create: hop_variant=%d (-1 = autotune, 0..%d)", p->hop_variant, ovl::kHopVariants - 1);
    if (p->hop_variant == ovl::kPackedVariant && p->precision != OVL_PREC_FP32)
        return fail(nullptr, OVL_E_ARG, "ovl_create: hop_variant=%d (packed pairs) needs FP32 modes", p->hop_variant);
    const long long V = (long long)p->N[0] * p->N[1] * p->N[2];
    if (V > (1LL << 30) / 8) return fail(nullptr, OVL_E_ARG, "ovl_create: lattice too large");

    ovl_ctx *c = new (std::nothrow) ovl_ctx();
    if (!c) return fail(nullptr, OVL_E_OOM, "ovl_create: host allocation failed");
    c->p = *p;
    c->nc = p->n_colours;
    c->comp = 4 * c->nc;
    c->link_doubles = c->nc == 3 ? 18 : 4;
    c->e_comp = c->nc == 3 ? 8 : 3;
    c->L = Lattice{p->N[0], p->N[1], p->N[2], (int)V};
    c->n_mb = (p->n_modes + ovl::kModeBlock - 1) / ovl::kModeBlock;
    c->elem_bytes = p->precision == OVL_PREC_FP64 ? 16 : 8;  // FP40: the 32-bit high words
    c->field_complex = (size_t)c->n_mb * V * c->comp * ovl::kModeBlock;
    const size_t n_link = (size_t)c->link_doubles * 3 * V, n_e = (size_t)c->e_comp * 3 * V;
    int rc = OVL_OK;
    auto bail = [&](int code) { g_err = c->err; ovl_destroy(c); return code; };
    if ((rc = set_device(c)) != OVL_OK) return bail(rc);
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, p->device);
    if (p->stream) {
        c->stream = reinterpret_cast<cudaStream_t>(p->stream);
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(c, OVL_E_CUDA, "ovl_create: stream creation failed"));
        c->own_stream = true;
    }
    const size_t field_bytes = c->field_complex * c->elem_bytes;
    auto alloc = [&](void **ptr, size_t bytes, const char *what) -> int {
        if (cudaMalloc(ptr, bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, OVL_E_OOM, "ovl_create: cannot allocate %zu bytes for %s", bytes, what);
        }
        return OVL_OK;
    };
    if (p->precision == OVL_PREC_FP40) {
        const size_t lo_bytes = c->field_complex * 2;
        if ((rc = alloc(&c->psi_lo, lo_bytes, "Psi extension bytes")) || (rc = alloc(&c->psimid_lo, lo_bytes, "PsiMid extension bytes")) ||
            (rc = alloc(&c->aux_src_lo, lo_bytes, "operator input extension")) ||
            (rc = alloc(&c->aux_dst_lo, lo_bytes, "operator output extension")))
            return bail(rc);
    }
    if ((rc = alloc(&c->psi, field_bytes, "Psi")) || (rc = alloc(&c->psimid, field_bytes, "PsiMid")) ||
        (rc = alloc((void **)&c->U, sizeof(double) * n_link, "links")) ||
        (rc = alloc((void **)&c->E, sizeof(double) * n_e, "efield")))
        return bail(rc);
    if (p->form == OVL_FORM_PLAIN) {
        int chunk = p->plain_chunk_modes > 0 ? p->plain_chunk_modes : p->n_modes;
        c->deriv_mb = std::min(c->n_mb, (chunk + ovl::kModeBlock - 1) / ovl::kModeBlock);
        if ((rc = alloc(&c->deriv, (size_t)c->deriv_mb * V * c->comp * ovl::kModeBlock * c->elem_bytes, "derivative buffer")))
            return bail(rc);
    }
    c->partial_doubles = std::max({ovl::currents_partial_doubles(c->L, c->n_mb), ovl::ncsdot_partial_doubles(c->L),
                                   ovl::bulk_partial_doubles(c->L), ovl::charges_partial_doubles(c->L, c->n_mb),
                                   ovl::force_partial_doubles(c->L, c->n_mb), ovl::energy_partial_doubles(),
                                   ovl::gauss_partial_doubles(c->L), ovl::su3_charges_partial_doubles(c->L, c->n_mb),
                                   ovl::su3_reduce_partial_doubles(c->L),
                                   ovl::su3_force_partial_doubles(c->L, c->n_mb)});
    if ((rc = alloc((void **)&c->partial, sizeof(double) * c->partial_doubles, "reduction scratch")) ||
        (rc = alloc((void **)&c->per_site, sizeof(double) * ovl::kCurrentsPerSite * V, "currents")) ||
        (rc = alloc((void **)&c->dev_small, sizeof(double) * 64, "results")) ||
        (rc = alloc((void **)&c->dev_int, sizeof(int) * 4, "flags")))
        return bail(rc);
    if (cudaMallocHost(&c->host_small, sizeof(double) * 64) != cudaSuccess)
        return bail(fail(c, OVL_E_OOM, "ovl_create: pinned host allocation failed"));
    if ((rc = alloc(&c->aux_src, field_bytes, "operator input")) || (rc = alloc(&c->aux_dst, field_bytes, "operator output")))
        return bail(rc);
    const size_t n_link32 = c->nc == 3 ? (size_t)ovl::kSu3Link32Floats * 3 * V : n_link;  // padded records
    if (p->precision == OVL_PREC_FP32 && (rc = alloc((void **)&c->U32, sizeof(float) * n_link32, "FP32 links")))
        return bail(rc);
    if (p->precision == OVL_PREC_FP32 && c->nc == 2 && p->fermion == OVL_FERMION_WILSON) {
        const size_t nb = sizeof(int) * ovl::pipeline_counters(c->n_mb);
        if ((rc = alloc((void **)&c->pipe, nb, "pipeline counters"))) return bail(rc);
        if (cudaMemset(c->pipe, 0, nb) != cudaSuccess) return bail(fail(c, OVL_E_CUDA, "ovl_create: counters"));
    }
    // three colours: the scalar stencil (0) or, FP32 only, the packed one (3); -1 tunes between them
    if (c->nc == 3)
        c->hop_variant = p->precision == OVL_PREC_FP32 && (p->hop_variant < 0 || p->hop_variant == ovl::kPackedVariant)
                             ? p->hop_variant
                             : 0;
    else
        c->hop_variant = p->hop_variant;
    // grouping applies to the fused two-colour Wilson form; fixed when the variant is fixed
    if (p->form != OVL_FORM_FUSED || p->fermion != OVL_FERMION_WILSON || c->nc == 3) c->mode_group = 0;
    else c->mode_group = p->mode_group;
    if (p->fermion == OVL_FERMION_OVERLAP && p->sign_method == OVL_SIGN_CHEBYSHEV) {
        ovl::ChebyshevWork &w = c->cw;
        if ((rc = alloc(&w.b0, field_bytes, "Clenshaw b")) || (rc = alloc(&w.b1, field_bytes, "Clenshaw b")) ||
            (rc = alloc(&w.b2, field_bytes, "Clenshaw b")) || (rc = alloc(&w.w, field_bytes, "Clenshaw temporary")))
            return bail(rc);
        c->cheb.assign(p->cheb_degree + 1, 0.0);
        ovl::chebyshev_inverse_sqrt(p->cheb_degree, p->cheb_eps, c->cheb.data());
    }
    if (p->fermion == OVL_FERMION_OVERLAP && p->sign_method == OVL_SIGN_ZOLOTAREV) {
        ovl::OverlapWork &w = c->ow;
        const size_t mp = (size_t)c->n_mb * ovl::kModeBlock, np = (size_t)p->zolo_poles;
        if ((rc = alloc(&w.r, field_bytes, "CG residual")) || (rc = alloc(&w.q, field_bytes, "CG direction image")) ||
            (rc = alloc(&w.t, field_bytes, "CG temporary")) || (rc = alloc(&w.x, field_bytes * np, "shifted solutions")) ||
            (rc = alloc(&w.p, field_bytes * np, "shifted directions")) ||
            (rc = alloc((void **)&w.part, sizeof(double) * ovl::kDotChunks * mp, "dot partials")) ||
            (rc = alloc((void **)&w.rnorm, sizeof(double) * mp * 5, "CG scalars")) ||
            (rc = alloc((void **)&w.alpha, sizeof(double) * mp * np * 4, "shift scalars")) ||
            (rc = alloc((void **)&w.active, sizeof(int) * (mp * 3 + 1), "CG flags")) ||
            (rc = alloc((void **)&w.dz, sizeof(double) * 2 * ovl::kMaxPoles, "Zolotarev coefficients")))
            return bail(rc);
        w.bnorm = w.rnorm + mp; w.betam = w.rnorm + 2 * mp; w.pap = w.rnorm + 3 * mp; w.rr = w.rnorm + 4 * mp;
        w.beta = w.alpha + mp * np; w.z = w.alpha + 2 * mp * np; w.g = w.alpha + 3 * mp * np;
        w.next = w.active + mp; w.iters = w.active + 2 * mp; w.count = w.active + 3 * mp;
        w.bz = w.dz + ovl::kMaxPoles;
        if (cudaMallocHost(&w.host_count, sizeof(int)) != cudaSuccess)
            return bail(fail(c, OVL_E_OOM, "ovl_create: pinned host allocation failed"));
    }
    cudaMemsetAsync(c->psi, 0, field_bytes, c->stream);
    cudaMemsetAsync(c->psimid, 0, field_bytes, c->stream);
    cudaMemsetAsync(c->E, 0, sizeof(double) * n_e, c->stream);
    // links start at the identity (GaugeLinks::SetIdentity)
    std::vector<double> unit(n_link, 0.0);
    for (long long l = 0; l < 3 * V; l++) {
        if (c->nc == 3) unit[18 * l] = unit[18 * l + 8] = unit[18 * l + 16] = 1.0;  // U_ii at 2 (i + 3 i)
        else unit[4 * l + 3] = 1.0;
    }
    cudaMemcpyAsync(c->U, unit.data(), sizeof(double) * n_link, cudaMemcpyHostToDevice, c->stream);
    refresh_links32(c);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(c, OVL_E_CUDA, "ovl_create: initialisation failed"));
    *out = c;
    return OVL_OK;
}

int ovl_destroy(ovl_ctx *c) {
    if (!c) return OVL_OK;
    cudaSetDevice(c->p.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void *bufs[] = {c->psi, c->psimid, c->U, c->E, c->deriv, c->per_site, c->partial, c->dev_small, c->dev_int,
                    c->aux_src, c->aux_dst, c->ow.r, c->ow.q, c->ow.t, c->ow.x, c->ow.p, c->ow.part, c->ow.rnorm,
                    c->ow.alpha, c->ow.active, c->ow.dz, c->u_old, c->u_mid, c->e_mid, c->u1,
                    c->cw.b0, c->cw.b1, c->cw.b2, c->cw.w, c->U32, c->u1_32, c->U_b, c->U32_b,
                    c->psi_lo, c->psimid_lo, c->aux_src_lo, c->aux_dst_lo, c->obs_partial, c->obs_scratch, c->pipe};
    if (c->ow.host_count) cudaFreeHost(c->ow.host_count);
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (c->host_small) cudaFreeHost(c->host_small);
    ovl::ritz_destroy(c->ritz);
    for (auto &v : c->prof)
        for (auto &pr : v) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return OVL_OK;
}

const char *ovl_last_error(const ovl_ctx *c) { return c ? c->err.c_str() : g_err.c_str(); }

int ovl_set_links(ovl_ctx *c, const double *links) {
    if (!c || !links) return fail(c, OVL_E_ARG, "ovl_set_links: null argument");
    const size_t n = (size_t)c->link_doubles * 3 * c->L.V;
    if (!all_finite(links, n)) return fail(c, OVL_E_NONFINITE, "ovl_set_links: non-finite link component");
    int rc = set_device(c);
    if (rc) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(c->U, links, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    refresh_links32(c);
    if (page_locked(links)) OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    return OVL_OK;
}

int ovl_get_links(ovl_ctx *c, double *links) {
    if (!c || !links) return fail(c, OVL_E_ARG, "ovl_get_links: null argument");
    int rc = set_device(c);
    if (rc) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(links, c->U, sizeof(double) * c->link_doubles * 3 * c->L.V, cudaMemcpyDeviceToHost,
                                c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    return OVL_OK;
}

int ovl_set_efield(ovl_ctx *c, const double *efield) {
    if (!c || !efield) return fail(c, OVL_E_ARG, "ovl_set_efield: null argument");
    const size_t n = (size_t)c->e_comp * 3 * c->L.V;
    if (!all_finite(efield, n)) return fail(c, OVL_E_NONFINITE, "ovl_set_efield: non-finite field component");
    int rc = set_device(c);
    if (rc) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(c->E, efield, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    if (page_locked(efield)) OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    return OVL_OK;
}

int ovl_upload_gauge_async(ovl_ctx *c, const double *links, const double *efield) {
    if (!c) return OVL_E_ARG;
    if ((links && !page_locked(links)) || (efield && !page_locked(efield)))
        return fail(c, OVL_E_ARG, "ovl_upload_gauge_async: the fields must be page-locked host memory");
    const size_t nl = (size_t)c->link_doubles * 3 * c->L.V, ne = (size_t)c->e_comp * 3 * c->L.V;
    if (links && !all_finite(links, nl)) return fail(c, OVL_E_NONFINITE, "ovl_upload_gauge_async: non-finite link component");
    if (efield && !all_finite(efield, ne))
        return fail(c, OVL_E_NONFINITE, "ovl_upload_gauge_async: non-finite field component");
    int rc = set_device(c);
    if (rc) return rc;
    if (links) {
        OVL_CUDA(c, cudaMemcpyAsync(c->U, links, sizeof(double) * nl, cudaMemcpyHostToDevice, c->stream));
        refresh_links32(c);
    }
    if (efield) OVL_CUDA(c, cudaMemcpyAsync(c->E, efield, sizeof(double) * ne, cudaMemcpyHostToDevice, c->stream));
    return OVL_OK;
}

int ovl_set_u1(ovl_ctx *c, const double *u1) {
    if (!c) return OVL_E_ARG;
    if (!u1) {
        c->u1_on = false;
        return OVL_OK;
    }
    const size_t n = (size_t)4 * c->L.N0 * c->L.N1;
    if (!all_finite(u1, n)) return fail(c, OVL_E_NONFINITE, "ovl_set_u1: non-finite phase");
    int rc = set_device(c);
    if (rc) return rc;
    if (!c->u1 && cudaMalloc(&c->u1, sizeof(double) * n) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, OVL_E_OOM, "ovl_set_u1: phases");
    }
    OVL_CUDA(c, cudaMemcpyAsync(c->u1, u1, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    if (fp32(c)) {
        if (!c->u1_32 && cudaMalloc(&c->u1_32, sizeof(float) * n) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, OVL_E_OOM, "ovl_set_u1: FP32 phases");
        }
        ovl::launch_links_to_f32(c->u1, c->u1_32, n, c->stream);
        c->launches++;
    }
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    c->u1_on = true;
    return OVL_OK;
}

int ovl_get_efield(ovl_ctx *c, double *efield) {
    if (!c || !efield) return fail(c, OVL_E_ARG, "ovl_get_efield: null argument");
    int rc = set_device(c);
    if (rc) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(efield, c->E, sizeof(double) * c->e_comp * 3 * c->L.V, cudaMemcpyDeviceToHost,
                                c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    return OVL_OK;
}

// ---------------------------------------------------------------------------
// Gauge configurations as text files in the reference's format
// (IO/SaveConfiguration.cpp:3-62, IO/LoadConfiguration.cpp:3-148): one line
// per link, z outermost, then y, x and the direction innermost.  Numbers are
// printed as the reference's streams print them at OUTPUT_PRECISION (the 15
// digits of std::numeric_limits<double>::digits10, default float format),
// which is printf's %.15g.

namespace {

struct FileCloser {
    void operator()(FILE *f) const {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<FILE, FileCloser>;

// Appends "%.15g" of v and the separator to a line buffer.
void put_number(std::string &line, double v, const char *sep_before, const char *sep_after) {
    char buf[40];
    std::snprintf(buf, sizeof buf, "%s%.15g%s", sep_before, v, sep_after);
    line += buf;
}

// Parses "x y z mu v_0 ... v_{n-1}" into the site/direction and n values;
// false when the line holds fewer numbers.  Extra numbers are ignored, as the
// reference's stream extraction ignores them.
bool parse_record(const char *line, int &x, int &y, int &z, int &mu, double *v, int n) {
    char *end = nullptr;
    const char *q = line;
    long coords[4];
    for (int k = 0; k < 4; k++) {
        coords[k] = std::strtol(q, &end, 10);
        if (end == q) return false;
        q = end;
    }
    x = (int)coords[0];
    y = (int)coords[1];
    z = (int)coords[2];
    mu = (int)coords[3];
    for (int k = 0; k < n; k++) {
        v[k] = std::strtod(q, &end);
        if (end == q) return false;
        q = end;
    }
    return true;
}

bool blank(const char *line) {
    for (const char *q = line; *q; q++)
        if (!std::isspace((unsigned char)*q)) return false;
    return true;
}

// Reads every record of `path` into dst[site][mu][n]; each link exactly once.
int read_records(ovl_ctx *c, const char *path, int n, std::vector<double> &dst, const char *what) {
    File f(std::fopen(path, "r"));
    if (!f) return fail(c, OVL_E_ARG, "ovl_load_configuration: cannot open %s file %s", what, path);
    const int V = c->L.V;
    dst.assign((size_t)n * 3 * V, 0.0);
    std::vector<unsigned char> seen((size_t)3 * V, 0);
    std::vector<char> line(64 + 64 * (size_t)n);
    std::vector<double> v(n);
    long records = 0, lineno = 0;
    while (std::fgets(line.data(), (int)line.size(), f.get())) {
        lineno++;
        const size_t len = std::strlen(line.data());
        if (len + 1 == line.size() && line[len - 1] != '\n')
            return fail(c, OVL_E_ARG, "ovl_load_configuration: %s file %s line %ld too long", what, path, lineno);
        if (blank(line.data())) continue;
        int x, y, z, mu;
        if (!parse_record(line.data(), x, y, z, mu, v.data(), n))
            return fail(c, OVL_E_ARG, "ovl_load_configuration: %s file %s line %ld: expected x y z mu and %d numbers",
                        what, path, lineno, n);
        if (x < 0 || x >= c->L.N0 || y < 0 || y >= c->L.N1 || z < 0 || z >= c->L.N2 || mu < 0 || mu > 2)
            return fail(c, OVL_E_ARG, "ovl_load_configuration: %s file %s line %ld: link (%d %d %d %d) outside %dx%dx%d",
                        what, path, lineno, x, y, z, mu, c->L.N0, c->L.N1, c->L.N2);
        const size_t link = 3 * ((size_t)x + (size_t)c->L.N0 * ((size_t)y + (size_t)c->L.N1 * z)) + mu;
        if (seen[link]++)
            return fail(c, OVL_E_ARG, "ovl_load_configuration: %s file %s line %ld: link (%d %d %d %d) given twice", what,
                        path, lineno, x, y, z, mu);
        std::memcpy(&dst[link * n], v.data(), sizeof(double) * n);
        records++;
    }
    if (records != 3L * V)
        return fail(c, OVL_E_ARG, "ovl_load_configuration: %s file %s holds %ld links, the lattice %ld", what, path,
                    records, 3L * V);
    return OVL_OK;
}

}  // namespace

int ovl_save_configuration(ovl_ctx *c, const char *u_path, const char *e_path) {
    if (!c) return OVL_E_ARG;
    const int V = c->L.V;
    std::vector<double> U, E;
    int rc;
    if (u_path) {
        U.resize((size_t)c->link_doubles * 3 * V);
        if ((rc = ovl_get_links(c, U.data()))) return rc;
    }
    if (e_path) {
        E.resize((size_t)c->e_comp * 3 * V);
        if ((rc = ovl_get_efield(c, E.data()))) return rc;
    }
    File fu(u_path ? std::fopen(u_path, "w") : nullptr), fe(e_path ? std::fopen(e_path, "w") : nullptr);
    if (u_path && !fu) return fail(c, OVL_E_ARG, "ovl_save_configuration: cannot write %s", u_path);
    if (e_path && !fe) return fail(c, OVL_E_ARG, "ovl_save_configuration: cannot write %s", e_path);
    std::string line;
    for (int z = 0; z < c->L.N2; z++)
        for (int y = 0; y < c->L.N1; y++)
            for (int x = 0; x < c->L.N0; x++)
                for (int mu = 0; mu < 3; mu++) {
                    const size_t link = 3 * ((size_t)x + (size_t)c->L.N0 * ((size_t)y + (size_t)c->L.N1 * z)) + mu;
                    char head[64];
                    std::snprintf(head, sizeof head, "%d %d %d %d", x, y, z, mu);
                    if (fu) {
                        // SUNcGroup::IO::MatrixToString: every number followed by a space
                        line = head;
                        line += ' ';
                        const double *u = &U[link * c->link_doubles];
                        for (int k = 0; k < c->link_doubles; k++) put_number(line, u[k], "", " ");
                        line += '\n';
                        std::fputs(line.c_str(), fu.get());
                    }
                    if (fe) {
                        line = head;
                        const double *e = &E[link * c->e_comp];
                        for (int a = 0; a < c->e_comp; a++) put_number(line, e[a], " ", "");
                        line += '\n';
                        std::fputs(line.c_str(), fe.get());
                    }
                }
    if ((fu && std::ferror(fu.get())) || (fe && std::ferror(fe.get())))
        return fail(c, OVL_E_ARG, "ovl_save_configuration: write error");
    if ((fu && std::fclose(fu.release()) != 0) || (fe && std::fclose(fe.release()) != 0))
        return fail(c, OVL_E_ARG, "ovl_save_configuration: write error on close");
    return OVL_OK;
}

int ovl_load_configuration(ovl_ctx *c, const char *u_path, const char *e_path) {
    if (!c) return OVL_E_ARG;
    std::vector<double> U, E;
    int rc;
    // both files are read and checked before either field changes
    if (u_path && (rc = read_records(c, u_path, c->link_doubles, U, "link"))) return rc;
    if (e_path && (rc = read_records(c, e_path, c->e_comp, E, "electric field"))) return rc;
    if (u_path && (rc = ovl_set_links(c, U.data()))) return rc;
    if (e_path && (rc = ovl_set_efield(c, E.data()))) return rc;
    return OVL_OK;
}

// Modes move through a device staging buffer in the reference layout, in
// chunks that bound the staging memory.
static int transfer_modes(ovl_ctx *c, int first, int count, const double *hpsi, const double *hmid, double *opsi,
                          double *omid, bool upload) {
    if (!c) return OVL_E_ARG;
    if (first < 0 || count < 0 || first + count > c->p.n_modes)
        return fail(c, OVL_E_ARG, "modes [%d, %d) outside [0, %d)", first, first + count, c->p.n_modes);
    if (count == 0) return OVL_OK;
    int rc = set_device(c);
    if (rc) return rc;
    const size_t per_mode = (size_t)c->L.V * c->comp * 2;  // doubles
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)count, ((size_t)256 << 20) / (per_mode * 8)));
    double *stage = nullptr;
    if (cudaMalloc(&stage, per_mode * 8 * chunk) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, OVL_E_OOM, "mode staging buffer (%zu bytes)", per_mode * 8 * chunk);
    }
    int status = OVL_OK;
    for (int f = 0; f < 2 && status == OVL_OK; f++) {
        const double *hin = f == 0 ? hpsi : hmid;
        double *hout = f == 0 ? opsi : omid;
        void *field = f == 0 ? c->psi : c->psimid;
        if (upload ? !hin : !hout) continue;
        for (int m = first; m < first + count && status == OVL_OK; m += chunk) {
            const int n = std::min(chunk, first + count - m);
            const size_t off = per_mode * (size_t)(m - first);
            if (upload) {
                cudaError_t e = cudaMemcpyAsync(stage, hin + off, per_mode * 8 * n, cudaMemcpyHostToDevice, c->stream);
                if (e != cudaSuccess) { status = cuda_fail(c, e, "mode upload"); break; }
                if (fp32(c)) ovl::launch_ref_to_blocks<float>(stage, field, c->L, m, n, c->stream, nullptr, c->nc);
                else ovl::launch_ref_to_blocks<double>(stage, field, c->L, m, n, c->stream, lo_of(c, field), c->nc);
                status = launched(c, 1, "ref_to_blocks");
            } else {
                if (fp32(c)) ovl::launch_blocks_to_ref<float>(field, stage, c->L, m, n, c->stream, nullptr, c->nc);
                else ovl::launch_blocks_to_ref<double>(field, stage, c->L, m, n, c->stream, lo_of(c, field), c->nc);
                status = launched(c, 1, "blocks_to_ref");
                if (status) break;
                cudaError_t e = cudaMemcpyAsync(hout + off, stage, per_mode * 8 * n, cudaMemcpyDeviceToHost, c->stream);
                if (e != cudaSuccess) { status = cuda_fail(c, e, "mode download"); break; }
            }
            cudaError_t e = cudaStreamSynchronize(c->stream);
            if (e != cudaSuccess) status = cuda_fail(c, e, "mode transfer");
        }
    }
    cudaFree(stage);
    return status;
}

int ovl_set_modes(ovl_ctx *c, int first, int count, const double *psi, const double *psimid) {
    if (!c) return OVL_E_ARG;
    return transfer_modes(c, first, count, psi, psimid, nullptr, nullptr, true);
}

int ovl_get_modes(ovl_ctx *c, int first, int count, double *psi, double *psimid) {
    if (!c) return OVL_E_ARG;
    return transfer_modes(c, first, count, nullptr, nullptr, psi, psimid, false);
}

int ovl_set_stochastic_modes(ovl_ctx *c, uint64_t seed, int total_pairs) {
    if (!c) return OVL_E_ARG;
    if (c->p.fermion != OVL_FERMION_WILSON) return fail(c, OVL_E_UNSUPPORTED, "ovl_set_stochastic_modes: Wilson fermions only");
    if (total_pairs < 0) return fail(c, OVL_E_ARG, "ovl_set_stochastic_modes: total_pairs=%d", total_pairs);
    if (total_pairs == 0) {
        if ((c->p.first_mode | c->p.n_modes) & 1)
            return fail(c, OVL_E_ARG, "ovl_set_stochastic_modes: pairs need an even first_mode and n_modes");
        total_pairs = c->p.n_modes / 2;
    }
    int rc = set_device(c);
    if (rc) return rc;
    const int chunk = std::min(c->n_mb, 64);
    const size_t bytes = sizeof(double) * 2 * (size_t)chunk * c->L.V * c->comp * ovl::kModeBlock;
    // stream-ordered scratch: its release does not wait for the other streams
    // of the device (a cudaFree would), so a context set up beside running
    // ones does not stall them
    double *a = nullptr, *b = nullptr;
    if (cudaMallocAsync(&a, bytes, c->stream) != cudaSuccess || cudaMallocAsync(&b, bytes, c->stream) != cudaSuccess) {
        cudaGetLastError();
        if (a) cudaFreeAsync(a, c->stream);
        cudaStreamSynchronize(c->stream);
        return fail(c, OVL_E_OOM, "ovl_set_stochastic_modes: scratch");
    }
    const int kind = fp40(c) ? 2 : fp32(c) ? 1 : 0;
    uint64_t nl = 0;
    ovl::launch_stochastic_modes(c->psi, c->psimid, c->psi_lo, c->psimid_lo, kind, c->L, c->n_mb, c->p.n_modes,
                                 c->p.first_mode, amass(c->p), c->p.dt, seed, total_pairs, a, b, chunk, c->stream, &nl,
                                 c->nc);
    rc = launched(c, (int)nl, "stochastic modes");
    cudaFreeAsync(a, c->stream);
    cudaFreeAsync(b, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(c, e, "ovl_set_stochastic_modes");
    return OVL_OK;
}

int ovl_set_free_fermions(ovl_ctx *c, int *n_bad) {
    if (!c) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    if (fp32(c))
        ovl::launch_free_fermions<float>(c->psi, c->psimid, c->L, c->p.n_modes, c->n_mb, c->p.first_mode, c->p.r_wilson,
                                         c->p.m_fermion, c->p.dt, c->dev_int, c->stream, nullptr, nullptr, c->nc,
                                         overlap(c), c->p.m_dw);
    else  // FP64, or FP40 (the extension arrays set)
        ovl::launch_free_fermions<double>(c->psi, c->psimid, c->L, c->p.n_modes, c->n_mb, c->p.first_mode, c->p.r_wilson,
                                          c->p.m_fermion, c->p.dt, c->dev_int, c->stream, c->psi_lo, c->psimid_lo,
                                          c->nc, overlap(c), c->p.m_dw);
    if ((rc = launched(c, 2, "free fermions"))) return rc;
    int bad = 0;
    OVL_CUDA(c, cudaMemcpyAsync(&bad, c->dev_int, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (n_bad) *n_bad = bad;
    return OVL_OK;
}

// The fermion force dH_F/dtheta into out (8 or 3 per link), or E += coef * it.
void launch_force(ovl_ctx *c, double *out, double *E, double coef) {
    const double *u1 = c->u1_on ? c->u1 : nullptr;
    if (su3(c) && fp32(c))
        ovl::su3_launch_color_force<float>(c->U, u1, c->psi, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->partial,
                                           out, E, coef, c->stream);
    else if (su3(c))
        ovl::su3_launch_color_force<double>(c->U, u1, c->psi, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->partial,
                                            out, E, coef, c->stream);
    else if (fp40(c))
        ovl::launch_color_force40(c->U, u1, c->psi, c->psi_lo, c->L, c->n_mb, c->p.n_modes, c->p.first_mode,
                                  c->partial, out, E, coef, c->stream);
    else if (fp32(c))
        ovl::launch_color_force<float>(c->U, u1, c->psi, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->partial, out,
                                       E, coef, c->stream);
    else
        ovl::launch_color_force<double>(c->U, u1, c->psi, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->partial,
                                        out, E, coef, c->stream);
}

// E += dt (staple force) + dt g^2 dH_F/dtheta after a step of the coupled
// evolution (ovl_params.gauge_force, ovl_params.backreaction).
int coupled_efield(ovl_ctx *c) {
    if (c->p.gauge_force) {
        {
            ProfScope ps(c, OVL_PROF_LINKS);
            if (su3(c)) ovl::su3_launch_update_efield(c->U, c->E, c->L, c->p.dt, c->stream);
            else ovl::launch_update_efield(c->U, c->E, nullptr, c->L, c->p.dt, c->stream);
        }
        int rc = launched(c, 1, "gauge force");
        if (rc) return rc;
    }
    if (c->p.backreaction != 0.0) {
        {
            ProfScope ps(c, OVL_PROF_OBS);
            launch_force(c, nullptr, c->E, c->p.dt * c->p.backreaction);
        }
        int rc = launched(c, 2, "fermion force");
        if (rc) return rc;
    }
    return OVL_OK;
}

// One leapfrog step of the fused Wilson form, group by group of mode blocks
// (ovl_params.mode_group).  The second half step needs the links of the half
// step while later groups' first half steps still need the step's starting
// links: the half-step links are built out of place in U_b (and U32_b), the
// step-end links are U_b advanced in place, and U/U_b swap.  Per element the
// arithmetic is that of ovl_step's ungrouped path.
int grouped_step(ovl_ctx *c, double *obs = nullptr) {
    const bool move = c->p.qs * (c->tsteps * c->p.dt) < c->p.t_sphaleron;  // Update.cpp:57
    const size_t nl = (size_t)12 * c->L.V;
    if (move && !c->U_b) {
        if (cudaMalloc(&c->U_b, sizeof(double) * nl) != cudaSuccess ||
            (c->U32 && cudaMalloc(&c->U32_b, sizeof(float) * nl) != cudaSuccess)) {
            cudaGetLastError();
            return fail(c, OVL_E_OOM, "ovl_step: half-step links");
        }
    }
    ovl::HopConfig h1 = hop_config(c), h2 = h1;
    if (move) {
        OVL_CUDA(c, cudaMemcpyAsync(c->U_b, c->U, sizeof(double) * nl, cudaMemcpyDeviceToDevice, c->stream));
        {
            ProfScope ps(c, OVL_PROF_LINKS);
            ovl::launch_update_links(c->U_b, c->E, c->L, 0.5 * c->p.dt, c->stream, c->U32_b, c->p.reunitarize != 0);
        }
        int rc = launched(c, 1, "update links");
        if (rc) return rc;
        h2.U = c->U_b;
        if (c->U32) h2.U32 = c->U32_b;
    }
    {
        ProfScope ps(c, OVL_PROF_HOP);
        grouped_pass(c, h1, h2, c->psimid, c->psi, c->psi, c->psimid, c->mode_group, obs);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "wilson (grouped)");
    if (move) {
        {
            ProfScope ps(c, OVL_PROF_LINKS);
            ovl::launch_update_links(c->U_b, c->E, c->L, 0.5 * c->p.dt, c->stream, c->U32_b, c->p.reunitarize != 0);
        }
        int rc = launched(c, 1, "update links");
        if (rc) return rc;
        std::swap(c->U, c->U_b);
        std::swap(c->U32, c->U32_b);
    }
    return OVL_OK;
}

// The error word of the pipelined steps enqueued since the last check (a
// second half step that waited past its bound left its tile undone).
int check_pipeline(ovl_ctx *c) {
    if (!c->pipe_ran) return OVL_OK;
    c->pipe_ran = false;
    int *err = reinterpret_cast<int *>(c->host_small + 63);  // a slot no other read uses
    OVL_CUDA(c, cudaMemcpyAsync(err, c->pipe + ovl::pipeline_counters(c->n_mb) - 1, sizeof(int),
                                cudaMemcpyDeviceToHost, c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (*err) {
        cudaMemsetAsync(c->pipe + ovl::pipeline_counters(c->n_mb) - 1, 0, sizeof(int), c->stream);
        return fail(c, OVL_E_TIMEOUT, "ovl_step: a pipelined half step timed out waiting for its first half");
    }
    return OVL_OK;
}

int ovl_step(ovl_ctx *c, int nsteps) {
    if (!c) return OVL_E_ARG;
    if (nsteps < 0) return fail(c, OVL_E_ARG, "ovl_step: nsteps=%d", nsteps);
    int rc = set_device(c);
    if (rc) return rc;
    if (!overlap(c) && !su3(c) && c->p.form == OVL_FORM_FUSED && nsteps > 0) {
        if (c->hop_variant < 0) rc = autotune(c, nullptr);
        else if (c->mode_group < 0) rc = autotune_groups(c);
        if (rc) return rc;
    }
    for (int n = 0; n < nsteps; n++) {
        if (!overlap(c) && c->p.form == OVL_FORM_FUSED && c->mode_group > 0 && c->mode_group < c->n_mb) {
            if ((rc = grouped_step(c))) return rc;
            c->tsteps++;
            if ((rc = coupled_efield(c))) return rc;
            continue;
        }
        const bool move = c->p.qs * (c->tsteps * c->p.dt) < c->p.t_sphaleron;  // Update.cpp:57
        if ((rc = half_step(c, c->psimid, c->psi))) return rc;
        if (move) {
            {
                ProfScope ps(c, OVL_PROF_LINKS);
                launch_links(c, c->U, c->U32, 0.5 * c->p.dt);
            }
            if ((rc = launched(c, 1, "update links"))) return rc;
        }
        if ((rc = half_step(c, c->psi, c->psimid))) return rc;
        if (move) {
            {
                ProfScope ps(c, OVL_PROF_LINKS);
                launch_links(c, c->U, c->U32, 0.5 * c->p.dt);
            }
            if ((rc = launched(c, 1, "update links"))) return rc;
        }
        c->tsteps++;
        if ((rc = coupled_efield(c))) return rc;
    }
    return check_pipeline(c);
}

// The steps of ovl_step_observe.  async: the charges are copied into `out`
// (page-locked) on the stream and the call returns without waiting (the fused
// two-colour forms; the others complete before returning); otherwise through
// the context's pinned mirror, waited for.
static int step_observe(ovl_ctx *c, int nsteps, double *out, bool async) {
    if (!c || !out) return OVL_E_ARG;
    if (nsteps < 1) return fail(c, OVL_E_ARG, "ovl_step_observe: nsteps=%d", nsteps);
    int rc = set_device(c);
    if (rc) return rc;
    const bool fused = !overlap(c) && !su3(c) && c->p.form == OVL_FORM_FUSED;
    if (fused && c->hop_variant < 0 && (rc = autotune(c, nullptr))) return rc;
    if (fused && c->mode_group < 0 && (rc = autotune_groups(c))) return rc;
    const bool grouped = c->mode_group > 0 && c->mode_group < c->n_mb;
    const ovl::HopConfig hc0 = hop_config(c);
    // the pipelined grouped step sums the charges in its second half steps
    const bool pipe_obs = fused && grouped && pipelined(c, hc0, hc0, c->psi, c->psi);
    if (!fused || (grouped && !pipe_obs)) {
        // other forms: the steps, then the charges kernel
        double ch[4];
        if ((rc = ovl_step(c, nsteps)) || (rc = ovl_charges(c, ch))) return rc;
        for (int k = 0; k < 3; k++) out[k] = ch[k];
        return OVL_OK;
    }
    if (nsteps > 1 && (rc = ovl_step(c, nsteps - 1))) return rc;
    if (!c->obs_partial) {
        if (cudaMalloc(&c->obs_partial, sizeof(double) * ovl::obs_partial_doubles(c->L, c->n_mb)) != cudaSuccess ||
            cudaMalloc(&c->obs_scratch, sizeof(double) * 3 * 256) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, OVL_E_OOM, "ovl_step_observe: partial sums");
        }
    }
    if (pipe_obs) {
        if ((rc = grouped_step(c, c->obs_partial))) return rc;
        c->tsteps++;
        if ((rc = coupled_efield(c))) return rc;
        {
            ProfScope ps(c, OVL_PROF_OBS);
            ovl::launch_obs_finish(c->obs_partial, ovl::pipeline_obs_rows(c->L, c->n_mb, c->mode_group),
                                   c->obs_scratch, 1.0 / (2.0 * c->L.V), c->dev_small + 32, c->stream);
        }
        if ((rc = launched(c, 2, "charges (observing step)"))) return rc;
        OVL_CUDA(c, cudaMemcpyAsync(async ? out : c->host_small + 32, c->dev_small + 32, sizeof(double) * 3,
                                    cudaMemcpyDeviceToHost, c->stream));
        if (async) return OVL_OK;  // a timed-out wait is reported by ovl_synchronize
        if ((rc = check_pipeline(c))) return rc;  // synchronizes the stream
        for (int k = 0; k < 3; k++) out[k] = c->host_small[32 + k];
        return OVL_OK;
    }
    // the last step (Update.cpp:48-79); its second half step reads psi at the
    // step's end and sums the charges on the way
    const bool move = c->p.qs * (c->tsteps * c->p.dt) < c->p.t_sphaleron;
    if ((rc = half_step(c, c->psimid, c->psi))) return rc;
    if (move) {
        {
            ProfScope ps(c, OVL_PROF_LINKS);
            launch_links(c, c->U, c->U32, 0.5 * c->p.dt);
        }
        if ((rc = launched(c, 1, "update links"))) return rc;
    }
    size_t obs_rows = ovl::obs_partial_doubles(c->L, c->n_mb) / 3;
    {
        ProfScope ps(c, OVL_PROF_HOP);
        const ovl::HopConfig hc = hop_config(c);
        if (fp40(c))
            ovl::launch_wilson40_observe(hc, c->psi, c->psi_lo, c->psimid, c->psimid_lo, c->L, c->n_mb, amass(c->p),
                                         c->p.dt, c->p.n_modes, c->p.first_mode, c->obs_partial, c->stream);
        else if (fp32(c))
            obs_rows = ovl::launch_wilson_observe<float>(hc, c->psi, c->psimid, c->L, c->n_mb, amass(c->p), c->p.dt,
                                                         c->p.n_modes, c->p.first_mode, c->obs_partial, c->stream);
        else
            obs_rows = ovl::launch_wilson_observe<double>(hc, c->psi, c->psimid, c->L, c->n_mb, amass(c->p), c->p.dt,
                                                          c->p.n_modes, c->p.first_mode, c->obs_partial, c->stream);
    }
    if ((rc = launched(c, 1, "wilson (fused, observing)"))) return rc;
    if (move) {
        {
            ProfScope ps(c, OVL_PROF_LINKS);
            launch_links(c, c->U, c->U32, 0.5 * c->p.dt);
        }
        if ((rc = launched(c, 1, "update links"))) return rc;
    }
    c->tsteps++;
    if ((rc = coupled_efield(c))) return rc;
    {
        ProfScope ps(c, OVL_PROF_OBS);
        ovl::launch_obs_finish(c->obs_partial, obs_rows, c->obs_scratch,
                               1.0 / (2.0 * c->L.V), c->dev_small + 32, c->stream);
    }
    if ((rc = launched(c, 2, "charges (observing step)"))) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(async ? out : c->host_small + 32, c->dev_small + 32, sizeof(double) * 3,
                                cudaMemcpyDeviceToHost, c->stream));
    if (async) return OVL_OK;
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 3; k++) out[k] = c->host_small[32 + k];
    return OVL_OK;
}

int ovl_step_observe(ovl_ctx *c, int nsteps, double out[3]) { return step_observe(c, nsteps, out, false); }

int ovl_step_observe_async(ovl_ctx *c, int nsteps, double *out) {
    if (!c || !out) return OVL_E_ARG;
    if (!page_locked(out)) return fail(c, OVL_E_ARG, "ovl_step_observe_async: out must be page-locked host memory");
    return step_observe(c, nsteps, out, true);
}

int ovl_get_step_count(const ovl_ctx *c, int *steps) {
    if (!c || !steps) return OVL_E_ARG;
    *steps = c->tsteps;
    return OVL_OK;
}

int ovl_set_step_count(ovl_ctx *c, int steps) {
    if (!c || steps < 0) return OVL_E_ARG;
    c->tsteps = steps;
    return OVL_OK;
}

int ovl_currents(ovl_ctx *c, double *jV, double *jA, double *jVw, double *jAw, double *PS, double *WA) {
    if (!c) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = run_currents(c))) return rc;
    const int V = c->L.V;
    std::vector<double> h((size_t)V * ovl::kCurrentsPerSite);
    OVL_CUDA(c, cudaMemcpyAsync(h.data(), c->per_site, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int s = 0; s < V; s++) {
        const double *q = h.data() + (size_t)s * ovl::kCurrentsPerSite;
        for (int mu = 0; mu < 4; mu++) {
            if (jV) jV[4 * s + mu] = q[mu];
            if (jA) jA[4 * s + mu] = q[4 + mu];
            if (jVw) jVw[4 * s + mu] = q[8 + mu];
            if (jAw) jAw[4 * s + mu] = q[12 + mu];
        }
        if (PS) PS[s] = q[16];
        if (WA) WA[s] = q[17];
    }
    return OVL_OK;
}

int ovl_charges(ovl_ctx *c, double out[4]) {
    if (!c || !out) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    if (overlap(c)) {
        if ((rc = run_currents(c))) return rc;
        ovl::launch_site_sums(c->per_site, c->L, c->partial, c->dev_small, c->stream);
        if ((rc = launched(c, 1, "site sums"))) return rc;
    } else if (su3(c)) {
        ProfScope ps(c, OVL_PROF_OBS);
        if (fp32(c))
            ovl::su3_launch_charges<float>(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->L, c->n_mb, c->p.n_modes,
                                           c->p.first_mode, c->p.r_wilson, c->partial, c->dev_small, c->stream);
        else
            ovl::su3_launch_charges<double>(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->L, c->n_mb, c->p.n_modes,
                                            c->p.first_mode, c->p.r_wilson, c->partial, c->dev_small, c->stream);
    } else {
        ProfScope ps(c, OVL_PROF_OBS);
        if (fp40(c))
            ovl::launch_charges40(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->psi_lo, c->L, c->n_mb, c->p.n_modes,
                                  c->p.first_mode, c->p.r_wilson, c->partial, c->dev_small, c->stream);
        else if (fp32(c))
            ovl::launch_charges<float>(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->p.r_wilson,
                                       c->partial, c->dev_small, c->stream);
        else
            ovl::launch_charges<double>(c->U, c->u1_on ? c->u1 : nullptr, c->psi, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->p.r_wilson,
                                        c->partial, c->dev_small, c->stream);
    }
    if ((rc = launched(c, 2, "charges"))) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(c->host_small, c->dev_small, sizeof(double) * 4, cudaMemcpyDeviceToHost, c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 4; k++) out[k] = c->host_small[k];
    return OVL_OK;
}

int ovl_ncsdot(ovl_ctx *c, double *out) {
    if (!c || !out) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    if (su3(c)) ovl::su3_launch_ncsdot(c->U, c->E, c->L, c->partial, c->dev_small, c->stream);
    else ovl::launch_ncsdot(c->U, c->E, c->L, c->partial, c->dev_small, c->stream);
    if ((rc = launched(c, 2, "ncsdot"))) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(c->host_small, c->dev_small, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    *out = c->host_small[0];
    return OVL_OK;
}

int ovl_ncs_update(ovl_ctx *c, double *delta, double *total) {
    if (!c) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    const size_t V = (size_t)c->L.V;
    if (!c->u_old) {
        if (cudaMalloc(&c->u_old, sizeof(double) * c->link_doubles * 3 * V) != cudaSuccess ||
            cudaMalloc(&c->u_mid, sizeof(double) * c->link_doubles * 3 * V) != cudaSuccess ||
            cudaMalloc(&c->e_mid, sizeof(double) * c->e_comp * 3 * V) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, OVL_E_OOM, "ovl_ncs_update: link copies");
        }
    }
    double d = 0.0;
    if (c->have_u_old) {
        // GetDeltaNCs(1): Simpson weights 1, 4, 1 at x = 0, 1/2, 1 (CoolingMethod.cpp:80-125)
        double *out = c->dev_small;
        if (su3(c)) {
            ovl::su3_launch_geodesic(c->u_old, c->U, 0.5, c->u_mid, c->e_mid, c->L, c->stream);
            ovl::su3_launch_ncsdot(c->u_mid, c->e_mid, c->L, c->partial, out, c->stream);
            ovl::su3_launch_ncsdot(c->u_old, c->e_mid, c->L, c->partial, out + 1, c->stream);
            ovl::su3_launch_ncsdot(c->U, c->e_mid, c->L, c->partial, out + 2, c->stream);
        } else {
            ovl::launch_geodesic(c->u_old, c->U, 0.5, c->u_mid, c->e_mid, c->L, c->stream);
            ovl::launch_ncsdot(c->u_mid, c->e_mid, c->L, c->partial, out, c->stream);
            ovl::launch_ncsdot(c->u_old, c->e_mid, c->L, c->partial, out + 1, c->stream);
            ovl::launch_ncsdot(c->U, c->e_mid, c->L, c->partial, out + 2, c->stream);
        }
        if ((rc = launched(c, 7, "ncs update"))) return rc;
        OVL_CUDA(c, cudaMemcpyAsync(c->host_small, out, sizeof(double) * 3, cudaMemcpyDeviceToHost, c->stream));
        OVL_CUDA(c, cudaStreamSynchronize(c->stream));
        const double *h = c->host_small;
        double value = 0.0, weight = 0.0;
        value += 4.0 * h[0]; weight += 4.0;
        value += h[1]; weight += 1.0;
        value += h[2]; weight += 1.0;
        d = value / weight;
        c->ncs_total += d;
    }
    OVL_CUDA(c, cudaMemcpyAsync(c->u_old, c->U, sizeof(double) * c->link_doubles * 3 * V, cudaMemcpyDeviceToDevice,
                                c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_u_old = true;
    if (delta) *delta = d;
    if (total) *total = c->ncs_total;
    return OVL_OK;
}

// ---------------------------------------------------------------------------
// Gradient-flow cooling and the Chern-Simons calibration
// (GRADIENTFLOW/GradientFlow.cpp:35-190, GRADIENTFLOW/Cooling.cpp:71-201,
// TOPOLOGY/CoolingMethod.cpp:129-200), Minkowski metric, aScale 1, lattice
// spacing a = 2^(blockings) in every direction.  With the reference's
// constants a cooling step is
//   E    = -2 aCube / a^4 (staple sum)        (UpdateElectricFields, set not added)
//   U   <- exp(i cU E) U, cU = -a^2 s^2 aCube^(2/3) / aCube
//   tau += s^2 aCube^(2/3),  s = SqrtDcTauOverSpacing = 0.5 / sqrt 2
// and the calibration adds DcTau/2 NCsDot(U, E) before and after the link
// update.  NCsDot carries a^2 / aCube and the bulk energies (a / aCube)^2 per
// direction; with a a power of two these factors are exact.

namespace {

struct CoolRun {
    ovl_ctx *c;
    double *U, *Ub, *E;  // the cooling links, the blocking target, the flow field
    double *vals;        // per log row: NCsDot before, after, bulk[10], vacuum
    ovl::Lattice L;
    double a = 1.0, aCube = 1.0;
    int steps = 0, blocking = 0;
    double tau = 0.0;
    std::vector<double> row_a, row_tau;  // per log row: spacing and cooling time
    std::vector<int> row_step;           // per log row: whether a step preceded it (its NCsDot pair)
    int rows = 0, max_rows = 0;
};

constexpr int kCoolVals = 13;

double flow_s2() {
    const double s = 0.5 / M_SQRT2;  // GradientFlow::SqrtDcTauOverSpacing
    return s * s;
}

int cool_record(CoolRun &r, bool after_step) {
    ovl_ctx *c = r.c;
    if (r.rows >= r.max_rows) return fail(c, OVL_E_ARG, "ovl_cool: log rows");
    double *v = r.vals + (size_t)kCoolVals * r.rows;
    if (su3(c)) ovl::su3_launch_bulk(r.U, r.E, r.L, c->partial, v + 2, c->stream);
    else ovl::launch_bulk(r.U, r.E, r.L, c->partial, v + 2, c->stream);
    ovl::launch_vacuum_ncs(r.U, r.L, c->nc, c->partial, v + 12, c->stream);
    r.row_a.push_back(r.a);
    r.row_tau.push_back(r.tau);
    r.row_step.push_back(after_step ? 1 : 0);
    r.rows++;
    return launched(c, 4, "cooling observables");
}

// GradientFlow::StandardUpdate / CalibrationUpdate.
int cool_step(CoolRun &r, bool calibrate) {
    ovl_ctx *c = r.c;
    const double s2 = flow_s2(), pw = std::pow(r.aCube, 2.0 / 3.0);
    const double DcTau = s2 * pw;                       // aScale = 1
    const double gamma = (-2.0) * r.aCube;              // MetricDeterminant = aScale = 1
    const double cE = 1.0 / (r.a * r.a);                // gUpMetric = 1
    const double cU = (-1.0) * (r.a * r.a * (s2 * pw)) / r.aCube;
    const size_t n_e = (size_t)c->e_comp * 3 * r.L.V;
    OVL_CUDA(c, cudaMemsetAsync(r.E, 0, sizeof(double) * n_e, c->stream));
    // the staple kernels add -2 dt (staple sum): dt = -gamma cE^2 / 2
    const double dt_e = -0.5 * gamma * cE * cE;
    if (su3(c)) ovl::su3_launch_update_efield(r.U, r.E, r.L, dt_e, c->stream);
    else ovl::launch_update_efield(r.U, r.E, nullptr, r.L, dt_e, c->stream);
    double *v = r.vals + (size_t)kCoolVals * r.rows;  // the row this step's calibration values go with
    if (calibrate) {
        if (su3(c)) ovl::su3_launch_ncsdot(r.U, r.E, r.L, c->partial, v, c->stream);
        else ovl::launch_ncsdot(r.U, r.E, r.L, c->partial, v, c->stream);
    }
    // the link kernels apply exp(-i dt E): dt = -cU
    if (su3(c)) ovl::su3_launch_update_links(r.U, r.E, r.L, -cU, nullptr, false, c->stream);
    else ovl::launch_update_links(r.U, r.E, r.L, -cU, c->stream);
    if (calibrate) {
        if (su3(c)) ovl::su3_launch_ncsdot(r.U, r.E, r.L, c->partial, v + 1, c->stream);
        else ovl::launch_ncsdot(r.U, r.E, r.L, c->partial, v + 1, c->stream);
    }
    r.steps++;
    r.tau += DcTau;
    return launched(c, calibrate ? 7 : 3, "cooling step");
}

// Block(&U), Block(&E): links onto the lattice of twice the spacing, E zero.
int cool_block(CoolRun &r) {
    ovl_ctx *c = r.c;
    ovl::Lattice Lb{r.L.N0 / 2, r.L.N1 / 2, r.L.N2 / 2, 0};
    Lb.V = Lb.N0 * Lb.N1 * Lb.N2;
    ovl::launch_block_links(r.U, r.L, r.Ub, Lb, c->nc, c->stream);
    std::swap(r.U, r.Ub);
    r.L = Lb;
    r.a *= 2.0;
    r.aCube = r.a * r.a * r.a;
    OVL_CUDA(c, cudaMemsetAsync(r.E, 0, sizeof(double) * c->e_comp * 3 * r.L.V, c->stream));
    r.blocking++;
    return launched(c, 2, "blocking");
}

// Cooling::Perform: up to max_steps steps in all, blocking every
// block_frequency 8^level steps while level < max_blocking; with calibrate,
// CalibrationUpdate and a log row before the first step and after each one.
int cool_perform(CoolRun &r, int max_steps, int max_blocking, int block_frequency, bool calibrate) {
    int rc;
    if (calibrate && (rc = cool_record(r, false))) return rc;
    while (r.steps < max_steps) {
        if ((rc = cool_step(r, calibrate))) return rc;
        if (calibrate && (rc = cool_record(r, true))) return rc;
        long long period = block_frequency;
        for (int k = 0; k < r.blocking; k++) period *= 8;
        if (r.steps % period == 0 && r.blocking < max_blocking && (rc = cool_block(r))) return rc;
    }
    return OVL_OK;
}

// The lattice sizes the schedule blocks at, checked before anything runs.
int cool_check_schedule(ovl_ctx *c, int standard_steps, int standard_blocking, int total_steps,
                        int calibration_blocking, int block_frequency) {
    int n[3] = {c->L.N0, c->L.N1, c->L.N2}, blocking = 0;
    for (int step = 1; step <= total_steps; step++) {
        const int max_b = step <= standard_steps ? standard_blocking : calibration_blocking;
        long long period = block_frequency;
        for (int k = 0; k < blocking && period < (1LL << 40); k++) period *= 8;
        if (step % period == 0 && blocking < max_b) {
            if (n[0] < 2 || n[1] < 2 || n[2] < 2)
                return fail(c, OVL_E_ARG, "ovl_cool: blocking %dx%dx%d at cooling step %d", n[0], n[1], n[2], step);
            for (int k = 0; k < 3; k++) n[k] /= 2;
            blocking++;
        }
    }
    return OVL_OK;
}

}  // namespace

int ovl_cool(ovl_ctx *c, int standard_steps, int standard_blocking, int calibration_steps, int calibration_blocking,
             int block_frequency, double *log, int *log_rows, double out[3], double *cooled_links, int cooled_N[3]) {
    if (!c) return OVL_E_ARG;
    if (standard_steps < 0 || calibration_steps < 0 || standard_blocking < 0 || calibration_blocking < 0 ||
        block_frequency < 1)
        return fail(c, OVL_E_ARG, "ovl_cool: steps %d, %d, blocking %d, %d, block frequency %d", standard_steps,
                    calibration_steps, standard_blocking, calibration_blocking, block_frequency);
    if ((long long)standard_steps + calibration_steps > (1LL << 30)) return fail(c, OVL_E_ARG, "ovl_cool: steps");
    int rc = set_device(c);
    if (rc) return rc;
    const int total = standard_steps + calibration_steps;
    if ((rc = cool_check_schedule(c, standard_steps, standard_blocking, total, calibration_blocking, block_frequency)))
        return rc;
    const size_t n_link = (size_t)c->link_doubles * 3 * c->L.V, n_e = (size_t)c->e_comp * 3 * c->L.V;
    CoolRun r;
    r.c = c;
    r.L = c->L;
    r.max_rows = calibration_steps + 1;
    double *mem = nullptr;
    const size_t doubles = 2 * n_link + n_e + (size_t)kCoolVals * r.max_rows;
    if (cudaMalloc(&mem, sizeof(double) * doubles) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, OVL_E_OOM, "ovl_cool: cooling fields");
    }
    auto done = [&](int status) {
        cudaStreamSynchronize(c->stream);
        cudaFree(mem);
        return status;
    };
    r.U = mem;
    r.Ub = mem + n_link;
    r.E = mem + 2 * n_link;
    r.vals = mem + 2 * n_link + n_e;
    // CoolNSave: the hot links, E zero, counters reset, standard cooling
    OVL_CUDA(c, cudaMemcpyAsync(r.U, c->U, sizeof(double) * n_link, cudaMemcpyDeviceToDevice, c->stream));
    OVL_CUDA(c, cudaMemsetAsync(r.E, 0, sizeof(double) * n_e, c->stream));
    if ((rc = cool_perform(r, standard_steps, standard_blocking, block_frequency, false))) return done(rc);
    if (cooled_N) {
        cooled_N[0] = r.L.N0;
        cooled_N[1] = r.L.N1;
        cooled_N[2] = r.L.N2;
    }
    if (cooled_links) {
        if (cudaMemcpyAsync(cooled_links, r.U, sizeof(double) * c->link_doubles * 3 * r.L.V, cudaMemcpyDeviceToHost,
                            c->stream) != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess)
            return done(fail(c, OVL_E_CUDA, "ovl_cool: cooled links"));
    }
    // Calibrate: continue from the cooled links (E zero) up to both phases' steps, with the log
    OVL_CUDA(c, cudaMemsetAsync(r.E, 0, sizeof(double) * c->e_comp * 3 * r.L.V, c->stream));
    if ((rc = cool_perform(r, total, calibration_blocking, block_frequency, true))) return done(rc);
    std::vector<double> h((size_t)kCoolVals * r.rows);
    if (cudaMemcpyAsync(h.data(), r.vals, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return done(fail(c, OVL_E_CUDA, "ovl_cool: log"));
    // rows in the reference's order: cooling time, magnetic, electric, Delta N_CS along the path, vacuum N_CS
    double dncs = 0.0;
    for (int k = 0; k < r.rows; k++) {
        const double *v = &h[(size_t)kCoolVals * k];
        const double a = r.row_a[k];
        if (r.row_step[k]) {
            // the step ran on the lattice of the row before any blocking that followed it
            const double s2 = flow_s2(), aCube = a * a * a;
            const double DcTau = s2 * std::pow(aCube, 2.0 / 3.0), cS = a * a / aCube;
            dncs += 0.5 * DcTau * (cS * v[0]);
            dncs += 0.5 * DcTau * (cS * v[1]);
        }
        const double cB = (a / (a * a * a)) * (a / (a * a * a));
        if (log) {
            double *row = log + 5 * (size_t)k;
            row[0] = r.row_tau[k];
            row[1] = cB * v[2 + 5];
            row[2] = cB * v[2 + 4];
            row[3] = dncs;
            row[4] = v[12];
        }
    }
    if (log_rows) *log_rows = r.rows;
    if (out) {
        out[0] = dncs;
        out[1] = r.tau;
        out[2] = r.blocking;
    }
    return done(OVL_OK);
}

int ovl_update_links(ovl_ctx *c, double dt_step) {
    if (!c) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    launch_links(c, c->U, c->U32, dt_step);
    return launched(c, 1, "update links");
}

int ovl_update_efield(ovl_ctx *c, double dt_step) {
    if (!c) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    if (su3(c)) ovl::su3_launch_update_efield(c->U, c->E, c->L, dt_step, c->stream);
    else ovl::launch_update_efield(c->U, c->E, nullptr, c->L, dt_step, c->stream);
    return launched(c, 1, "update efield");
}

int ovl_color_force(ovl_ctx *c, double *out) {
    if (!c || !out) return OVL_E_ARG;
    if (c->p.fermion != OVL_FERMION_WILSON) return fail(c, OVL_E_UNSUPPORTED, "ovl_color_force: Wilson fermions only");
    int rc = set_device(c);
    if (rc) return rc;
    double *dev = nullptr;
    const size_t n = (size_t)c->e_comp * 3 * c->L.V;
    if (cudaMalloc(&dev, sizeof(double) * n) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, OVL_E_OOM, "ovl_color_force: output buffer");
    }
    launch_force(c, dev, nullptr, 0.0);
    rc = launched(c, 2, "fermion force");
    cudaError_t e = rc ? cudaSuccess : cudaMemcpyAsync(out, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && !rc) e = cudaStreamSynchronize(c->stream);
    cudaFree(dev);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(c, e, "ovl_color_force: copy");
    return OVL_OK;
}

int ovl_fermion_energy(ovl_ctx *c, double *out) {
    if (!c || !out) return OVL_E_ARG;
    if (c->p.fermion != OVL_FERMION_WILSON) return fail(c, OVL_E_UNSUPPORTED, "ovl_fermion_energy: Wilson fermions only");
    int rc = set_device(c);
    if (rc) return rc;
    const double *u1 = c->u1_on ? c->u1 : nullptr;
    if (su3(c)) {
        if (fp32(c)) {
            ovl::su3_launch_hop<float>(su3_links(c), c->psi, c->aux_dst, c->L, 0, c->n_mb, amass(c->p), 0.0, false,
                                       c->stream);
            ovl::su3_launch_fermion_energy<float>(c->psi, c->aux_dst, c->L, c->n_mb, c->p.n_modes, c->p.first_mode,
                                                  c->partial, c->dev_small, c->stream);
        } else {
            ovl::su3_launch_hop<double>(su3_links(c), c->psi, c->aux_dst, c->L, 0, c->n_mb, amass(c->p), 0.0, false,
                                        c->stream);
            ovl::su3_launch_fermion_energy<double>(c->psi, c->aux_dst, c->L, c->n_mb, c->p.n_modes, c->p.first_mode,
                                                   c->partial, c->dev_small, c->stream);
        }
    } else if (fp40(c)) {
        ovl::HopConfig h;
        h.U = c->U;
        h.u1 = u1;
        ovl::launch_wilson40(h, c->psi, c->psi_lo, c->aux_dst, c->aux_dst_lo, c->L, 0, c->n_mb, amass(c->p), 0.0, false,
                             c->stream);
        ovl::launch_fermion_energy40(c->psi, c->psi_lo, c->aux_dst, c->aux_dst_lo, c->L, c->n_mb, c->p.n_modes,
                                     c->p.first_mode, c->partial, c->dev_small, c->stream);
    } else if (fp32(c)) {
        ovl::launch_wilson<float>(c->U, u1, c->psi, c->aux_dst, c->L, 0, c->n_mb, amass(c->p), 0.0, false, c->stream);
        ovl::launch_fermion_energy<float>(c->psi, c->aux_dst, c->L, c->n_mb, c->p.n_modes, c->p.first_mode, c->partial,
                                          c->dev_small, c->stream);
    } else {
        ovl::launch_wilson<double>(c->U, u1, c->psi, c->aux_dst, c->L, 0, c->n_mb, amass(c->p), 0.0, false, c->stream);
        ovl::launch_fermion_energy<double>(c->psi, c->aux_dst, c->L, c->n_mb, c->p.n_modes, c->p.first_mode,
                                           c->partial, c->dev_small, c->stream);
    }
    if ((rc = launched(c, 3, "fermion energy"))) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(c->host_small, c->dev_small, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    *out = c->host_small[0];
    return OVL_OK;
}

int ovl_set_qed_eigenmodes(ovl_ctx *c, double *eigenvalues, double *h_ov, int *n_bad) {
    if (!c) return OVL_E_ARG;
    if (su3(c) || !overlap(c))
        return fail(c, OVL_E_UNSUPPORTED, "ovl_set_qed_eigenmodes: two-colour overlap contexts only");
    const long long D = 4LL * c->nc * c->L.V;
    if (c->p.first_mode + (long long)c->p.n_modes > D)
        return fail(c, OVL_E_ARG, "ovl_set_qed_eigenmodes: modes %d..%d beyond the %lld eigenmodes", c->p.first_mode,
                    c->p.first_mode + c->p.n_modes - 1, D);
    if (D * D > (1LL << 31)) return fail(c, OVL_E_ARG, "ovl_set_qed_eigenmodes: dense %lld x %lld beyond 2^31", D, D);
    int rc = set_device(c);
    if (rc) return rc;
    const size_t stage = sizeof(double2) * (size_t)c->p.n_modes * c->L.V * c->comp;
    double2 *a = nullptr, *b = nullptr;
    if (cudaMalloc(&a, stage) != cudaSuccess || cudaMalloc(&b, stage) != cudaSuccess) {
        cudaGetLastError();
        if (a) cudaFree(a);
        return fail(c, OVL_E_OOM, "ovl_set_qed_eigenmodes: staging");
    }
    int zero = 0, bad = 0;
    const int r = ovl::qed_eigenmodes(c->u1_on ? c->u1 : nullptr, c->L, amass(c->p), c->p.m_dw, c->p.m_fermion,
                                      c->p.dt, c->p.first_mode, c->p.n_modes, a, b, eigenvalues, h_ov, &zero, &bad,
                                      c->sm_count, c->stream);
    if (r == 0) {
        const double *pa = reinterpret_cast<const double *>(a), *pb = reinterpret_cast<const double *>(b);
        if (fp40(c)) {
            ovl::launch_ref_to_blocks<double>(pa, c->psi, c->L, 0, c->p.n_modes, c->stream, c->psi_lo);
            ovl::launch_ref_to_blocks<double>(pb, c->psimid, c->L, 0, c->p.n_modes, c->stream, c->psimid_lo);
        } else if (fp32(c)) {
            ovl::launch_ref_to_blocks<float>(pa, c->psi, c->L, 0, c->p.n_modes, c->stream);
            ovl::launch_ref_to_blocks<float>(pb, c->psimid, c->L, 0, c->p.n_modes, c->stream);
        } else {
            ovl::launch_ref_to_blocks<double>(pa, c->psi, c->L, 0, c->p.n_modes, c->stream);
            ovl::launch_ref_to_blocks<double>(pb, c->psimid, c->L, 0, c->p.n_modes, c->stream);
        }
        c->launches += 7;
    }
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(a);
    cudaFree(b);
    if (r == 2) return fail(c, OVL_E_OOM, "ovl_set_qed_eigenmodes: dense matrices of %lld x %lld", D, D);
    if (r == 3) return fail(c, OVL_E_NOT_CONVERGED, "ovl_set_qed_eigenmodes: diagonalisation did not converge");
    if (r != 0) return fail(c, OVL_E_CUDA, "ovl_set_qed_eigenmodes: cuSOLVER / cuBLAS call failed");
    if (e != cudaSuccess) return cuda_fail(c, e, "ovl_set_qed_eigenmodes");
    if (n_bad) *n_bad = bad + zero;
    return OVL_OK;
}

int ovl_set_handmade_sphaleron(ovl_ctx *c, double r_sphaleron, double t_sphaleron, double *u_final) {
    if (!c) return OVL_E_ARG;
    if (su3(c)) return fail(c, OVL_E_UNSUPPORTED, "ovl_set_handmade_sphaleron: two colours only");
    if (!(r_sphaleron > 0.0) || !(t_sphaleron > 0.0))
        return fail(c, OVL_E_ARG, "ovl_set_handmade_sphaleron: r=%g t=%g", r_sphaleron, t_sphaleron);
    int rc = set_device(c);
    if (rc) return rc;
    const size_t n = (size_t)12 * c->L.V;
    double *uf = nullptr;
    if (u_final && cudaMalloc(&uf, sizeof(double) * n) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, OVL_E_OOM, "ovl_set_handmade_sphaleron: final links");
    }
    ovl::launch_sphaleron(c->U, c->E, uf, c->L, r_sphaleron, t_sphaleron, c->stream);
    refresh_links32(c);
    rc = launched(c, 1, "handmade sphaleron");
    cudaError_t e = cudaSuccess;
    if (!rc && uf) e = cudaMemcpyAsync(u_final, uf, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream);
    if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (uf) cudaFree(uf);
    if (rc) return rc;
    return e == cudaSuccess ? OVL_OK : cuda_fail(c, e, "ovl_set_handmade_sphaleron");
}

int ovl_set_quasi_particles(ovl_ctx *c, double n0, double qs, uint64_t seed, int gauss_max_iter, int *iterations) {
    if (!c) return OVL_E_ARG;
    if (!(n0 >= 0.0) || !(qs > 0.0) || gauss_max_iter < 0)
        return fail(c, OVL_E_ARG, "ovl_set_quasi_particles: n0=%g qs=%g gauss_max_iter=%d", n0, qs, gauss_max_iter);
    int rc = set_device(c);
    if (rc) return rc;
    void *scratch = nullptr;
    const size_t bytes = ovl::quasi_particle_scratch_bytes(c->L, c->nc);
    if (cudaMalloc(&scratch, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, OVL_E_OOM, "ovl_set_quasi_particles: %zu bytes of momentum-space fields", bytes);
    }
    ovl::launch_quasi_particles(c->U, c->E, scratch, c->L, c->nc, n0, qs, seed, c->sm_count, c->stream);
    refresh_links32(c);
    rc = launched(c, 5, "quasi-particles");
    const cudaError_t e = rc ? cudaSuccess : cudaStreamSynchronize(c->stream);
    cudaFree(scratch);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(c, e, "ovl_set_quasi_particles");
    if (iterations) *iterations = 0;
    if (gauss_max_iter > 0) return ovl_gauss_restore(c, gauss_max_iter, 1e-14, iterations, nullptr);
    return OVL_OK;
}

int ovl_gauss_restore(ovl_ctx *c, int max_iter, double tol, int *iterations, double out[2]) {
    if (!c) return OVL_E_ARG;
    if (max_iter < 0 || !(tol >= 0.0)) return fail(c, OVL_E_ARG, "ovl_gauss_restore: max_iter=%d tol=%g", max_iter, tol);
    int rc = set_device(c);
    if (rc) return rc;
    double *G = nullptr;
    if (cudaMalloc(&G, sizeof(double) * c->e_comp * (size_t)c->L.V) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, OVL_E_OOM, "ovl_gauss_restore: violation buffer");
    }
    auto done = [&](int status) { cudaFree(G); return status; };
    double *dv = c->dev_small + 16;  // {sum G^2, max}
    auto violation = [&]() -> int {
        if (su3(c)) ovl::su3_launch_gauss_violation(c->U, c->E, c->L, G, c->partial, dv, c->stream);
        else ovl::launch_gauss_violation(c->U, c->E, c->L, G, c->partial, dv, c->stream);
        return launched(c, 2, "gauss violation");
    };
    auto read_max = [&](double &mx) -> int {
        cudaError_t e = cudaMemcpyAsync(c->host_small, dv, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "ovl_gauss_restore");
        mx = c->host_small[1];
        return OVL_OK;
    };
    // GaussRestore.cpp:132-168: three damped steps per iteration while the
    // signed maximum of the violation exceeds tol (reference: 1e-14, 10000)
    static const double gammas[3] = {7.0 / 24.0, 7.0 / 48.0, 7.0 / 72.0};
    double mx = 0.0;
    if ((rc = violation()) || (rc = read_max(mx))) return done(rc);
    int n = 0;
    while (n < max_iter && mx > tol) {
        for (double g : gammas) {
            if ((rc = violation())) return done(rc);
            if (su3(c)) ovl::su3_launch_gauss_update(c->U, G, c->E, c->L, g, c->stream);
            else ovl::launch_gauss_update(c->U, G, c->E, c->L, g, c->stream);
            if ((rc = launched(c, 1, "gauss update"))) return done(rc);
        }
        n++;
        if ((rc = read_max(mx))) return done(rc);
    }
    if (iterations) *iterations = n;
    if (out) {
        out[0] = c->host_small[1];
        out[1] = std::sqrt(c->host_small[0] / ((double)c->e_comp * c->L.V));  // GaussLawViolation.cpp:64
    }
    return done(OVL_OK);
}

int ovl_bulk(ovl_ctx *c, double out[10]) {
    if (!c || !out) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    if (su3(c)) ovl::su3_launch_bulk(c->U, c->E, c->L, c->partial, c->dev_small, c->stream);
    else ovl::launch_bulk(c->U, c->E, c->L, c->partial, c->dev_small, c->stream);
    if ((rc = launched(c, 2, "bulk"))) return rc;
    OVL_CUDA(c, cudaMemcpyAsync(c->host_small, c->dev_small, sizeof(double) * 10, cudaMemcpyDeviceToHost, c->stream));
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 10; k++) out[k] = c->host_small[k];
    return OVL_OK;
}

int ovl_synchronize(ovl_ctx *c) {
    if (!c) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_pipeline(c);  // a timed-out wait of a step queued without waiting
}

int ovl_device_modes(ovl_ctx *c, void **psi, void **psimid, size_t *bytes) {
    if (!c) return OVL_E_ARG;
    if (psi) *psi = c->psi;
    if (psimid) *psimid = c->psimid;
    if (bytes) *bytes = c->field_complex * c->elem_bytes;
    return OVL_OK;
}

int ovl_launch_count(const ovl_ctx *c, uint64_t *count) {
    if (!c || !count) return OVL_E_ARG;
    *count = c->launches;
    return OVL_OK;
}

int ovl_ritz_bounds(ovl_ctx *c, const double *start, double out[2], double raw[2], int iters[2]) {
    if (!c || !out) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    return ritz_bounds(c, start, out, raw, iters);
}

int ovl_set_spectral_bounds(ovl_ctx *c, const double *pairs, int count) {
    if (!c || !pairs || count < 1) return fail(c, OVL_E_ARG, "ovl_set_spectral_bounds: need at least one pair");
    for (int i = 0; i < count; i++)
        if (!(pairs[2 * i] > 0.0) || !(pairs[2 * i + 1] > pairs[2 * i]) || !std::isfinite(pairs[2 * i + 1]))
            return fail(c, OVL_E_ARG, "ovl_set_spectral_bounds: pair %d = (%g, %g) is not 0 < min < max", i, pairs[2 * i],
                        pairs[2 * i + 1]);
    c->bounds.assign(pairs, pairs + 2 * (size_t)count);
    c->bound_next = 0;
    return OVL_OK;
}

int ovl_apply(ovl_ctx *c, int count, const double *phi, double *out) {
    if (!c || !phi || !out) return OVL_E_ARG;
    if (count < 1 || count > c->p.n_modes) return fail(c, OVL_E_ARG, "ovl_apply: count=%d outside [1, %d]", count, c->p.n_modes);
    int rc = set_device(c);
    if (rc) return rc;
    const size_t per_mode = (size_t)c->L.V * c->comp * 2;
    const int n_mb = (count + ovl::kModeBlock - 1) / ovl::kModeBlock;
    double *stage = nullptr;
    if (cudaMalloc(&stage, per_mode * 8 * (size_t)count) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, OVL_E_OOM, "ovl_apply: staging buffer");
    }
    auto done = [&](int status) { cudaFree(stage); return status; };
    cudaMemsetAsync(c->aux_src, 0, c->field_complex * c->elem_bytes, c->stream);
    if (cudaMemcpyAsync(stage, phi, per_mode * 8 * count, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        return done(fail(c, OVL_E_CUDA, "ovl_apply: upload"));
    if (fp40(c)) {
        cudaMemsetAsync(c->aux_src_lo, 0, c->field_complex * 2, c->stream);
        ovl::launch_ref_to_blocks<double>(stage, c->aux_src, c->L, 0, count, c->stream, c->aux_src_lo);
    } else if (fp32(c)) ovl::launch_ref_to_blocks<float>(stage, c->aux_src, c->L, 0, count, c->stream, nullptr, c->nc);
    else ovl::launch_ref_to_blocks<double>(stage, c->aux_src, c->L, 0, count, c->stream, nullptr, c->nc);
    if ((rc = launched(c, 1, "ref_to_blocks"))) return done(rc);
    if (overlap(c)) {
        if ((rc = run_overlap(c, c->aux_src, c->aux_dst, n_mb, count, false, false))) return done(rc);
    } else if (su3(c)) {
        if (fp32(c)) ovl::su3_launch_hop<float>(su3_links(c), c->aux_src, c->aux_dst, c->L, 0, n_mb, amass(c->p), 0.0, false, c->stream);
        else ovl::su3_launch_hop<double>(su3_links(c), c->aux_src, c->aux_dst, c->L, 0, n_mb, amass(c->p), 0.0, false, c->stream);
        if ((rc = launched(c, 1, "wilson operator"))) return done(rc);
    } else if (fp40(c)) {
        ovl::HopConfig h;
        h.U = c->U;
        h.u1 = c->u1_on ? c->u1 : nullptr;
        ovl::launch_wilson40(h, c->aux_src, c->aux_src_lo, c->aux_dst, c->aux_dst_lo, c->L, 0, n_mb, amass(c->p), 0.0,
                             false, c->stream);
        if ((rc = launched(c, 1, "wilson operator"))) return done(rc);
    } else {
        if (fp32(c)) ovl::launch_wilson<float>(c->U, c->u1_on ? c->u1 : nullptr, c->aux_src, c->aux_dst, c->L, 0, n_mb, amass(c->p), 0.0, false, c->stream);
        else ovl::launch_wilson<double>(c->U, c->u1_on ? c->u1 : nullptr, c->aux_src, c->aux_dst, c->L, 0, n_mb, amass(c->p), 0.0, false, c->stream);
        if ((rc = launched(c, 1, "wilson operator"))) return done(rc);
    }
    if (fp40(c)) ovl::launch_blocks_to_ref<double>(c->aux_dst, stage, c->L, 0, count, c->stream, c->aux_dst_lo);
    else if (fp32(c)) ovl::launch_blocks_to_ref<float>(c->aux_dst, stage, c->L, 0, count, c->stream, nullptr, c->nc);
    else ovl::launch_blocks_to_ref<double>(c->aux_dst, stage, c->L, 0, count, c->stream, nullptr, c->nc);
    if ((rc = launched(c, 1, "blocks_to_ref"))) return done(rc);
    if (cudaMemcpyAsync(out, stage, per_mode * 8 * count, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
        return done(fail(c, OVL_E_CUDA, "ovl_apply: download"));
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return done(fail(c, OVL_E_CUDA, "ovl_apply: synchronise"));
    return done(OVL_OK);
}

int ovl_tuning(const ovl_ctx *c, int *variant, int *mode_group) {
    if (!c) return OVL_E_ARG;
    if (variant) *variant = c->hop_variant;
    if (mode_group) *mode_group = c->mode_group;
    return OVL_OK;
}

int ovl_pipeline_selftest(ovl_ctx *c, int *code) {
    if (!c || !code) return OVL_E_ARG;
    const ovl::HopConfig h = hop_config(c);
    if (!pipelined(c, h, h, c->aux_dst, c->aux_dst) || c->n_mb < 2)
        return fail(c, OVL_E_UNSUPPORTED, "ovl_pipeline_selftest: needs FP32 Wilson modes, hop variant 3, 2+ mode blocks");
    int rc = set_device(c);
    if (rc) return rc;
    if ((rc = check_pipeline(c))) return rc;  // nothing pending from earlier steps
    // groups of one block; tickets start past H1(0)'s tiles, which nobody takes
    const int tiles = (int)(ovl::pipeline_obs_rows(c->L, 1, 1));
    ovl::launch_wilson_pipeline(h, h, c->psimid, c->aux_dst, c->aux_src, c->L, c->n_mb, 1, amass(c->p), c->p.dt,
                                c->pipe, c->sm_count, 0, 0, nullptr, c->stream, tiles);
    c->launches += 2;
    c->pipe_ran = true;
    *code = check_pipeline(c);
    c->err.clear();
    return OVL_OK;
}

int ovl_autotune(ovl_ctx *c, int *variant, double ms[OVL_HOP_VARIANTS]) {
    if (!c) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    double t[ovl::kHopVariants];
    if ((rc = su3(c) ? su3_autotune(c, t) : autotune(c, t))) return rc;
    if (variant) *variant = c->hop_variant;
    if (ms)
        for (int v = 0; v < ovl::kHopVariants; v++) ms[v] = t[v];
    return OVL_OK;
}

int ovl_zolotarev(double lambda_min, double lambda_max, double tol, int npoles, double *b, double *d, double *eps) {
    if (!b || !d || npoles < 1 || npoles > ovl::kMaxPoles || !(lambda_min > 0.0) || !(lambda_max > lambda_min) ||
        !(tol > 0.0))
        return fail(nullptr, OVL_E_ARG, "ovl_zolotarev: invalid interval, tolerance or pole count");
    const double e = ovl::zolotarev(lambda_min, lambda_max, tol, npoles, b, d);
    if (eps) *eps = e;
    return OVL_OK;
}

int ovl_solver_stats(const ovl_ctx *c, int out[3]) {
    if (!c || !out) return OVL_E_ARG;
    out[0] = c->ostats.iterations;
    out[1] = c->ostats.max_mode_iterations;
    out[2] = c->ostats.not_converged;
    return OVL_OK;
}

int ovl_profile_enable(ovl_ctx *c, int on) {
    if (!c) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (auto &v : c->prof) {
        for (auto &pr : v) { c->event_pool.push_back(pr.first); c->event_pool.push_back(pr.second); }
        v.clear();
    }
    c->profiling = on != 0;
    return OVL_OK;
}

int ovl_profile_read(ovl_ctx *c, double ms[OVL_PROF_KINDS], uint64_t launches[OVL_PROF_KINDS]) {
    if (!c || !ms || !launches) return OVL_E_ARG;
    int rc = set_device(c);
    if (rc) return rc;
    OVL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < OVL_PROF_KINDS; k++) {
        double t = 0.0;
        for (auto &pr : c->prof[k]) {
            float e = 0.0f;
            OVL_CUDA(c, cudaEventElapsedTime(&e, pr.first, pr.second));
            t += e;
        }
        ms[k] = t;
        launches[k] = c->prof[k].size();
    }
    return OVL_OK;
}

// ---------------------------------------------------------------- ensembles --

}  // extern "C"

struct ovl_ensemble {
    std::vector<ovl_ctx *> members;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;  // created here (members[0].stream was 0)
    bool fp32 = true;
    int sites = 0;  // tile shape of the batched hop (ovl_ensemble_set_tile); 0 until tuned
    double tile_ms[OVL_ENSEMBLE_TILES] = {0.0, 0.0, 0.0};
    std::vector<ovl::BatchMember> host;  // members in group order (colours, then U(1) background)
    std::vector<int> ts_host;             // step counters, uploaded with the descriptors
    ovl::BatchMember *dev = nullptr;
    int *dev_tsteps = nullptr;
    size_t dev_capacity = 0;  // members dev and dev_tsteps hold (grown by doubling)
    // groups: 2 x (nc - 2) + (U(1) on): two colours without / with U(1), three colours without / with
    int groups[4] = {0, 0, 0, 0};
    int step_launches = 0;  // kernels in the captured step graph
    long long tiles = 0, links = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<ovl::BatchMember> captured;    // descriptors the captured graph holds by value
    std::unique_ptr<ovl::BatchGroup> param = std::make_unique<ovl::BatchGroup>();
    uint64_t launches = 0;
    std::string err;
};

namespace {

std::string g_ens_err;

int ens_fail(ovl_ensemble *e, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (e) e->err = buf; else g_ens_err = buf;
    return code;
}

// Descriptors of all members for tiles of `sites` sites; `tuning`: the hop
// writes each member's operator buffer instead of psi (the state is kept).
int ens_group(const ovl_ctx *c) { return 2 * (c->nc - 2) + (c->u1_on ? 1 : 0); }

void ens_describe(ovl_ensemble *e, int sites, bool tuning) {
    e->host.resize(e->members.size());
    // members in group order (one kernel instance per group)
    std::vector<int> order;
    for (int g = 0; g < 4; g++)
        for (size_t i = 0; i < e->members.size(); i++)
            if (ens_group(e->members[i]) == g) order.push_back((int)i);
    for (int &n : e->groups) n = 0;
    long long tile = 0, link = 0;
    for (size_t k = 0; k < order.size(); k++) {
        const int i = order[k];
        ovl_ctx *c = e->members[i];
        ovl::BatchMember &m = e->host[k];
        e->groups[ens_group(c)]++;
        m.psi = tuning ? c->aux_dst : c->psi;
        m.psimid = c->psimid;
        m.U = c->U;
        m.u1 = c->u1_on ? c->u1 : nullptr;
        m.U32 = c->U32;
        m.u1_32 = c->u1_on ? c->u1_32 : nullptr;
        m.E = c->E;
        m.tsteps = e->dev_tsteps + i;
        m.N0 = c->L.N0;
        m.N1 = c->L.N1;
        m.N2 = c->L.N2;
        m.V = c->L.V;
        m.n_mb = c->n_mb;
        m.reunit = c->p.reunitarize != 0;
        m.nc = c->nc;
        m.comp = c->comp;
        m.amass = amass(c->p);
        m.dt = c->p.dt;
        m.qs = c->p.qs;
        m.t_sphaleron = c->p.t_sphaleron;
        m.tile0 = tile;
        m.link0 = link;
        tile += ovl::batch_tiles(c->L.V, c->n_mb, sites, c->nc, e->fp32);
        link += 3LL * c->L.V;
    }
    e->tiles = tile;
    e->links = link;
}

// The descriptors and step counters go up from pageable host vectors: each
// copy has been staged when cudaMemcpyAsync returns, so the vectors may change
// at once and the host does not wait for the stream (the ensemble's earlier
// work, or work it was made to wait for, may still be running).
int ens_upload(ovl_ensemble *e) {
    e->ts_host.resize(e->members.size());
    for (size_t i = 0; i < e->ts_host.size(); i++) e->ts_host[i] = e->members[i]->tsteps;
    cudaError_t r = cudaMemcpyAsync(e->dev, e->host.data(), sizeof(ovl::BatchMember) * e->host.size(),
                                    cudaMemcpyHostToDevice, e->stream);
    if (r == cudaSuccess)
        r = cudaMemcpyAsync(e->dev_tsteps, e->ts_host.data(), sizeof(int) * e->ts_host.size(),
                            cudaMemcpyHostToDevice, e->stream);
    if (r == cudaSuccess && (page_locked(e->host.data()) || page_locked(e->ts_host.data())))
        r = cudaStreamSynchronize(e->stream);
    return r == cudaSuccess ? OVL_OK : ens_fail(e, OVL_E_CUDA, "ensemble: descriptor upload: %s", cudaGetErrorString(r));
}

void ens_free_graph(ovl_ensemble *e) {
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->exec = nullptr;
    e->graph = nullptr;
    e->captured.clear();
}

bool ens_same_graph(const ovl_ensemble *e) {
    return e->exec && e->captured.size() == e->host.size() &&
           std::memcmp(e->captured.data(), e->host.data(), sizeof(ovl::BatchMember) * e->host.size()) == 0;
}

// The launches of one batched half step: each member group by its kernel, in
// chunks of at most kParamMembers descriptors passed by value (a captured
// graph holds them: it is recaptured when they change).
int ens_hop(ovl_ensemble *e, int sites, int phase) {
    int first = 0, n_launch = 0;
    for (int g = 0; g < 4; g++) {
        const int n = e->groups[g];
        for (int c0 = 0; c0 < n; c0 += ovl::kParamMembers) {
            ovl::BatchGroup &bg = *e->param;
            bg.count = std::min(ovl::kParamMembers, n - c0);
            long long tiles = 0;
            for (int k = 0; k < bg.count; k++) {
                const ovl::BatchMember &m = e->host[first + c0 + k];
                bg.m[k] = m;
                tiles += ovl::batch_tiles(m.V, m.n_mb, sites, m.nc, e->fp32);
            }
            ovl::launch_batch_hop_param(bg, tiles, sites, phase, e->fp32, (g & 1) != 0, e->stream, g >= 2 ? 3 : 2);
            n_launch++;
        }
        first += n;
    }
    return n_launch;
}

}  // namespace

extern "C" {

int ovl_ensemble_create(const ovl_params *members, int count, ovl_ensemble **out) {
    if (!members || !out || count < 1) return ens_fail(nullptr, OVL_E_ARG, "ovl_ensemble_create: need members");
    *out = nullptr;
    const ovl_params &p0 = members[0];  // sets the precision and device of the ensemble
    for (int i = 0; i < count; i++) {
        const ovl_params &p = members[i];
        if (p.fermion != OVL_FERMION_WILSON || p.form != OVL_FORM_FUSED)
            return ens_fail(nullptr, OVL_E_UNSUPPORTED, "ovl_ensemble_create: member %d: Wilson fermions, fused form only", i);
        if (p.precision != OVL_PREC_FP32 && p.precision != OVL_PREC_FP64)
            return ens_fail(nullptr, OVL_E_UNSUPPORTED, "ovl_ensemble_create: member %d: FP32 or FP64 modes only", i);
        if (p.precision != p0.precision || p.device != p0.device)
            return ens_fail(nullptr, OVL_E_ARG, "ovl_ensemble_create: member %d: one precision and device for all", i);
        if (p.backreaction != 0.0 || p.gauge_force)
            return ens_fail(nullptr, OVL_E_UNSUPPORTED, "ovl_ensemble_create: member %d: no coupled evolution", i);

    }
    ovl_ensemble *e = new (std::nothrow) ovl_ensemble();
    if (!e) return ens_fail(nullptr, OVL_E_OOM, "ovl_ensemble_create: host allocation");
    auto bail = [&](int code) {
        g_ens_err = e->err;
        ovl_ensemble_destroy(e);
        return code;
    };
    e->device = p0.device;
    e->fp32 = p0.precision == OVL_PREC_FP32;
    if (cudaSetDevice(e->device) != cudaSuccess)
        return bail(ens_fail(e, OVL_E_CUDA, "ovl_ensemble_create: device %d", e->device));
    if (p0.stream) {
        e->stream = reinterpret_cast<cudaStream_t>(p0.stream);
    } else {
        if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(ens_fail(e, OVL_E_CUDA, "ovl_ensemble_create: stream"));
        e->own_stream = true;
    }
    for (int i = 0; i < count; i++) {
        ovl_params p = members[i];
        p.stream = reinterpret_cast<uint64_t>(e->stream);
        // stepped alone, a member runs variant 0 or, FP32 and asked for, the packed kernel
        p.hop_variant = p.precision == OVL_PREC_FP32 && p.hop_variant == ovl::kPackedVariant ? ovl::kPackedVariant : 0;
        p.mode_group = 0;
        ovl_ctx *c = nullptr;
        int rc = ovl_create(&p, &c);
        if (rc) return bail(ens_fail(e, rc, "ovl_ensemble_create: member %d: %s", i, ovl_last_error(nullptr)));
        e->members.push_back(c);
    }
    const size_t cap = std::max<size_t>(16, (size_t)count);
    if (cudaMalloc(&e->dev, sizeof(ovl::BatchMember) * cap) != cudaSuccess ||
        cudaMalloc(&e->dev_tsteps, sizeof(int) * cap) != cudaSuccess) {
        cudaGetLastError();
        return bail(ens_fail(e, OVL_E_OOM, "ovl_ensemble_create: descriptors"));
    }
    e->dev_capacity = cap;
    *out = e;
    return OVL_OK;
}

int ovl_ensemble_destroy(ovl_ensemble *e) {
    if (!e) return OVL_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    ens_free_graph(e);
    for (ovl_ctx *c : e->members) ovl_destroy(c);
    if (e->dev) cudaFree(e->dev);
    if (e->dev_tsteps) cudaFree(e->dev_tsteps);
    if (e->stream && e->own_stream) cudaStreamDestroy(e->stream);
    delete e;
    return OVL_OK;
}

const char *ovl_ensemble_last_error(const ovl_ensemble *e) { return e ? e->err.c_str() : g_ens_err.c_str(); }

int ovl_ensemble_add(ovl_ensemble *e, const ovl_params *member, int *index) {
    if (!e || !member) return OVL_E_ARG;
    const ovl_params &p = *member;
    if (p.fermion != OVL_FERMION_WILSON || p.form != OVL_FORM_FUSED)
        return ens_fail(e, OVL_E_UNSUPPORTED, "ovl_ensemble_add: Wilson fermions, fused form only");
    if ((p.precision == OVL_PREC_FP32) != e->fp32 || (p.precision != OVL_PREC_FP32 && p.precision != OVL_PREC_FP64) ||
        p.device != e->device)
        return ens_fail(e, OVL_E_ARG, "ovl_ensemble_add: the ensemble's precision and device");
    if (p.backreaction != 0.0 || p.gauge_force) return ens_fail(e, OVL_E_UNSUPPORTED, "ovl_ensemble_add: no coupled evolution");

    if (cudaSetDevice(e->device) != cudaSuccess) return ens_fail(e, OVL_E_CUDA, "ovl_ensemble_add: device");
    ovl_params q = p;
    q.stream = reinterpret_cast<uint64_t>(e->stream);
    q.hop_variant = q.precision == OVL_PREC_FP32 && q.hop_variant == ovl::kPackedVariant ? ovl::kPackedVariant : 0;
    q.mode_group = 0;
    ovl_ctx *c = nullptr;
    int rc = ovl_create(&q, &c);
    if (rc) return ens_fail(e, rc, "ovl_ensemble_add: %s", ovl_last_error(nullptr));
    // descriptor arrays for the new count, grown by doubling (a cudaFree
    // waits for the whole device); the step graph bakes in their address,
    // the count and the tiles: it is captured again
    const size_t n = e->members.size() + 1;
    cudaStreamSynchronize(e->stream);
    if (n > e->dev_capacity) {
        const size_t cap = std::max(n, 2 * e->dev_capacity);
        ovl::BatchMember *dev = nullptr;
        int *ts = nullptr;
        if (cudaMalloc(&dev, sizeof(ovl::BatchMember) * cap) != cudaSuccess ||
            cudaMalloc(&ts, sizeof(int) * cap) != cudaSuccess) {
            cudaGetLastError();
            if (dev) cudaFree(dev);
            ovl_destroy(c);
            return ens_fail(e, OVL_E_OOM, "ovl_ensemble_add: descriptors");
        }
        cudaFree(e->dev);
        cudaFree(e->dev_tsteps);
        e->dev = dev;
        e->dev_tsteps = ts;
        e->dev_capacity = cap;
    }
    ens_free_graph(e);
    e->members.push_back(c);
    if (index) *index = (int)n - 1;
    return OVL_OK;
}

int ovl_ensemble_remove(ovl_ensemble *e, int index) {
    if (!e || index < 0 || index >= (int)e->members.size())
        return ens_fail(e, OVL_E_ARG, "ovl_ensemble_remove: index %d", index);
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    ens_free_graph(e);
    ovl_destroy(e->members[index]);
    e->members.erase(e->members.begin() + index);
    return OVL_OK;
}

int ovl_ensemble_size(const ovl_ensemble *e) { return e ? (int)e->members.size() : 0; }

int ovl_ensemble_member(ovl_ensemble *e, int index, ovl_ctx **ctx) {
    if (!e || !ctx || index < 0 || index >= (int)e->members.size())
        return ens_fail(e, OVL_E_ARG, "ovl_ensemble_member: index %d", index);
    *ctx = e->members[index];
    return OVL_OK;
}

}  // extern "C"

namespace {

// Sites per tile of the batched hop: times tiles of 8 and 4 sites (and, FP32,
// the packed-pair tiles) on a half step that writes the members' operator
// buffers (the state is kept), by time_candidates: a sustained window per
// candidate where a half step takes a millisecond or more.
int ens_tune(ovl_ensemble *e) {
    for (ovl_ctx *c : e->members) cudaMemsetAsync(c->aux_dst, 0, c->field_complex * c->elem_bytes, e->stream);
    // tile shapes in the order of tile_ms; the packed tiles only for FP32
    const int cand[OVL_ENSEMBLE_TILES] = {8, 4, ovl::kBatchPacked};
    const int n = e->fp32 ? OVL_ENSEMBLE_TILES : 2;
    int rc = OVL_OK, cur = -1;
    auto run = [&](int k) -> uint64_t {
        if (k != cur) {  // describe and upload when the candidate changes (in an untimed warm-up launch)
            ens_describe(e, cand[k], true);
            if (rc == OVL_OK) rc = ens_upload(e);
            cur = k;
        }
        return rc == OVL_OK ? (uint64_t)ens_hop(e, cand[k], 0) : 0;
    };
    double ms[OVL_ENSEMBLE_TILES] = {0.0, 0.0, 0.0};
    uint64_t nl = 0;
    if (!time_candidates(e->stream, n, run, ms, nl)) return ens_fail(e, OVL_E_CUDA, "ensemble: events");
    e->launches += nl;
    int pick = 0;
    for (int k = 0; k < n; k++) {
        e->tile_ms[k] = ms[k];
        if (ms[k] < ms[pick]) pick = k;
    }
    cudaError_t r = cudaGetLastError();
    if (rc == OVL_OK && r != cudaSuccess) rc = ens_fail(e, OVL_E_CUDA, "ensemble tuning: %s", cudaGetErrorString(r));
    e->sites = cand[pick];
    return rc;
}

// One leapfrog step of every member (Update.cpp:48-79 per member): half step,
// links, half step, links, step counters.  Returns the launches enqueued.
int ens_enqueue_step(ovl_ensemble *e) {
    const int n = (int)e->members.size();
    int nl = ens_hop(e, e->sites, 0);
    ovl::launch_batch_links(e->dev, n, e->links, e->stream);
    nl += ens_hop(e, e->sites, 1);
    ovl::launch_batch_links(e->dev, n, e->links, e->stream);
    ovl::launch_batch_advance(e->dev, n, e->stream);
    return nl + 3;
}

int ens_capture(ovl_ensemble *e) {
    ens_free_graph(e);
    cudaError_t r = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
    if (r == cudaSuccess) {
        e->step_launches = ens_enqueue_step(e);
        r = cudaStreamEndCapture(e->stream, &e->graph);
    }
    if (r == cudaSuccess) r = cudaGraphInstantiate(&e->exec, e->graph, 0);
    if (r != cudaSuccess) {
        cudaGetLastError();
        ens_free_graph(e);
        return ens_fail(e, OVL_E_CUDA, "ensemble: step graph: %s", cudaGetErrorString(r));
    }
    e->captured = e->host;
    return OVL_OK;
}

}  // namespace

extern "C" {

int ovl_ensemble_step(ovl_ensemble *e, int nsteps) {
    if (!e) return OVL_E_ARG;
    if (nsteps < 0) return ens_fail(e, OVL_E_ARG, "ovl_ensemble_step: nsteps=%d", nsteps);
    if (nsteps == 0 || e->members.empty()) return OVL_OK;
    if (cudaSetDevice(e->device) != cudaSuccess) return ens_fail(e, OVL_E_CUDA, "ovl_ensemble_step: device");
    int rc;
    if (e->sites == 0 && (rc = ens_tune(e))) return rc;
    // descriptors are rebuilt every call (links, phases and counters may have
    // been set on the members); the captured graph reads them from device memory
    ens_describe(e, e->sites, false);
    if ((rc = ens_upload(e))) return rc;
    if (!ens_same_graph(e) && (rc = ens_capture(e))) return rc;
    for (int n = 0; n < nsteps; n++) {
        cudaError_t r = cudaGraphLaunch(e->exec, e->stream);
        if (r != cudaSuccess) return ens_fail(e, OVL_E_CUDA, "ovl_ensemble_step: graph launch: %s", cudaGetErrorString(r));
    }
    e->launches += (uint64_t)e->step_launches * nsteps;
    for (ovl_ctx *c : e->members) c->tsteps += nsteps;
    cudaError_t r = cudaGetLastError();
    return r == cudaSuccess ? OVL_OK : ens_fail(e, OVL_E_CUDA, "ovl_ensemble_step: %s", cudaGetErrorString(r));
}

int ovl_ensemble_charges(ovl_ensemble *e, double *out) {
    if (!e || !out) return OVL_E_ARG;
    for (size_t i = 0; i < e->members.size(); i++) {
        int rc = ovl_charges(e->members[i], out + 4 * i);
        if (rc) return ens_fail(e, rc, "ovl_ensemble_charges: member %zu: %s", i, e->members[i]->err.c_str());
    }
    return OVL_OK;
}

int ovl_ensemble_set_tile(ovl_ensemble *e, int sites) {
    if (!e) return OVL_E_ARG;
    if (sites != 0 && sites != 4 && sites != 8 && sites != ovl::kBatchPacked)
        return ens_fail(e, OVL_E_ARG, "ovl_ensemble_set_tile: sites=%d (0 = tune, 4, 8 or %d)", sites, ovl::kBatchPacked);
    if (sites != e->sites) {
        // the captured step launches the old tile kernels even where the
        // descriptors come out the same (a single member starts at tile 0)
        if (cudaSetDevice(e->device) != cudaSuccess) return ens_fail(e, OVL_E_CUDA, "ovl_ensemble_set_tile: device");
        ens_free_graph(e);
        e->sites = sites;
    }
    return OVL_OK;
}

int ovl_ensemble_info(const ovl_ensemble *e, int *sites, double tile_ms[OVL_ENSEMBLE_TILES], uint64_t *launches) {
    if (!e) return OVL_E_ARG;
    if (sites) *sites = e->sites;
    if (tile_ms)
        for (int k = 0; k < OVL_ENSEMBLE_TILES; k++) tile_ms[k] = e->tile_ms[k];
    if (launches) *launches = e->launches;
    return OVL_OK;
}

int ovl_ensemble_synchronize(ovl_ensemble *e) {
    if (!e) return OVL_E_ARG;
    cudaSetDevice(e->device);
    cudaError_t r = cudaStreamSynchronize(e->stream);
    return r == cudaSuccess ? OVL_OK : ens_fail(e, OVL_E_CUDA, "ovl_ensemble_synchronize: %s", cudaGetErrorString(r));
}

uint64_t ovl_ensemble_stream(const ovl_ensemble *e) { return e ? reinterpret_cast<uint64_t>(e->stream) : 0; }

}  // extern "C"
