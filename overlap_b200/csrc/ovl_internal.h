// Launchers shared between the overlap_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace ovl {

struct Lattice;

constexpr int kSitesPerCta = 8;  // sites per CTA of the Wilson kernels (8 warps)

// Wilson operator on mode blocks [mb_first, mb_first + n_mb) of src.
// accumulate: dst(+same offset) += dt * D src; otherwise dst (a buffer of
// n_mb blocks) = D src.
// u1: U(1) background phases (complex per (x, y) plane site and mu = 0, 1), or null.
template <typename T>
void launch_wilson(const double *links, const double *u1, const void *src, void *dst, const Lattice &L, int mb_first,
                   int n_mb, double amass, double dt, bool accumulate, cudaStream_t stream);
// Link sources and kernel variant of the leapfrog half step (chosen by the
// autotuner, see ovl_autotune): U/u1 FP64 links and phases; U32/u1_32 their FP32
// copies (used by the FP32 path when set); variant 0..3.  Variant 3 (FP32
// with the FP32 link copy only) is the packed-pair kernel: two modes per
// thread on the paired FP32 instructions; FP64 runs variant 0 in its place.
struct HopConfig {
    const double *U = nullptr, *u1 = nullptr;
    const float *U32 = nullptr, *u1_32 = nullptr;
    int variant = 0;
};
constexpr int kHopVariants = 4;
constexpr int kPackedVariant = 3;
template <typename T>
void launch_wilson_tuned(const HopConfig &hc, const void *src, void *dst, const Lattice &L, int mb_first, int n_mb,
                         double amass, double dt, bool accumulate, cudaStream_t stream);
void launch_links_to_f32(const double *U, float *U32, size_t n, cudaStream_t stream);
// The fused half step dst += dt D src that also sums the local charges of src
// (N_V, N_5, PS: the vacuum-weighted bilinears psi^+ psi, psi^+ g5 psi and
// psi^+ i g0 g5 psi summed over modes and sites, Currents.cpp:44-92) on the way:
// 3 doubles per CTA into `partial` (obs_partial_doubles), reduced by
// launch_obs_finish into out3 (scaled by 1/2V).  FP32/FP64 modes (variant 0
// stencil, or the packed kernel for FP32 when hc.variant is kPackedVariant) or
// FP40 (src_lo / dst_lo set).  partial holds obs_partial_doubles; the launch
// returns the rows it wrote.
size_t obs_partial_doubles(const Lattice &L, int n_mb);
template <typename T>
size_t launch_wilson_observe(const HopConfig &hc, const void *src, void *dst, const Lattice &L, int n_mb, double amass,
                             double dt, int n_modes, int first_mode, double *partial, cudaStream_t stream);
void launch_wilson40_observe(const HopConfig &hc, const void *src, const void *src_lo, void *dst, void *dst_lo,
                             const Lattice &L, int n_mb, double amass, double dt, int n_modes, int first_mode,
                             double *partial, cudaStream_t stream);
void launch_obs_finish(const double *partial, size_t rows, double *scratch, double scale, double *out3,
                       cudaStream_t stream);
// The grouped fused step in one persistent launch (FP32 packed pairs, hop
// variant 3): b += dt D a with links h1 and then c += dt D b with links h2,
// group by group of `group` mode blocks, each group's second half step while
// its fields are still in L2.  counters: pipeline_counters(n_mb) ints, the last
// an error word the launch sets (and never clears) when a wait times out.
// partial (or null): the local charges of b summed in the second half steps,
// kObsVals per row, pipeline_obs_rows rows.  first_ticket > 0 (self-test
// only) starts the ticket counter there, so the tiles before it are never
// taken and the second half steps that wait on them time out.
int pipeline_counters(int n_mb);
size_t pipeline_obs_rows(const Lattice &L, int n_mb, int group);
void launch_wilson_pipeline(const HopConfig &h1, const HopConfig &h2, const void *a, void *b, void *c,
                            const Lattice &L, int n_mb, int group, double amass, double dt, int *counters, int sm_count,
                            int n_modes, int first_mode, double *partial, cudaStream_t stream, int first_ticket = 0);
// Half step on 40-bit storage (uint2 high words + packed extension bytes,
// ovl_fp40.cuh), FP64 arithmetic and FP64 links (hc.U, hc.u1); accumulate:
// dst += dt D src, else dst (a buffer of n_mb blocks) = D src.  hc.variant:
// 0 = 128 registers (2 CTAs per SM), 1 = 80 registers (3 CTAs per SM).
constexpr int kFp40Variants = 2;
void launch_wilson40(const HopConfig &hc, const void *src, const void *src_lo, void *dst, void *dst_lo,
                     const Lattice &L, int mb_first, int n_mb, double amass, double dt, bool accumulate,
                     cudaStream_t stream);

template <typename T>
void launch_axpy(void *dst, const void *deriv, size_t n_complex, double dt, int sm_count, cudaStream_t stream);

// Gauge fields (FP64).
void launch_update_links(double *U, const double *E, const Lattice &L, double dt_step, cudaStream_t stream,
                         float *U32 = nullptr, bool reunit = false);
void launch_update_efield(const double *U, double *E, double *dE, const Lattice &L, double dt_step, cudaStream_t stream);

// Reductions.  partial: caller-provided device scratch of reduce_partial_doubles()
// doubles; out: device array of the result size.
size_t ncsdot_partial_doubles(const Lattice &L);
void launch_ncsdot(const double *U, const double *E, const Lattice &L, double *partial, double *out, cudaStream_t stream);
int ncsdot_blocks_exact(const Lattice &L);
void launch_ncsdot_into(const double *U, const double *E, const Lattice &L, int blocks, double *partial, double *out,
                        cudaStream_t stream);
// Overlap eigenmodes in the U(1) background (ovl_eigen.cu): modes
// [first_mode, first_mode + count) of the dense, exactly diagonalised h_ov
// into psi_ref / mid_ref (reference layout, device); 0 on success, 1 library
// error, 2 out of memory, 3 no convergence.
int qed_eigenmodes(const double *u1, const Lattice &L, double amass, double mdw, double mf, double dt, int first_mode,
                   int count, double2 *psi_ref, double2 *mid_ref, double *omega_host, double *h_host, int *zero_modes,
                   int *bad, int sm_count, cudaStream_t stream);
// Quasi-particle gauge fields (ovl_quasi.cu): links and E of nc colours from
// occupancy n0 below qs, noise from `seed`; scratch holds
// quasi_particle_scratch_bytes.
size_t quasi_particle_scratch_bytes(const Lattice &L, int nc);
void launch_quasi_particles(double *U, double *E, void *scratch, const Lattice &L, int nc, double n0, double qs,
                            uint64_t seed, int sm_count, cudaStream_t stream);
// The handmade sphaleron start: U = 1, E carrying it to G(x) G(x+mu)^+ in time
// t (written to Ufinal when set).
void launch_sphaleron(double *U, double *E, double *Ufinal, const Lattice &L, double r, double t, cudaStream_t stream);
void launch_geodesic(const double *Uold, const double *Unew, double c, double *Umid, double *Emid, const Lattice &L,
                     cudaStream_t stream);
size_t bulk_partial_doubles(const Lattice &L);
// Gradient-flow cooling (GRADIENTFLOW/Cooling.cpp): blocking to twice the
// spacing and the vacuum N_CS estimate; both colours; the estimate needs
// ncsdot_partial_doubles of partial.
void launch_block_links(const double *U, const Lattice &L, double *Uout, const Lattice &Lout, int nc,
                        cudaStream_t stream);
void launch_vacuum_ncs(const double *U, const Lattice &L, int nc, double *partial, double *out, cudaStream_t stream);
// Gauss-law restoration: violation G[3V] with out[0] = sum G^2, out[1] = signed
// max; then E_mu -= gamma (G - U G(x+mu) U^+).
size_t gauss_partial_doubles(const Lattice &L);
void launch_gauss_violation(const double *U, const double *E, const Lattice &L, double *G, double *partial,
                            double *out, cudaStream_t stream);
void launch_gauss_update(const double *U, const double *G, double *E, const Lattice &L, double gamma,
                         cudaStream_t stream);
void launch_bulk(const double *U, const double *E, const Lattice &L, double *partial, double *out, cudaStream_t stream);

// Currents: 16 doubles per site (jV[4], jA[4], jVw[4], jAw[4]) + PS + WA = 18.
constexpr int kCurrentsPerSite = 18;
int currents_groups(int n_mb);
size_t currents_partial_doubles(const Lattice &L, int n_mb);
template <typename T>
void launch_currents(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                     int first_mode, double r_wilson, double *partial, double *per_site, cudaStream_t stream);
void launch_site_sums(const double *per_site, const Lattice &L, double *partial, double *out4, cudaStream_t stream);
void launch_currents_finish(const double *partial, int groups, const Lattice &L, double *per_site, cudaStream_t stream);
void launch_overlap_currents(const void *psi, const void *opsi, const Lattice &L, int n_mb, int n_modes,
                             int first_mode, double *partial, double *per_site, cudaStream_t stream, bool fp32 = false,
                             int nc = 2);
// Fermion back-reaction: dH_F/dtheta^a_mu(x) per link (24 doubles of colour
// bilinears per site and group in `partial`); into out[9 V] when out is set,
// else E += coef * force.  Fermion energy H_F from psi and dpsi = D psi.
constexpr int kForcePerSite = 24;
size_t force_partial_doubles(const Lattice &L, int n_mb);
template <typename T>
void launch_color_force(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                        int first_mode, double *partial, double *out, double *E, double coef, cudaStream_t stream);
size_t energy_partial_doubles();
template <typename T>
void launch_fermion_energy(const void *psi, const void *dpsi, const Lattice &L, int n_mb, int n_modes, int first_mode,
                           double *partial, double *out, cudaStream_t stream);
// Ritz solver for the overlap spectral bounds (ovl_ritz.cu): work space for a
// lattice of V sites, the start vector buffer (compact [V][8] double2), a
// seeded uniform start vector, and the run: out = {lambda_min, -lambda_max}.
void *ritz_create(int V, int nc);
void ritz_destroy(void *work);
double2 *ritz_start_buffer(void *work);
void launch_ritz_random_start(void *work, uint64_t seed, uint64_t call, cudaStream_t stream);
cudaError_t ritz_run(void *work, const double *U, const double *u1, const Lattice &L, double amass, int max_iter,
                     int nrestart, double delitr, double out[2], int iters[2], cudaStream_t stream,
                     uint64_t *launches);
// The same observables on 40-bit storage (hi words + extension bytes).
void launch_currents40(const double *U, const double *u1, const void *hi, const void *lo, const Lattice &L, int n_mb,
                       int n_modes, int first_mode, double r_wilson, double *partial, double *per_site,
                       cudaStream_t stream);
void launch_charges40(const double *U, const double *u1, const void *hi, const void *lo, const Lattice &L, int n_mb,
                      int n_modes, int first_mode, double r_wilson, double *partial, double *out4, cudaStream_t stream);
void launch_color_force40(const double *U, const double *u1, const void *hi, const void *lo, const Lattice &L, int n_mb,
                          int n_modes, int first_mode, double *partial, double *out, double *E, double coef,
                          cudaStream_t stream);
void launch_fermion_energy40(const void *hi, const void *lo, const void *dhi, const void *dlo, const Lattice &L,
                             int n_mb, int n_modes, int first_mode, double *partial, double *out, cudaStream_t stream);
// Ensembles (ovl_batch.cu): one descriptor per member in device memory.
// tile0: first tile of the member in the batched hop launch (batch_tiles tiles,
// member by member); link0: first link in the batched link update.  tsteps:
// the member's step counter on the device.
struct BatchMember {
    void *psi, *psimid;
    double *U;
    const double *u1;
    float *U32;
    const float *u1_32;
    const double *E;
    int *tsteps;
    int N0, N1, N2, V;
    int n_mb;
    int reunit;
    int nc, comp;  // colours (2 or 3) and complex components per mode and site (4 nc)
    double amass, dt, qs, t_sphaleron;
    long long tile0, link0;
};
// Tiles of a member in the batched hop: `sites` = 4 or 8 sites x one mode
// block (a warp per site), or kBatchPacked: FP32 two-colour members in
// packed-pair tiles of 8 sites x 8 mode blocks (hop variant 3's kernel body),
// the other members in tiles of 8 sites.
constexpr int kBatchPacked = 16;
long long batch_tiles(int V, int n_mb, int sites, int nc, bool fp32);
// Up to kParamMembers descriptors of a group passed by value (kernel
// parameter space; 128 x 136 bytes stays inside the 32 KB parameter limit).
constexpr int kParamMembers = 128;
struct BatchGroup {
    int count;
    BatchMember m[kParamMembers];
};
static_assert(sizeof(BatchGroup) <= 32764, "kernel parameter limit");
void launch_batch_hop_param(const BatchGroup &g, long long tiles, int sites, int phase, bool fp32, bool u1,
                            cudaStream_t stream, int nc = 2);
void launch_batch_links(const BatchMember *members, int count, long long total_links, cudaStream_t stream);
void launch_batch_advance(const BatchMember *members, int count, cudaStream_t stream);
// Stochastic vacuum modes (ovl_stochastic.cu): kind 0 FP64, 1 FP32, 2 FP40
// storage; scratch_a/b: FP64 buffers of chunk_mb mode blocks each.
void launch_stochastic_modes(void *psi, void *psimid, void *psi_lo, void *psimid_lo, int kind, const Lattice &L,
                             int n_mb, int n_modes, int first_mode, double amass, double dt, uint64_t seed, int pairs,
                             double *scratch_a, double *scratch_b, int chunk_mb, cudaStream_t stream,
                             uint64_t *launches, int nc = 2);
// Lattice sums N_V, N_5, PS, WA straight from the modes (no per-site maps).
size_t charges_partial_doubles(const Lattice &L, int n_mb);
template <typename T>
void launch_charges(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                    int first_mode, double r_wilson, double *partial, double *out4, cudaStream_t stream);

// Layout conversion between the reference layout (double, [mode][site][comp])
// and the mode-block layout of precision T.  Modes [m0, m0+count); nc colours.
template <typename T>
void launch_ref_to_blocks(const double *ref, void *blocks, const Lattice &L, int m0, int count, cudaStream_t stream,
                          void *lo = nullptr, int nc = 2);
template <typename T>
void launch_blocks_to_ref(const void *blocks, double *ref, const Lattice &L, int m0, int count, cudaStream_t stream,
                          const void *lo = nullptr, int nc = 2);

// ------------------------------------------------------------------ overlap --
// Zolotarev coefficients on the host (ovl_zolotarev.cpp); returns the relative
// error estimate of the approximation.
double zolotarev(double amin, double amax, double errtol, int npoles, double *b, double *d);

constexpr int kMaxPoles = 64;
constexpr int kDotChunks = 64;  // site chunks per mode in the two-stage dot products

struct OverlapCoeffs {
    int npoles;
    double b[kMaxPoles], d[kMaxPoles];
    double cg_tol;
    int cg_max_iter;
};

// Device work space of the batched multi-shift CG (all FP64, mode-block layout).
struct OverlapWork {
    void *r = nullptr, *q = nullptr, *t = nullptr;  // one field each
    void *x = nullptr, *p = nullptr;                // npoles fields each
    double *part = nullptr;                         // kDotChunks x modes
    double *rnorm = nullptr, *bnorm = nullptr, *betam = nullptr, *pap = nullptr, *rr = nullptr;
    double *alpha = nullptr, *beta = nullptr, *z = nullptr, *g = nullptr;  // npoles x modes
    int *active = nullptr, *next = nullptr, *iters = nullptr, *count = nullptr;
    int *host_count = nullptr;                      // pinned
    double *dz = nullptr, *bz = nullptr;            // npoles
};

struct OverlapStats {
    uint64_t launches = 0;
    int iterations = 0;           // lockstep iterations of the last application
    int max_mode_iterations = 0;  // largest per-mode count
    int not_converged = 0;        // modes stopped by the iteration limit
};

// dst = out or dst += dt * out, out = -i h_ov src, for all modes.
void overlap_apply(OverlapWork &w, const double *U, const double *u1, const void *src, void *dst, const Lattice &L, int n_mb,
                   int n_modes, const OverlapCoeffs &co, double amass, double mdw, double mf, double dt,
                   bool accumulate, int sm_count, cudaStream_t stream, OverlapStats *stats);

// Chebyshev form of the overlap sign function (ovl_chebyshev.cu).
constexpr int kMaxChebDegree = 1024;
void chebyshev_inverse_sqrt(int K, double eps, double *c);
// Clenshaw vectors b0, b1, b2 and the temporary w = D b (one field each, mode
// precision).
struct ChebyshevWork {
    void *b0 = nullptr, *b1 = nullptr, *b2 = nullptr, *w = nullptr;
};
// The overlap operator with the Chebyshev series on all mode blocks; FP32 modes
// take the FP32 link copy when hc.U32 is set.
template <typename T>
void chebyshev_apply(ChebyshevWork &w, const HopConfig &hc, const void *src, void *dst, const Lattice &L, int n_mb,
                     const double *coeff, int K, double eps, double lambda_max, double amass, double mdw, double mf,
                     double dt, bool accumulate, int sm_count, cudaStream_t stream, uint64_t *launches);

// Free plane waves for local modes [0, n_modes) (global index first_mode + m):
// Wilson spinors, or overlap spinors of Wilson kernel mass -m_dw.
template <typename T>
void launch_free_fermions(void *psi, void *psimid, const Lattice &L, int n_modes, int n_mb, int first_mode,
                          double r_wilson, double m_fermion, double dt, int *bad, cudaStream_t stream,
                          void *lo_psi = nullptr, void *lo_mid = nullptr, int nc = 2, bool overlap = false,
                          double m_dw = 0.0);

// ------------------------------------------------------------ three colours --
// ovl_su3.cu; layouts in ovl_su3.cuh.  Links of the hop kernels: FP64 (U,
// u1) for FP64 modes, the FP32 copies (U32, u1_32) for FP32 modes; u1 / u1_32
// null without a U(1) background.
constexpr int kSu3Link32Floats = 20;  // FP32 link copy: 18 floats per link padded to 80 bytes
// variant: 0 the scalar three-colour stencil (one mode per thread); 3 (FP32
// with the FP32 link copy only) the packed-pair stencil (two modes per thread
// on the paired FP32 instructions, ovl_su3_packed.cuh).
struct Su3Links {
    const double *U = nullptr, *u1 = nullptr;
    const float *U32 = nullptr, *u1_32 = nullptr;
    int variant = 0;
};
template <typename T>
void su3_launch_hop(const Su3Links &lk, const void *src, void *dst, const Lattice &L, int mb0, int n_mb, double amass,
                    double dt, bool accumulate, cudaStream_t stream);
void su3_launch_update_links(double *U, const double *E, const Lattice &L, double dt_step, float *U32, bool reunit,
                             cudaStream_t stream);
void su3_launch_update_efield(const double *U, double *E, const Lattice &L, double dt_step, cudaStream_t stream);
void su3_launch_links_to_f32(const double *U, float *U32, const Lattice &L, cudaStream_t stream);
template <typename T>
void su3_chebyshev_apply(ChebyshevWork &w, const Su3Links &lk, const void *src, void *dst, const Lattice &L, int n_mb,
                         const double *coeff, int K, double eps, double lambda_max, double amass, double mdw, double mf,
                         double dt, bool accumulate, int sm_count, cudaStream_t stream, uint64_t *launches);
size_t su3_charges_partial_doubles(const Lattice &L, int n_mb);
// Per-site Wilson currents (kCurrentsPerSite values per site, as launch_currents).
template <typename T>
void su3_launch_currents(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                         int first_mode, double r_wilson, double *partial, double *per_site, cudaStream_t stream);
template <typename T>
void su3_launch_charges(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                        int first_mode, double r_wilson, double *partial, double *out4, cudaStream_t stream);
size_t su3_reduce_partial_doubles(const Lattice &L);
void su3_launch_ncsdot(const double *U, const double *E, const Lattice &L, double *partial, double *out,
                       cudaStream_t stream);
void su3_launch_geodesic(const double *Uold, const double *Unew, double c, double *Umid, double *Emid, const Lattice &L,
                         cudaStream_t stream);
void su3_launch_bulk(const double *U, const double *E, const Lattice &L, double *partial, double *out,
                     cudaStream_t stream);
// out2 = {sum of G^2, signed maximum}; G holds 8 components per site.
void su3_launch_gauss_violation(const double *U, const double *E, const Lattice &L, double *G, double *partial,
                                double *out2, cudaStream_t stream);
void su3_launch_gauss_update(const double *U, const double *G, double *E, const Lattice &L, double gamma,
                             cudaStream_t stream);
// dH_F/dtheta^a per link into out[8 per link], or E += coef * it when out is null.
size_t su3_force_partial_doubles(const Lattice &L, int n_mb);
template <typename T>
void su3_launch_color_force(const double *U, const double *u1, const void *psi, const Lattice &L, int n_mb, int n_modes,
                            int first_mode, double *partial, double *out, double *E, double coef, cudaStream_t stream);
// H_F = sum_m w_m Re <psi_m, i (D psi)_m> / 2V from psi and D psi.
template <typename T>
void su3_launch_fermion_energy(const void *psi, const void *dpsi, const Lattice &L, int n_mb, int n_modes,
                               int first_mode, double *partial, double *out, cudaStream_t stream);

}  // namespace ovl
