/* ovl.h -- C ABI of overlap_b200: the OVERLAP real-time fermion + SU(2) gauge
 * evolution hot path on one NVIDIA B200 (sm_100a).
 *
 * Plain C types only (no CUDA or torch types); every function returns an
 * ovl_status and leaves a message retrievable with ovl_last_error().  A context
 * owns one lattice, its gauge fields and one batch of fermion modes resident in
 * device memory.  A context is not thread-safe: drive each one from one host
 * thread.  Host arrays use the reference's layouts (SU(2), spacing 1):
 *
 *   links   double[V][3][4]  U = u3 + i u_k sigma_k   (LATTICE/GaugeLinks.cpp:27-36,
 *                                                       SUNc/SU2/GroupOperations.cpp:4-9)
 *   efield  double[V][3][3]  E^a_mu                    (LATTICE/ElectricFields.cpp:36-42)
 *   modes   double[M][V][2 colour][4 spin][2 re,im]    (FERMIONS/FermionField.cpp:8-9,533-545)
 *   site    x + N0*(y + N1*z)
 *
 * Mode m of a context is the reference's global mode first_mode + m; its
 * parity gives the vacuum weight +1/-1 of the current sums
 * (FERMIONS/FermionField.cpp:109-122).
 */
#ifndef OVL_H
#define OVL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Layout version of ovl_params and of the entry points; ovl_abi_version()
 * returns the value the library was built with.  A caller compiled against
 * another version must not pass its ovl_params to the library. */
#define OVL_ABI_VERSION 7

typedef enum {
    OVL_OK = 0,
    OVL_E_ARG = 1,            /* invalid argument or size */
    OVL_E_OOM = 2,            /* device allocation failed */
    OVL_E_NOT_CONVERGED = 3,  /* iterative solver hit its iteration limit */
    OVL_E_TIMEOUT = 4,        /* bounded device wait expired */
    OVL_E_NONFINITE = 5,      /* NaN/Inf detected in a field */
    OVL_E_CUDA = 6,           /* CUDA runtime error */
    OVL_E_STATE = 7,          /* call out of order (e.g. fields not set) */
    OVL_E_UNSUPPORTED = 8     /* configuration not built */
} ovl_status;

typedef enum { OVL_FERMION_WILSON = 0, OVL_FERMION_OVERLAP = 1 } ovl_fermion;

/* FP64: modes and arithmetic in FP64.  FP32: modes and hop arithmetic in FP32
 * (FP64 links).  FP40: each real of the modes stored as the top 40 bits of its
 * FP64 value (sign, exponent, 28 mantissa bits; relative rounding 2^-29), hop
 * arithmetic, observables and links in FP64: 1.25x the bytes of FP32, and an
 * axial-charge error against FP64 far below FP32's (Wilson, fused form). */
typedef enum { OVL_PREC_FP64 = 0, OVL_PREC_FP32 = 1, OVL_PREC_FP40 = 2 } ovl_precision;

/* OVL_FORM_PLAIN keeps the reference's two-phase half step (Update.cpp:6-27):
 * the operator writes a derivative buffer, then psi += dt * derivative.
 * OVL_FORM_FUSED applies psi_dst += dt * D psi_src in one pass. */
typedef enum { OVL_FORM_PLAIN = 0, OVL_FORM_FUSED = 1 } ovl_form;

typedef struct {
    int N[3];             /* lattice extents N0, N1, N2 */
    int n_colours;        /* colours: 2 (SU(2), the reference's) or 3 (SU(3): links 9 complex
                             doubles per (site, mu) at U_ij = i + 3j, SUNc/SU3/GroupOperations.cpp:4-12;
                             E 8 per (site, mu); modes [mode][site][colour 3][spin 4]) */
    int n_modes;          /* modes held by this context */
    int first_mode;       /* global index of local mode 0 (MPI/ModePartition.cpp:12-24) */
    int fermion;          /* ovl_fermion */
    int precision;        /* ovl_precision of the modes and of the hopping arithmetic */
    int form;             /* ovl_form */
    double r_wilson;      /* rWilson */
    double m_fermion;     /* mFermion */
    double m_dw;          /* MDWHeight; the Wilson mass is 6r + 2m - 2 MDWHeight (WilsonOperator.cpp:39) */
    double dt;            /* Dynamics::dTau */
    double qs;            /* Qs: Time() = qs * steps * dt (Dynamics.cpp:20-22) */
    double t_sphaleron;   /* links move while Time() < t_sphaleron (Update.cpp:57-60) */
    int device;           /* CUDA device ordinal */
    int plain_chunk_modes;/* OVL_FORM_PLAIN: modes per derivative-buffer chunk (0 = all) */
    uint64_t stream;      /* cudaStream_t to issue work on; 0 = the context creates its own */
    /* overlap sign function (FERMIONS/OVERLAP/OPERATOR/OverlapOperator.cpp:13-18) */
    int zolo_poles;       /* NumofZolotarevCoeffs = 25 */
    double zolo_tol;      /* ZolotarevErrTol = 1e-12 */
    int cg_max_iter;      /* MaximumCGIter = 1000 */
    double cg_tol;        /* ConGradErr = 1e-16 */
    /* OVL_SIGN_ZOLOTAREV (the reference's rational approximation, FP64) or
     * OVL_SIGN_CHEBYSHEV: (h_W^2)^(-1/2) as a degree-cheb_degree Chebyshev
     * series of x^(-1/2) on [cheb_eps, 1] after scaling h_W^2 by lambda_max
     * (FP32 or FP64).  With ritz_auto lambda_max = 1.05 times the Ritz estimate
     * (ovl_ritz_bounds) before every application; without a bounds schedule or
     * ritz_auto lambda_max = (|6r + 2m - 2M|/2 + 3)^2, a bound on h_W^2 for every
     * gauge field.  Three colours: Chebyshev only. */
    int sign_method;
    int cheb_degree;
    double cheb_eps;
    /* Leapfrog hop kernel variant: -1 = time the variants on the first step and
     * keep the fastest (ovl_autotune); 0 .. OVL_HOP_VARIANTS-1 = fixed (3: FP32
     * only).  All variants apply the same operator; they differ in the order
     * of the FP32/FP64 roundings only. */
    int hop_variant;
    /* 1: project every link back onto SU(2) after each update (U / |U|,
     * MaxTraceProjection, SUNc/SU2/GroupOperations.cpp:261-281), or onto SU(3)
     * (Gram-Schmidt of the rows, unit determinant).  The reference
     * only measures the unitarity violation (OBSERVABLES/UnitarityViolation.cpp),
     * so 0 reproduces it. */
    int reunitarize;
    /* Coupled gauge + fermion evolution (no reference counterpart: the
     * reference keeps E fixed under the fermion loop, FERMIONS/WILSON/Update.cpp:48-79).
     * After each leapfrog step, E += dt (gauge_force ? staple force : 0)
     *                             + dt backreaction dH_F/dtheta
     * from the links and modes at the end of the step, with
     * H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m> (ovl_fermion_energy) and
     * backreaction the coupling g^2; H_gauge + g^2 H_F is then conserved to
     * O(dt^2).  0 and 0 reproduce the reference.  Wilson fermions only. */
    int gauge_force;
    double backreaction;
    /* Overlap spectral bounds when no schedule is set (ovl_set_spectral_bounds):
     * 1 = compute them on the GPU before every overlap application, as
     * Dynamics::Fermions::ComputeRitzEigenvalues does before every half step and
     * every current measurement (OverlapUpdate.cpp:100-125,
     * OverlapCurrents.cpp:106-110), from a fresh start vector drawn from the
     * context's generator (seed ritz_seed); 0 = an unset schedule is an error. */
    int ritz_auto;
    uint64_t ritz_seed;
    /* Fused Wilson form: the two half steps of a leapfrog step run group by
     * group of mode_group mode blocks (32 modes each), so that a group's fields,
     * written by the first half step, are still in L2 when the second reads
     * them (4 instead of 6 field passes through HBM per step; the same
     * arithmetic, so the same results).  0 (default) = whole batch per half
     * step; k > 0 = k blocks; -1 = chosen by the autotuner with the hop
     * variant.  On B200 at 16^3 the launch overhead of the groups outweighs the
     * L2 reuse, and the autotuner keeps the whole batch. */
    int mode_group;
} ovl_params;

typedef enum { OVL_SIGN_ZOLOTAREV = 0, OVL_SIGN_CHEBYSHEV = 1 } ovl_sign_method;

typedef struct ovl_ctx ovl_ctx;

/* Fills p with the reference's defaults (Simulation.cpp:74,168,194-200,
 * Dynamics.cpp:17): SU(2) Wilson, FP64 plain, r = 1, m = 0, MDWHeight = 1.4,
 * dt = 0.02, Qs = 1, tSphaleron = 6. */
int ovl_params_init(ovl_params *p);

/* OVL_ABI_VERSION of the library (compare with the header's before
 * ovl_params_init). */
int ovl_abi_version(void);

/* Allocates the device state for p.  Replaces Lattice::Init, Fermions::Init and
 * EvolutionOperator::Init (Simulation.cpp:251-307, FermionField.cpp:632-641). */
int ovl_create(const ovl_params *p, ovl_ctx **out);
int ovl_destroy(ovl_ctx *ctx);
const char *ovl_last_error(const ovl_ctx *ctx);

/* Gauge fields, host <-> device, reference layouts (GLinks::U->U, EFields::E->E). */
/* The uploads return once the host array may be reused: at once for pageable
 * memory (the copy has been staged), after the copy for page-locked memory. */
int ovl_set_links(ovl_ctx *ctx, const double *links);
int ovl_get_links(ovl_ctx *ctx, double *links);
int ovl_set_efield(ovl_ctx *ctx, const double *efield);
int ovl_get_efield(ovl_ctx *ctx, double *efield);

/* U(1) background of the hopping term: u1 = complex double[N1][N0][2] (re, im),
 * index mu + 2 (x + N0 y), the layout of QED::U (QED/QED.cpp:6-23); the x and y
 * links of every z slice are multiplied by these phases, the z links by 1.
 * NULL removes the background.  In the reference the U(1) field enters only the
 * initial eigenmodes (INITIALCONDITIONS/FERMIONS/BASIS/OverlapQEDEigenfunctions.cpp:20-49);
 * coupling it into the evolution is an extension without a reference counterpart.
 * QED::SetConstantMagneticField (QED.cpp:62-84) gives the flux-n_B field. */
int ovl_set_u1(ovl_ctx *ctx, const double *u1);

/* Modes first..first+count-1 of Psi / PsiMid in the reference layout; either
 * pointer may be NULL to skip that field.  Replaces writing
 * Fermions::Psi/PsiMid->GetMode(s) on the host. */
int ovl_set_modes(ovl_ctx *ctx, int first, int count, const double *psi, const double *psimid);
int ovl_get_modes(ovl_ctx *ctx, int first, int count, double *psi, double *psimid);

/* InitialConditions::SetFreeFermions (INITIALCONDITIONS/FERMIONS/SetFreeFermions.cpp:3-56):
 * free Wilson plane waves, computed on the device.  *n_bad receives the number of
 * modes failing the eigen-residual/normalisation self-check (FermionField.cpp:270-312). */
int ovl_set_free_fermions(ovl_ctx *ctx, int *n_bad);

/* Spectral bounds (lambda_min, lambda_max) of h_W^2 that place the Zolotarev
 * approximation of the overlap sign function, as pairs[2*i], pairs[2*i+1] for
 * the i-th overlap application (two per leapfrog step, one per ovl_currents
 * call), consumed in order; with count == 1 the one pair serves every
 * application.  Replaces Dynamics::Fermions::ComputeRitzEigenvalues
 * (FERMIONS/OVERLAP/OverlapUpdate.cpp:61-97), whose Ritz iteration starts from
 * a random vector drawn from the reference's RNG. */
int ovl_set_spectral_bounds(ovl_ctx *ctx, const double *pairs, int count);

/* out = D phi for `count` modes given in the reference layout (host), with the
 * context's current links: D = -i h_W, WilsonEvoOperator::Compute
 * (FERMIONS/WILSON/OPERATOR/WilsonOperator.cpp:30-114), or D = -i h_ov,
 * OverlapOperator::Compute (FERMIONS/OVERLAP/OPERATOR/OverlapOperator.cpp:25-65),
 * using the current spectral bounds without consuming them.  The context's
 * modes are not touched. */
int ovl_apply(ovl_ctx *ctx, int count, const double *phi, double *out);

/* Times the hop-kernel variants of the leapfrog half step on this context's
 * fields (its state is not changed) and keeps the fastest for later steps:
 * 0 = one site per warp (32 modes), 8 consecutive sites per CTA; 1 = the same
 * on a 4 x 2 (x, y) tile of sites per CTA; 2 = (x, y) columns marching in z
 * with register reuse; 3 (FP32 only) = two modes per thread on the paired
 * FP32 instructions, links built once per CTA in shared memory.  *variant
 * receives the choice, ms[v] the time of one half step with variant v (0 for
 * a variant the precision does not have). */
#define OVL_HOP_VARIANTS 4
int ovl_autotune(ovl_ctx *ctx, int *variant, double ms[OVL_HOP_VARIANTS]);

/* Failure-detection self-test of the pipelined grouped step (FP32 Wilson
 * modes, hop variant 3, at least two mode blocks): runs one pipelined pass on
 * the operator buffers with the first group's first-half tiles never handed
 * out, so the second-half tiles that wait on them give up after their bounded
 * wait (1 s) and set the error word.  *code receives what ovl_step would have
 * returned (OVL_E_TIMEOUT when the detection works).  The context's modes and
 * links are not touched. */
int ovl_pipeline_selftest(ovl_ctx *ctx, int *code);

/* The hop variant and mode grouping in use (after the autotuner ran, or as
 * set in ovl_params); -1 before either is known. */
int ovl_tuning(const ovl_ctx *ctx, int *variant, int *mode_group);

/* Zolotarev coefficients of the overlap sign function for spectral bounds
 * [lambda_min, lambda_max] of h_W^2: (h_W^2)^(-1/2) ~ sum_l b[l] / (h_W^2 + d[l]),
 * l < npoles (OverlapOperations::ZolotarevCoefficients,
 * FERMIONS/OVERLAP/OPERATOR/ZolotarevCoefficients.cpp:71-175).  *eps receives the
 * relative error estimate of the approximation on the interval. */
int ovl_zolotarev(double lambda_min, double lambda_max, double tol, int npoles, double *b, double *d, double *eps);

/* Dynamics::Fermions::ComputeRitzEigenvalues (OverlapUpdate.cpp:61-97) on the
 * GPU: OverlapOperations::RitzSolver (OPERATOR/RitzSolver.cpp:91-292) with the
 * reference's settings (one eigenvalue, 2000 iterations, restarts every 100,
 * NormRatio 1e-16) for the smallest and the largest eigenvalue of h_W^2 on the
 * context's links, both from `start` (one mode, complex [V][Nc][4]; NULL: a
 * vector of the reference's distribution from the context's generator).
 * out = {MinEValue, MaxEValue} = {0.95 lambda_min, 1.05 lambda_max};
 * raw = {lambda_min, lambda_max} and iters = iterations per problem when not
 * NULL.  Works for both fermion kinds (the Wilson kernel of the context) and
 * both colour counts (the reference's solver is written for two; for three
 * the same iteration runs on the three-colour h_W^2, start [V][3][4]). */
int ovl_ritz_bounds(ovl_ctx *ctx, const double *start, double out[2], double raw[2], int iters[2]);

/* Statistics of the last overlap application.  Zolotarev: out[0] = lockstep
 * CG iterations, out[1] = largest per-mode iteration count, out[2] = modes
 * stopped by cg_max_iter (the reference prints a warning and keeps the
 * result, OverlapU.cpp:113-117).  Chebyshev: out[0] = out[1] = degree,
 * out[2] = 1 when the bounds put lambda_min below cheb_eps * lambda_max (the
 * spectrum leaves the approximation interval). */
int ovl_solver_stats(const ovl_ctx *ctx, int out[3]);

/* nsteps x Dynamics::Fermions::Update(U, E, Psi, PsiMid)
 * (FERMIONS/WILSON/Update.cpp:48-79; overlap: FERMIONS/OVERLAP/OverlapUpdate.cpp:99-135):
 * psi += dt D(psimid); links half step while Time() < tSphaleron;
 * psimid += dt D(psi); links half step; step counter + 1.
 * Asynchronous on the context's stream (overlap: synchronises once per CG iteration).
 * OVL_E_TIMEOUT (only the pipelined grouped step, FP32 hop variant 3 with
 * mode_group > 0, waits on the device) is read once at the end of the call:
 * the modes and the step counter are then undefined, and the caller restores
 * them from its last saved state. */
int ovl_step(ovl_ctx *ctx, int nsteps);

/* nsteps leapfrog steps as ovl_step, returning out = {N_V, N_5, PS} of the
 * modes at the end (ovl_charges' first three values): in the fused Wilson form
 * (two colours) they are summed inside the last step's second half step, which
 * reads psi anyway, so the observation costs no extra pass over the modes
 * (Currents.cpp:44-92 bilinears; the Wilson-term sum WA needs ovl_charges);
 * in every other form the steps are followed by the charges kernel. */
int ovl_step_observe(ovl_ctx *ctx, int nsteps, double out[3]);

/* Leapfrog step counter Dynamics::tSteps. */
int ovl_get_step_count(const ovl_ctx *ctx, int *steps);
int ovl_set_step_count(ovl_ctx *ctx, int steps);

/* Fermions::Observables::ComputeCurrents (FERMIONS/WILSON/Currents.cpp:7-309) of
 * this context's modes, i.e. the arrays it MPI_Reduces (:326-333): jV, jA, jVw, jAw
 * double[V][4]; PS, WA double[V].  NULL pointers are skipped.  Overlap contexts
 * compute the overlap currents (FERMIONS/OVERLAP/OverlapCurrents.cpp:5-290): jV, jA
 * with the -i/2 g0 G g0 h_ov term; jVw, jAw, PS, WA are zero. */
int ovl_currents(ovl_ctx *ctx, double *jV, double *jA, double *jVw, double *jAw, double *PS, double *WA);

/* Lattice sums of the current densities: out[0] = sum_x jV^0 (vector charge),
 * out[1] = sum_x jA^0 (axial charge N_5), out[2] = sum_x PS, out[3] = sum_x WA. */
int ovl_charges(ovl_ctx *ctx, double out[4]);

/* ChernSimonsNumber::NCsDot(U, E): improved E.B / (8 pi^2)
 * (TOPOLOGY/ChernSimonsDerivative.cpp:31-49, CALC/ChernSimonsOperators.cpp:128-439). */
int ovl_ncsdot(ovl_ctx *ctx, double *out);

/* ChernSimonsNumber::CoolingMethod::Update(1) with cooling switched off (the
 * production driver runs it with zero cooling steps, Simulation.cpp:258,504-511):
 * the change of the Chern-Simons number between the links stored by the
 * previous call (U_old) and the current links (U_new), by the Simpson rule of
 * GetDeltaNCs(1) (TOPOLOGY/CoolingMethod.cpp:80-125) along the geodesic
 * U_old -> U_new; then U_old = U_new.  *delta receives the change and *total the
 * running sum DeltaNCsCoolRealTime.  The first call only stores U_old
 * (CoolingMethod::Start) and returns 0. */
int ovl_ncs_update(ovl_ctx *ctx, double *delta, double *total);

/* Stochastic vacuum modes in place of the complete plane-wave basis (no
 * reference counterpart): modes 2r and 2r+1 (global index) are P+ eta_r and
 * P- eta_r times sqrt(V / total_pairs) (the plane-wave modes have
 * |psi(x)|^2 = 1 per site), with eta_r complex Z2 noise
 * ((+-1 +- i)/sqrt 2 per component, drawn in momentum space from `seed`) and
 * P+- the projectors on the positive- and negative-energy states of the free
 * Wilson Hamiltonian (those the plane-wave particles and antiparticles span);
 * psimid = exp(-i h dt/2) psi.  The vacuum-weighted mode sums of the currents
 * are then unbiased estimates of the complete basis's, and the free vacuum
 * energy is reproduced exactly.  total_pairs: pairs over all contexts that
 * share the estimate (0: n_modes / 2 of this one; first_mode and n_modes even). */
int ovl_set_stochastic_modes(ovl_ctx *ctx, uint64_t seed, int total_pairs);

/* Dynamics::UpdateGaugeLinks over the whole lattice (DYNAMICS/Dynamics.cpp:97-138):
 * U <- exp(-i dt_step E^a t^a) U. */
int ovl_update_links(ovl_ctx *ctx, double dt_step);

/* Dynamics::UpdateElectricFields over the whole lattice (Dynamics.cpp:145-197):
 * E_mu += -2 dt_step sum over the staples of U_mu of Re tr(i t^a U_plaq). */
int ovl_update_efield(ovl_ctx *ctx, double dt_step);

/* Fermion force on the links: out[a + 3 (mu + 3 site)] = dH_F/dtheta^a_mu(site)
 * for U_mu(site) -> exp(i theta^a t^a) U_mu(site) and
 * H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m> (mode weights w_m as the
 * currents, FermionField.cpp:109-122).  No reference counterpart.  Wilson only. */
int ovl_color_force(ovl_ctx *ctx, double *out);

/* H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m> of the current modes and links.
 * No reference counterpart.  Wilson only. */
int ovl_fermion_energy(ovl_ctx *ctx, double *out);

/* InitialConditions::HandmadeSphaleron::Setup (INITIALCONDITIONS/HandmadeSphaleron.cpp:114-170),
 * the production driver's gauge start (Simulation.cpp:580): the links become
 * the unit links and E the field that carries them, by the link update of the
 * leapfrog, to the pure gauge G(x) G(x+mu)^+ in the time t_sphaleron, with
 * G(x) in SU(2) from the reference's map of the lattice torus onto S^3 of
 * width r_sphaleron (rSphaleron, Simulation.cpp:168).  u_final (host
 * double[V][3][4], or NULL) receives G(x) G(x+mu)^+.  Create the context with
 * t_sphaleron equal to the transition time, so the leapfrog moves the links
 * while Time() < t_sphaleron and stops at the final ones.  Two colours. */
int ovl_set_handmade_sphaleron(ovl_ctx *ctx, double r_sphaleron, double t_sphaleron, double *u_final);

/* InitialConditions::SetOverlapQEDEigenfunctions (INITIALCONDITIONS/FERMIONS/
 * SetOverlapQEDEigenfunctions.cpp:5-86), the reference's production fermion
 * start: the context's modes become eigenmodes of the overlap Hamiltonian of
 * OverlapQEDEigenfunctions::Setup (BASIS/OverlapQEDEigenfunctions.cpp:141-591)
 * -- links carrying the context's U(1) background (ovl_set_u1; none: phases 1)
 * in colour (0,0) and zero elsewhere, as ConvertU1GaugeLinks sets them --
 * with global mode g at particle index g % 2 and level g / 2: particles on the
 * positive eigenvalues from the smallest up, antiparticles on the negative ones
 * from the one nearest zero down; psi = sqrt(V) v, psimid = psi e^{-i omega dt/2}.
 * The reference reconstructs h_ov from overlap applications (Zolotarev sign
 * function) and calls LAPACK's zheev; here h_ov is built densely with the
 * exact sign function and diagonalised on the device (cuSOLVER), so it agrees
 * with the reference's to the accuracy of the reference's approximation.
 * Eigenvectors are defined up to a phase (and within a degenerate level up to
 * a unitary mixing): the modes' bilinears summed over complete levels do not
 * depend on that choice.  eigenvalues (host double[D], D = 8 V, or NULL):
 * ascending; h_ov (host complex double[D][D] column-major, index
 * site + V (spin + 4 colour), or NULL): the matrix; *n_bad (or NULL): modes
 * whose frequency has the wrong sign for their particle index, plus zero
 * eigenvalues of h_W.  Two-colour overlap contexts with first_mode + n_modes <= D;
 * dense D x D matrices limit it to D^2 < 2^31 (lattices up to about 16^3). */
int ovl_set_qed_eigenmodes(ovl_ctx *ctx, double *eigenvalues, double *h_ov, int *n_bad);

/* InitialConditions::SetQuasiParticles (INITIALCONDITIONS/SetQuasiParticles.cpp:28-220)
 * on the device, unit spacing, Minkowski metric, two or three colours:
 * transverse gauge-field modes with occupancy n0 / sqrt(p^2/Qs^2 + 0.1) below
 * qs (zero above), E = i omega A per mode, backward Fourier transform, links
 * U = exp(-i A^a t^a); then, when gauss_max_iter > 0, GaussLawRestoration::Restore
 * with tolerance 1e-14 (as SetQuasiParticles does; *iterations receives its
 * iterations).  The complex Gaussian amplitudes of each (momentum, colour
 * component) come from a counter-based generator keyed by `seed` (SplitMix64
 * with Box-Muller; the reference draws them from GSL in loop order), so the
 * fields are reproducible and independent of the launch shape. */
int ovl_set_quasi_particles(ovl_ctx *ctx, double n0, double qs, uint64_t seed, int gauss_max_iter, int *iterations);

/* GaussLawRestoration::Restore (GAUSSLAWFIXING/GaussRestore.cpp:132-168) on the
 * context's links and E: while the signed maximum of the Gauss-law violation
 * exceeds tol and fewer than max_iter iterations ran, three damped steps
 * E_mu -= gamma (G(x) - U_mu(x) G(x+mu) U_mu(x)^+), gamma = 7/24, 7/48, 7/72.
 * The reference uses max_iter 10000, tol 1e-14.  *iterations = iterations
 * run; out = {signed max, rms} of the last violation computed (either may be
 * NULL). */
int ovl_gauss_restore(ovl_ctx *ctx, int max_iter, double tol, int *iterations, double out[2]);

/* Gradient-flow cooling of a copy of the context's links and the Chern-Simons
 * calibration along it: ChernSimonsNumber::CoolingMethod's standard cooling
 * (Cooling::CoolNSave, GRADIENTFLOW/Cooling.cpp:162-183) followed by its
 * calibration (CoolingMethod::Calibrate -> Cooling::ContinueCooling,
 * TOPOLOGY/CoolingMethod.cpp:168-196, Cooling.cpp:185-199).
 *   Standard phase: the links, E = 0, cooling time and step count reset;
 *   standard_steps steps of GradientFlow::StandardUpdate
 *   (GRADIENTFLOW/GradientFlow.cpp:35-175), blocking to twice the lattice
 *   spacing (LATTICE/GaugeLinks.cpp:126-153) after every step whose count is a
 *   multiple of block_frequency 8^level while level < standard_blocking.
 *   Calibration phase: from the cooled links, E = 0, Delta N_CS = 0, the count
 *   and time continuing, steps of GradientFlow::CalibrationUpdate up to
 *   standard_steps + calibration_steps in all, blocking while level <
 *   calibration_blocking; each step adds DcTau/2 NCsDot(U, E) before and after
 *   its link update.
 * log (may be NULL): calibration_steps + 1 rows of 5 doubles, the rows of the
 * reference's calibration log (Cooling.cpp:87-108): cooling time, magnetic and
 * electric energy (Observables::Bulk at the current spacing), Delta N_CS along
 * the calibration path so far, and the vacuum N_CS estimate
 * (TOPOLOGY/VacuumEstimator.cpp:7-85) -- before the first step and after each.
 * *log_rows = rows written; out = {Delta N_CS along the calibration path,
 * cooling time at the end, blocking level at the end}; cooled_links (may be
 * NULL; room for the context's links suffices) receives the links after the
 * standard phase, on the lattice cooled_N (may be NULL).  The context's own
 * links are not changed.  Each blocking needs every lattice extent >= 2 when
 * it happens (OVL_E_ARG before anything runs otherwise).  The reference's
 * driver (Simulation.cpp:258-265) calls this with block_frequency 32, standard_blocking 0 and
 * calibration_blocking 2. */
int ovl_cool(ovl_ctx *ctx, int standard_steps, int standard_blocking, int calibration_steps, int calibration_blocking,
             int block_frequency, double *log, int *log_rows, double out[3], double *cooled_links, int cooled_N[3]);

/* The context's links and E written as the reference's configuration files
 * (IO::SaveConfiguration, IO/SaveConfiguration.cpp:3-62): one line per link,
 * z outermost, then y, x and the direction mu innermost.  Link file: "x y z
 * mu " and the link's numbers each followed by a space (two colours: the four
 * real parameters in the layout of ovl_set_links; three colours: the nine
 * elements as "re im" pairs); E file: "x y z mu" and the Nc^2-1 components,
 * each preceded by a space.  Numbers as %.15g (the reference's
 * OUTPUT_PRECISION of 15 digits).  A NULL path skips that file.  File names
 * are the caller's (the reference composes "UOutT<t>ID<seed>.txt"). */
int ovl_save_configuration(ovl_ctx *ctx, const char *u_path, const char *e_path);

/* IO::LoadConfiguration (IO/LoadConfiguration.cpp:3-148): reads link and E
 * files in that format (lines in any order, blank lines skipped) into the
 * context.  Every link must appear exactly once, inside the lattice; the
 * reference exits when the count is wrong, this returns OVL_E_ARG naming the
 * file and line and leaves both fields unchanged.  A NULL path skips that
 * field.  Non-finite numbers give OVL_E_NONFINITE. */
int ovl_load_configuration(ovl_ctx *ctx, const char *u_path, const char *e_path);

/* Observables::Bulk::Update + GaussLaw + Unitarity (OBSERVABLES/BulkObservables.cpp:133-143,
 * GaussLawViolation.cpp:13-61, UnitarityViolation.cpp:13-51):
 * out = {T00, TXX, TYY, TZZ, electric, magnetic, gauss max, gauss avg, unitarity max, unitarity avg}. */
int ovl_bulk(ovl_ctx *ctx, double out[10]);

/* Waits for all work queued on the context's stream; reports OVL_E_TIMEOUT
 * for a pipelined half step queued by ovl_step_observe_async that timed out. */
int ovl_synchronize(ovl_ctx *ctx);

/* Asynchronous forms for callers that keep the GPU busy across steps (a step
 * loop that uploads each step's gauge fields and reads each step's charges):
 * the work is queued on the context's stream and the call returns.
 * ovl_upload_gauge_async: ovl_set_links and ovl_set_efield (either may be
 * NULL) from page-locked host memory (OVL_E_ARG otherwise), which the copy
 * reads until the stream reaches it: keep the buffers unchanged until then
 * (ovl_synchronize, or an event recorded on the stream after the call).
 * ovl_step_observe_async: ovl_step_observe with its three charges copied into
 * `out`, page-locked host memory (OVL_E_ARG otherwise), valid once the
 * stream has passed the call.  Fused two-colour Wilson forms queue without
 * waiting; the other forms complete before returning.  No counterpart in the
 * reference (its steps are synchronous). */
int ovl_upload_gauge_async(ovl_ctx *ctx, const double *links, const double *efield);
int ovl_step_observe_async(ovl_ctx *ctx, int nsteps, double *out);

/* Device addresses and layout of the mode fields, for callers that keep their
 * own device buffers.  Layout: [mode/32][site][colour*4+spin][mode%32] complex of
 * the context precision (float2 or double2); *bytes is the size of one field. */
int ovl_device_modes(ovl_ctx *ctx, void **psi, void **psimid, size_t *bytes);

/* NCsDot of fields the caller already holds in device memory, computed without
 * allocating anything; the only entry point without a counterpart in the
 * reference.  For callers that cannot allocate device memory: a time-step loop
 * that must never block on an allocation, or code whose device memory belongs
 * to another allocator.  links: device double[V][3][4], efield: device
 * double[V][3][3], out: device double[1]; work is queued on `stream`
 * (a cudaStream_t, 0 for the default stream) of the current device.  Scratch is
 * a fixed 8 KiB device array inside the library, so lattices above 262144
 * sites (64^3) are rejected with OVL_E_ARG.  The first call on a device looks
 * up that array's address: make it before any stream capture.  Calls share the
 * array: calls that overlap on the GPU race and must be serialised.  Devices
 * with an ordinal of 64 or more give OVL_E_UNSUPPORTED; a failed launch gives
 * OVL_E_CUDA, while a CUDA error left pending by other work is not reported
 * (nor cleared) by this call. */
int ovl_ncsdot_noalloc(const double *links, const double *efield, int N0, int N1, int N2, double *out,
                       uint64_t stream);

/* Number of CUDA kernel launches this context has issued (for launch accounting). */
int ovl_launch_count(const ovl_ctx *ctx, uint64_t *count);

/* Per-kernel timing with CUDA events recorded on the context's stream around
 * each launch.  Kinds: */
enum {
    OVL_PROF_HOP = 0,      /* Wilson operator kernel (fused half step or derivative) */
    OVL_PROF_AXPY = 1,     /* plain form: psi += dt * derivative */
    OVL_PROF_LINKS = 2,    /* link update */
    OVL_PROF_OBS = 3,      /* currents / charges / NCsDot / bulk */
    OVL_PROF_KINDS = 4
};
/* Turns recording on (1) or off (0); turning it on clears earlier records. */
int ovl_profile_enable(ovl_ctx *ctx, int on);
/* Synchronises the stream and returns, per kind, the summed kernel time in ms
 * and the number of launches timed since recording was enabled. */
int ovl_profile_read(ovl_ctx *ctx, double ms[OVL_PROF_KINDS], uint64_t launches[OVL_PROF_KINDS]);

/* ------------------------------------------------------------ ensembles --
 * An ensemble: independent trajectories (members), each a context of its own
 * lattice size, mode count, physics and gauge fields, advanced together.  A
 * leapfrog step of all members is one launch for all hop work per half step,
 * one launch for all link updates per half step and one for the step counters
 * (Update.cpp:48-79 per member, its tSphaleron gate evaluated on the device),
 * captured once as a CUDA graph and replayed per step.  The reference has no
 * counterpart: its MPI ranks split the modes of one trajectory.  Members:
 * Wilson fermions, fused form, FP32 or FP64 (one precision and device for
 * all), no coupled evolution.  Members are set up and measured through their
 * contexts (ovl_ensemble_member; do not destroy them: the ensemble owns them).
 * The ensemble's stream is members[0].stream when not 0 (the caller keeps it
 * alive until ovl_ensemble_destroy; a stream of high priority puts the
 * ensemble's kernels ahead of other streams' on the GPU), else a non-blocking
 * stream of its own; all members run on it (their own streams are ignored). */
typedef struct ovl_ensemble ovl_ensemble;
int ovl_ensemble_create(const ovl_params *members, int count, ovl_ensemble **out);
int ovl_ensemble_destroy(ovl_ensemble *ens);
const char *ovl_ensemble_last_error(const ovl_ensemble *ens);
int ovl_ensemble_member(ovl_ensemble *ens, int index, ovl_ctx **ctx);
/* nsteps leapfrog steps of every member.  Unless a tile shape was set
 * (ovl_ensemble_set_tile), the first call times the tile shapes of the batched
 * hop on the members' operator buffers and keeps the fastest. */
int ovl_ensemble_step(ovl_ensemble *ens, int nsteps);
/* Tile shape of the batched hop: 0 = time them on the next step (the
 * default); 8 or 4 = that many sites x 32 modes per CTA, a warp per site;
 * 16 = packed-pair tiles (8 sites x 256 modes per CTA) for FP32 two-colour members
 * (the kernel body of hop variant 3: two modes per thread on the paired FP32
 * instructions; the other members use tiles of 8).  The packed tiles lose a
 * short timing to the 8-site tiles but draw less power per mode-site, which
 * wins sustained runs under the power cap. */
#define OVL_ENSEMBLE_TILES 3
int ovl_ensemble_set_tile(ovl_ensemble *ens, int sites);
/* Continuous batching: add a member (created on the ensemble's device and
 * stream, same precision; *index = its position) or remove member `index`
 * (its context is destroyed; later members move down by one).  Either makes
 * the next step capture its graph again. */
int ovl_ensemble_add(ovl_ensemble *ens, const ovl_params *member, int *index);
int ovl_ensemble_remove(ovl_ensemble *ens, int index);
int ovl_ensemble_size(const ovl_ensemble *ens);
/* ovl_charges of every member: out[4 i + k]. */
int ovl_ensemble_charges(ovl_ensemble *ens, double *out);
/* Tile shape in use (0 before the first step), the tuning times (ms, for 8,
 * 4 and 16 (packed, FP32 only) sites; 0 where not timed) and the kernels
 * launched. */
int ovl_ensemble_info(const ovl_ensemble *ens, int *sites, double tile_ms[OVL_ENSEMBLE_TILES], uint64_t *launches);
int ovl_ensemble_synchronize(ovl_ensemble *ens);
/* The ensemble's CUDA stream (cudaStream_t as an integer). */
uint64_t ovl_ensemble_stream(const ovl_ensemble *ens);

#ifdef __cplusplus
}
#endif
#endif
