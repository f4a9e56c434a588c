/* ovl_oracle: plain-C CPU restatement of the OVERLAP fermion-gauge hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load this library, and only as the checker.
 * The product (overlap_b200) never links or calls it.
 *
 * Pinned against the reference's own code: tests/test_oracle_pin.py compares
 * every function below with the reference compiled from source
 * (oracle/_ref/libovlref_*.so, built by oracle/Makefile) and with the golden
 * vectors under tests/golden/ that the reference produced.
 *
 * Conventions (all the reference's, SU(2), lattice spacing 1, Minkowski metric):
 *   site       = x + N0*(y + N1*z)                     LATTICE/GaugeLinks.cpp:27-36
 *   links U    = double[4] per (site, mu) at 4*(mu+3*site); U = u3 + i u_k sigma_k
 *                                                      SUNc/SU2/GroupOperations.cpp:4-9
 *   E field    = double[3] per (site, mu) at a+3*(mu+3*site)   LATTICE/ElectricFields.cpp:36-42
 *   modes      = per mode V sites x [colour 2][spin 4] complex (re,im)
 *                                                      FERMIONS/FermionField.cpp:8-9
 */
#ifndef OVL_ORACLE_H
#define OVL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int N[3];
    double r_wilson;     /* rWilson */
    double m_fermion;    /* mFermion */
    double m_dw;         /* MDWHeight */
    double dt;           /* Dynamics::dTau */
    double qs;           /* Qs: Time() = qs * tsteps * dt */
    double t_sphaleron;  /* links move while Time() < t_sphaleron */
} orc_params;

/* U(1) background phases for the hopping term (the x and y links are
 * multiplied by u1[mu + 2 (x + N0 y)], complex), used by orc_wilson_apply,
 * orc_wilson_leapfrog and orc_wilson_currents until reset with NULL.  An
 * extension: the reference couples the U(1) field only into its initial
 * eigenmodes (OverlapQEDEigenfunctions.cpp:20-49). */
void orc_set_u1(const double *u1);

/* out = -i h_W phi for one mode (WilsonEvoOperator::Compute, WilsonOperator.cpp:30-114). */
void orc_wilson_apply(const orc_params *p, const double *U, const double *phi, double *out);

/* U <- exp(-i dt_step E^a t^a) U on every link (Dynamics::UpdateGaugeLinks,
 * DYNAMICS/Dynamics.cpp:97-138). */
void orc_update_links(const orc_params *p, double *U, const double *E, double dt_step);

/* E += staple force (Dynamics::UpdateElectricFields, Dynamics.cpp:145-197, with
 * the plaquette conventions of oracle/ref/ovl_calc_macros.h). */
void orc_update_efield(const orc_params *p, const double *U, double *E, double dt_step);

/* nsteps of Dynamics::Fermions::Update (FERMIONS/WILSON/Update.cpp:48-79) on
 * nmodes modes; *tsteps is the step counter read by Time(). */
void orc_wilson_leapfrog(const orc_params *p, double *U, const double *E, double *psi, double *psimid,
                         int nmodes, int *tsteps, int nsteps);

/* InitialConditions::SetFreeFermions for global modes first..first+nmodes-1
 * (SetFreeFermions.cpp:3-56, FermionField.cpp:145-328).  Returns the number of
 * modes whose eigen-residual or normalisation check failed (the reference prints
 * these, FermionField.cpp:297-312). */
int orc_free_fermions(const orc_params *p, int first, int nmodes, double *psi, double *psimid);

/* Fermions::Observables::ComputeCurrents, Wilson (FERMIONS/WILSON/Currents.cpp:7-309):
 * jV,jA,jVw,jAw: 4V doubles (component mu + 4*site), PS,WA: V doubles.  Any
 * pointer may be NULL.  first = global index of local mode 0 (vacuum sign). */
void orc_wilson_currents(const orc_params *p, const double *U, const double *psi, int nmodes, int first,
                         double *jV, double *jA, double *jVw, double *jAw, double *PS, double *WA);

/* ChernSimonsNumber::NCsDot: improved E.B / (8 pi^2)
 * (CALC/ChernSimonsOperators.cpp:128-439, TOPOLOGY/ChernSimonsDerivative.cpp:31-49). */
double orc_ncsdot(const orc_params *p, const double *U, const double *E);

/* Observables::Bulk, GaussLaw, Unitarity (OBSERVABLES/BulkObservables.cpp,
 * GaussLawViolation.cpp, UnitarityViolation.cpp):
 * out = {T00, TXX, TYY, TZZ, E part, B part, gauss max, gauss avg, unit max, unit avg}. */
void orc_bulk(const orc_params *p, const double *U, const double *E, double *out);

/* QED::SetConstantMagneticField (QED/QED.cpp:62-84): out = 2*N0*N1 complex,
 * index mu + 2*(x + N0*y). */
void orc_u1_flux(const orc_params *p, int nb, double *out);

/* Fermion back-reaction (an extension: the reference keeps E fixed in the
 * fermion loop).  out[a + 3 (mu + 3 site)] = dH_F/dtheta^a_mu(site) for
 * H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m> and U_mu -> exp(i theta^a t^a) U_mu. */
void orc_color_force(const orc_params *p, const double *U, const double *psi, int nmodes, int first, double *out);
/* H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m>. */
double orc_fermion_energy(const orc_params *p, const double *U, const double *psi, int nmodes, int first);
/* nsteps of: the reference leapfrog step, then E += dt (staple force if gauge)
 * + dt g2 dH_F/dtheta (modes and links at the integer time). */
void orc_coupled_leapfrog(const orc_params *p, double *U, double *E, double *psi, double *psimid, int nmodes, int first,
                          int *tsteps, int nsteps, double g2, int gauge);

/* RitzSolver (FERMIONS/OVERLAP/OPERATOR/RitzSolver.cpp:91-292) with one
 * eigenvalue: smallest eigenvalue of sign * h_W^2 from `start` ([V][Nc][4]
 * complex); *iters = iterations.  The reference calls it with max_iter 2000,
 * nrestart 100, delitr 1e-16 (OverlapUpdate.cpp:53-58). */
double orc_ritz(const orc_params *p, const double *U, const double *start, double sign, int max_iter, int nrestart,
                double delitr, int *iters);

/* GaussLawRestoration::Restore (GAUSSLAWFIXING/GaussRestore.cpp:132-168): the
 * reference runs max_iter 10000, tol 1e-14.  Returns the iterations; out2 =
 * {signed max, rms} of the last violation computed. */
int orc_gauss_restore(const orc_params *p, const double *U, double *E, int max_iter, double tol, double *out2);

/* InitialConditions::HandmadeSphaleron::Setup (INITIALCONDITIONS/HandmadeSphaleron.cpp:114-170)
 * with sphaleron width r_sph and transition time t_sph: the gauge transformation
 * G(x) (torus map, projection to R^3, inverse stereographic projection onto S^3,
 * :7-70) written to G (double[V][4], or NULL); U = unit links; Ufinal =
 * G(x) G(x+mu)^+ (or NULL); E = -i log(Ufinal) / t_sph (GeodesicInterpolation
 * from the unit links, :73-101). */
void orc_handmade_sphaleron(const orc_params *p, double r_sph, double t_sph, double *U, double *E, double *Ufinal,
                            double *G);

/* ---- SU(3) (three colours; no reference counterpart, see ovl_oracle.c) ----
 * links double[V][3][9][2] (U_ij at i + 3j), E double[V][3][8],
 * modes [mode][site][colour 3][spin 4][re, im]. */
void orc3_exp(double c, const double alpha[8], double out[18]);
/* Plane waves of orc_free_fermions / orc3_free_fermions: 0 Wilson spinors
 * (default), 1 overlap spinors (FermionField.cpp:331-517). */
void orc_set_free_kind(int overlap);
void orc3_wilson_apply(const orc_params *p, const double *U, const double *phi, double *out);
void orc3_update_links(const orc_params *p, double *U, const double *E, double dt_step);
void orc3_update_efield(const orc_params *p, const double *U, double *E, double dt_step);
void orc3_wilson_leapfrog(const orc_params *p, double *U, const double *E, double *psi, double *psimid, int nmodes,
                          int *tsteps, int nsteps);
int orc3_free_fermions(const orc_params *p, int first, int nmodes, double *psi, double *psimid);
void orc3_charges(const orc_params *p, const double *U, const double *psi, int nmodes, int first, double out[4]);
double orc3_ncsdot(const orc_params *p, const double *U, const double *E);
double orc3_delta_ncs(const orc_params *p, const double *Uold, const double *Unew);
void orc3_bulk(const orc_params *p, const double *U, const double *E, double *out);
int orc3_gauss_restore(const orc_params *p, const double *U, double *E, int max_iter, double tol, double *out2);
void orc3_color_force(const orc_params *p, const double *U, const double *psi, int nmodes, int first, double *out);
double orc3_fermion_energy(const orc_params *p, const double *U, const double *psi, int nmodes, int first);
void orc3_coupled_leapfrog(const orc_params *p, double *U, double *E, double *psi, double *psimid, int nmodes,
                           int first, int *tsteps, int nsteps, double g2, int gauge);
void orc_chebyshev_coeffs(int K, double eps, double *c);
void orc3_overlap_apply(const orc_params *p, const double *U, const double *phi, double *out, int K, double eps,
                        double lambda_max);
void orc3_overlap_leapfrog(const orc_params *p, double *U, const double *E, double *psi, double *psimid, int nmodes,
                           int *tsteps, int nsteps, int K, double eps, double lambda_max);

/* Gradient-flow cooling (nc = 2 or 3): the vacuum N_CS estimate
 * (TOPOLOGY/VacuumEstimator.cpp:7-85), blocking to twice the spacing
 * (LATTICE/GaugeLinks.cpp:126-153, Uout on N/2), and the standard cooling then
 * the calibration of ChernSimonsNumber::CoolingMethod (Cooling.cpp:71-201,
 * CoolingMethod.cpp:168-196) with the rows of its calibration log:
 * {cooling time, magnetic, electric, Delta N_CS, vacuum N_CS}; out = {Delta
 * N_CS, final cooling time, final blocking level}; cooled = the links after
 * the standard phase on cooled_N. */
double orc_vacuum_ncs(const orc_params *p, int nc, const double *U);
void orc_block_links(const orc_params *p, int nc, const double *U, double *Uout);
int orc_cool(const orc_params *p, int nc, const double *U0, int standard_steps, int standard_blocking,
             int calibration_steps, int calibration_blocking, int block_frequency, double *log, int *rows,
             double out[3], double *cooled, int cooled_N[3]);

#ifdef __cplusplus
}
#endif
#endif
