/* Reference harness: compiles markmace/OVERLAP's own hot-path sources (found on
 * the include path, never copied) into a shared library with a small C API.
 * TEST INFRASTRUCTURE ONLY: the product never links or calls this library; the
 * tests use it as the checker and bench.py times it as the CPU reference arm.
 *
 * Build: oracle/Makefile (one library per fermion kind, FERMION_FLAG=666 Wilson,
 * 777 overlap).  Deviations from the reference build, each forced by the tree:
 *  - stub mpi.h / gsl / fftw3.h headers (single process; see oracle/ref/stub);
 *  - restated CALC macros (oracle/ref/ovl_calc_macros.h), missing from the tree;
 *  - Dynamics::dTau is `static const 0.02` (DYNAMICS/Dynamics.cpp:17); every file
 *    included after Dynamics.cpp sees `dTau` and `Time` redirected to runtime
 *    values (harness_dt, harness_time) by macro, so the fermion leapfrog
 *    (Update.cpp, OverlapUpdate.cpp) and SetFreeFermions run at the requested dt
 *    without editing the reference.  Time() keeps its definition
 *    Qs*(tSteps*dt) (Dynamics.cpp:20-22).
 *  - the overlap build records (MinEValue, MaxEValue) each time the leapfrog
 *    reads Time(), which it does once after each half step
 *    (OverlapUpdate.cpp:110,124), so the Ritz bounds used by every half step can
 *    be handed to the GPU path. */
#include <cstdio>
#include <chrono>
#include <vector>
#include <sstream>

#include "Definitions.cpp"
#define SU_Nc_FLAG SU2_FLAG
#define METRIC_FLAG MINKOWSKI_FLAG
#ifndef FERMION_FLAG
#define FERMION_FLAG WILSON_FLAG
#endif

ovlref_reduce_hook_t ovlref_reduce_hook = nullptr;

#include "MPI/Basic.cpp"
#include "MISC/Timing.cpp"
#include "SUNc/Definitions.cpp"
#include "MISC/RNG/GSLRandomNumberGenerator.cpp"
#include "IO/StringManipulation.cpp"
#include "IO/OutputManagement.cpp"
#include "LATTICE/3DGrid.cpp"
#include "LATTICE/GaugeLinks.cpp"
#include "LATTICE/ElectricFields.cpp"
#include "LATTICE/GLinksEFields.cpp"
#include "ovl_calc_macros.h"

/* Globals the reference defines in Simulation.cpp:74,168,194-200. */
DOUBLE Qs = 1.0;
DOUBLE tSphaleron = 6.0;
DOUBLE mFermion = 0.0;
DOUBLE rWilson = 1.0;
DOUBLE MDWHeight = 1.4;
INT BFlux = 1;

#include "CALC/ChernSimonsOperators.cpp"
#include "TOPOLOGY/ChernSimonsDerivative.cpp"
#include "DYNAMICS/Dynamics.cpp"

namespace Dynamics {
DOUBLE harness_dt = 0.02;
std::vector<double> harness_bounds;
DOUBLE harness_time();
}
#define dTau harness_dt
#define Time harness_time

#include "OBSERVABLES/BulkObservables.cpp"
#include "OBSERVABLES/GaussLawViolation.cpp"
#include "OBSERVABLES/UnitarityViolation.cpp"
#include "GAUSSLAWFIXING/GaussRestore.cpp"
#include "IO/InputManagement.cpp"
#include "IO/SaveConfiguration.cpp"
#include "IO/LoadConfiguration.cpp"
/* The handmade sphaleron initial condition and what it calls
 * (INITIALCONDITIONS/HandmadeSphaleron.cpp:114-170; rSphaleron is a global of
 * Simulation.cpp:168). */
DOUBLE rSphaleron = 6.0;
#include "LATTICE/GaugeTransformations.cpp"
#include "GAUGETRANSFORMATION/GaugeTransformation.cpp"
#include "INITIALCONDITIONS/SetZero.cpp"
#include "TOPOLOGY/VacuumEstimator.cpp"
#include "LATTICE/Indexing.cpp"
#include "TOPOLOGY/WindingNumber.cpp"
#include "TOPOLOGY/IntegralEstimateMethod.cpp"
#include "INITIALCONDITIONS/HandmadeSphaleron.cpp"
#include "GRADIENTFLOW/GradientFlow.cpp"
#include "GRADIENTFLOW/Cooling.cpp"
#include "TOPOLOGY/CoolingMethod.cpp"
#include "QED/QED.cpp"
#include "DiracAlgebra.cpp"
#include "FERMIONS/FermionField.cpp"
#if FERMION_FLAG == WILSON_FLAG
#include "FERMIONS/WILSON/EvolutionOperator.cpp"
#include "FERMIONS/WILSON/Update.cpp"
#include "FERMIONS/WILSON/Currents.cpp"
#else
#include "FERMIONS/OVERLAP/OverlapEvolutionOperator.cpp"
#include "FERMIONS/OVERLAP/OverlapUpdate.cpp"
#include "FERMIONS/OVERLAP/OverlapCurrents.cpp"
#endif
#include "INITIALCONDITIONS/FERMIONS/SetFreeFermions.cpp"
#if FERMION_FLAG == OVERLAP_FLAG
/* The U(1)-background overlap eigenmodes (INITIALCONDITIONS/FERMIONS/BASIS/
 * OverlapQEDEigenfunctions.cpp): only the construction of the Hamiltonian is
 * run here.  Its Eigensystem class calls LAPACK's zheev, absent from this
 * machine: the symbol is defined below so the class links; the harness never
 * calls Diagonalize. */
#include "MISC/LapackDiagonalization.cpp"
#include "INITIALCONDITIONS/FERMIONS/BASIS/OverlapQEDEigenfunctions.cpp"
extern "C" void zheev(char const *, char const *, INT *, COMPLEX *, INT *, DOUBLE *, COMPLEX *, int *, DOUBLE *, INT *info) {
    *info = 1;  // not available
}
#endif

namespace Dynamics {
DOUBLE harness_time() {
#if FERMION_FLAG == OVERLAP_FLAG
    harness_bounds.push_back(Dynamics::Fermions::MinEValue);
    harness_bounds.push_back(Dynamics::Fermions::MaxEValue);
#endif
    return Qs * (tSteps * harness_dt);
}
}

namespace {
bool g_ready = false;
std::vector<std::vector<double>> g_reduced;
void capture_reduce(const double *data, int count) { g_reduced.emplace_back(data, data + count); }

/* Silences std::cout/std::cerr (the reference prints progress and debug lines). */
struct Quiet {
    std::streambuf *out, *err;
    std::ostringstream sink;
    Quiet() : out(std::cout.rdbuf(sink.rdbuf())), err(std::cerr.rdbuf(sink.rdbuf())) {}
    ~Quiet() { std::cout.rdbuf(out); std::cerr.rdbuf(err); }
};
}

extern "C" {

/* Sets up a lattice N0 x N1 x N2 and the mode partition of MPI rank `rank` of
 * `nranks` (MPI/ModePartition.cpp:12-24).  Returns the number of local modes,
 * or -1 when the modes do not divide evenly. */
int ovlref_init(int N0, int N1, int N2, int nranks, int rank, double m_fermion, double r_wilson,
                double m_dw, double t_sphaleron, double dt, double qs, long seed) {
    Quiet q;
    if (nranks <= 0 || rank < 0 || rank >= nranks) return -1;
    if ((2 * 2 * Nc * N0 * N1 * N2) % nranks != 0) return -1;
    Lattice::N[0] = N0; Lattice::N[1] = N1; Lattice::N[2] = N2;
    Lattice::Volume = N0 * N1 * N2;
    MPIBasic::NumberOfNodes = nranks;
    MPIBasic::ID = rank;
    mFermion = m_fermion; rWilson = r_wilson; MDWHeight = m_dw; tSphaleron = t_sphaleron; Qs = qs;
    Dynamics::harness_dt = dt;
    IO::OutputDirectory = "/dev/null/";  /* current maps are captured, not written */
    RandomNumberGenerator::Init(seed);
    Lattice::Init();
    QED::Init();
    QED::SetZero();
    Fermions::Init();
    EvolutionOperator::Init();
    Dynamics::Reset();
    GLinks::U->SetIdentity(0, 0, 0, 0);
    EFields::E->SetZero();
    Dynamics::harness_bounds.clear();
    g_ready = true;
    return MPIModePartition::ModesPerNode;
}

int ovlref_nc(void) { return Nc; }
int ovlref_first_mode(void) { return MPIModePartition::FirstIndex; }
int ovlref_local_modes(void) { return MPIModePartition::ModesPerNode; }
int ovlref_step_count(void) { return Dynamics::tSteps; }
void ovlref_set_step_count(int t) { Dynamics::tSteps = t; }

void ovlref_set_links(const double *U) {
    std::memcpy(GLinks::U->U, U, sizeof(double) * 4 * 3 * Lattice::Volume);
}
void ovlref_get_links(double *U) {
    std::memcpy(U, GLinks::U->U, sizeof(double) * 4 * 3 * Lattice::Volume);
}
void ovlref_set_efield(const double *E) {
    std::memcpy(EFields::E->E, E, sizeof(double) * 3 * 3 * Lattice::Volume);
}
void ovlref_get_efield(double *E) {
    std::memcpy(E, EFields::E->E, sizeof(double) * 3 * 3 * Lattice::Volume);
}

/* Modes in the reference layout: local mode s, site, colour, spin, (re, im)
 * (FERMIONS/FermionField.cpp:8-9,533-545). */
void ovlref_set_modes(const double *psi, const double *psimid) {
    size_t per_mode = sizeof(wcf) * Lattice::Volume;
    for (int s = 0; s < MPIModePartition::ModesPerNode; s++) {
        if (psi) std::memcpy(Fermions::Psi->GetMode(s), (const char *)psi + per_mode * s, per_mode);
        if (psimid) std::memcpy(Fermions::PsiMid->GetMode(s), (const char *)psimid + per_mode * s, per_mode);
    }
}
void ovlref_get_modes(double *psi, double *psimid) {
    size_t per_mode = sizeof(wcf) * Lattice::Volume;
    for (int s = 0; s < MPIModePartition::ModesPerNode; s++) {
        if (psi) std::memcpy((char *)psi + per_mode * s, Fermions::Psi->GetMode(s), per_mode);
        if (psimid) std::memcpy((char *)psimid + per_mode * s, Fermions::PsiMid->GetMode(s), per_mode);
    }
}

/* InitialConditions::SetFreeFermions (SetFreeFermions.cpp:59-75). */
void ovlref_set_free_fermions(void) {
    Quiet q;
    InitialConditions::SetFreeFermions(Fermions::Psi, Fermions::PsiMid);
}

/* nsteps x Dynamics::Fermions::Update (Update.cpp:48-79 / OverlapUpdate.cpp:99-135).
 * Returns wall seconds. */
double ovlref_step(int nsteps) {
    Quiet q;
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < nsteps; i++) Dynamics::Fermions::Update(GLinks::U, EFields::E, Fermions::Psi, Fermions::PsiMid);
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

/* Fermions::Observables::ComputeCurrents (Currents.cpp:396 / OverlapCurrents.cpp:292);
 * the arrays are the ones it reduces: Wilson jV,jA,jVw,jAw (4V each), PS,WA (V);
 * overlap jV,jA.  Pointers may be null.  Returns the number of arrays captured. */
int ovlref_currents(double *jV, double *jA, double *jVw, double *jAw, double *PS, double *WA) {
    Quiet q;
    g_reduced.clear();
    size_t recorded = Dynamics::harness_bounds.size();
    ovlref_reduce_hook = capture_reduce;
    Fermions::Observables::ComputeCurrents(GLinks::U, Fermions::Psi);
    ovlref_reduce_hook = nullptr;
    Dynamics::harness_bounds.resize(recorded);  /* its output lines also read Time() */
    double *outs[6] = {jV, jA, jVw, jAw, PS, WA};
    for (size_t k = 0; k < g_reduced.size() && k < 6; k++)
        if (outs[k]) std::memcpy(outs[k], g_reduced[k].data(), sizeof(double) * g_reduced[k].size());
    return (int)g_reduced.size();
}

/* ChernSimonsNumber::CoolingMethod::GetDeltaNCs(1) with zero cooling steps
 * (TOPOLOGY/CoolingMethod.cpp:37-125), from the reference's
 * GeodesicInterpolation and NCsDot; CoolingMethod.cpp itself needs the
 * gradient-flow module, so the Simpson combination of :80-125 is spelt out. */
double ovlref_delta_ncs(const double *Uold_in, const double *Unew_in) {
    GaugeLinks UOld(Lattice::N[0], Lattice::N[1], Lattice::N[2], 1, 1, 1), UNew(Lattice::N[0], Lattice::N[1], Lattice::N[2], 1, 1, 1),
        UMid(Lattice::N[0], Lattice::N[1], Lattice::N[2], 1, 1, 1);
    ElectricFields EMid(Lattice::N[0], Lattice::N[1], Lattice::N[2], 1, 1, 1);
    const size_t nl = 4 * 3 * (size_t)Lattice::Volume;
    std::memcpy(UOld.U, Uold_in, sizeof(double) * nl);
    std::memcpy(UNew.U, Unew_in, sizeof(double) * nl);
    for (INT z = 0; z < Lattice::N[2]; z++)
        for (INT y = 0; y < Lattice::N[1]; y++)
            for (INT x = 0; x < Lattice::N[0]; x++)
                for (INT mu = 0; mu < 3; mu++)
                    SUNcGroup::AdvancedOperations::GeodesicInterpolation(0.5, UOld.Get(x, y, z, mu), UNew.Get(x, y, z, mu),
                                                                         UMid.Get(x, y, z, mu), EMid.Get(x, y, z, mu, 0));
    double value = 4.0 * ChernSimonsNumber::NCsDot(&UMid, &EMid);
    value += ChernSimonsNumber::NCsDot(&UOld, &EMid);
    value += ChernSimonsNumber::NCsDot(&UNew, &EMid);
    return value / 6.0;
}

/* ChernSimonsNumber::NCsDot (TOPOLOGY/ChernSimonsDerivative.cpp:31-49). */
double ovlref_ncsdot(void) { return ChernSimonsNumber::NCsDot(GLinks::U, EFields::E); }

/* Dynamics::UpdateGaugeLinks / UpdateElectricFields over the whole lattice
 * (Dynamics.cpp:97-138, 145-197); the latter with the restated staple macros. */
void ovlref_update_links(double dt_step) {
    Dynamics::SetMetric();
    Dynamics::UpdateGaugeLinks(0, Lattice::N[0] - 1, 0, Lattice::N[1] - 1, 0, Lattice::N[2] - 1, GLinks::U, EFields::E, dt_step);
}
void ovlref_update_efield(double dt_step) {
    Dynamics::SetMetric();
    Dynamics::UpdateElectricFields(0, Lattice::N[0] - 1, 0, Lattice::N[1] - 1, 0, Lattice::N[2] - 1, GLinks::U, EFields::E, dt_step);
}

/* GaussLawRestoration::Restore (GAUSSLAWFIXING/GaussRestore.cpp:132-168) on the
 * current links and E; out2 = {GlobalMaxViolation, GlobalAvgViolation} after it. */
void ovlref_gauss_restore(double *out2) {
    Quiet q;
    GaussLawRestoration::Restore(GLinks::U, EFields::E);
    out2[0] = GaussLawRestoration::GlobalMaxViolation;
    out2[1] = GaussLawRestoration::GlobalAvgViolation;
}

/* InitialConditions::HandmadeSphaleron::Setup(GLinks::U, UFinal, EFields::E, G)
 * with rSphaleron = r_sph and tSphaleron = t_sph: the links become the unit
 * links, E the geodesic field that carries them to UFinal = G(x) G(x+mu)^+ in
 * the time t_sph.  u_final (double[V][3][4], or NULL) receives UFinal, g
 * (double[V][4], or NULL) the gauge transformation, out4 (or NULL)
 * {WindingNumber::Measure(G), WindingNumber::IntegralEstimate::Measure(G),
 *  VacuumEstimator::NCS(unit links), VacuumEstimator::NCS(UFinal)}. */
void ovlref_handmade_sphaleron(double r_sph, double t_sph, double *u_final, double *g, double *out4) {
    Quiet q;
    rSphaleron = r_sph;
    tSphaleron = t_sph;
    Dynamics::SetMetric();
    GaugeTransformations *&G = GaugeTransformation::G;
    if (G && (G->N[0] != Lattice::N[0] || G->N[1] != Lattice::N[1] || G->N[2] != Lattice::N[2])) {
        delete G;  // sized for an earlier lattice
        G = nullptr;
    }
    if (!G) GaugeTransformation::Init();
    GaugeLinks UFinal(Lattice::N[0], Lattice::N[1], Lattice::N[2], 1, 1, 1);
    InitialConditions::HandmadeSphaleron::Setup(GLinks::U, &UFinal, EFields::E, GaugeTransformation::G);
    const INT V = Lattice::Volume;
    if (u_final) std::memcpy(u_final, UFinal.U, sizeof(double) * 12 * V);
    if (g) std::memcpy(g, GaugeTransformation::G->G, sizeof(double) * 4 * V);
    if (out4) {
        out4[0] = WindingNumber::Measure(GaugeTransformation::G);
        out4[1] = WindingNumber::IntegralEstimate::Measure(GaugeTransformation::G);
        out4[2] = ChernSimonsNumber::VacuumEstimator::NCS(GLinks::U);
        out4[3] = ChernSimonsNumber::VacuumEstimator::NCS(&UFinal);
    }
}

#if FERMION_FLAG == OVERLAP_FLAG
/* The overlap Hamiltonian in the U(1) background of n_b flux quanta, built as
 * OverlapQEDEigenfunctions::Setup builds it (:141-440): links
 * ConvertU1GaugeLinks(QED::U) -- the U(1) phase in colour (0,0), every other
 * entry zero --, spectral bounds by the reference's Ritz solver
 * (ComputeRitzEigenvalues, a start vector from its RNG), then column j of
 * H = i OverlapOperator::Compute(e_j).  Setup applies the operator to a random
 * orthonormal basis and transforms back; the standard basis e_j gives the same
 * matrix without that round-off.  H: complex double[D][D] column-major,
 * D = 4 Nc V, index site + V (spin + 4 colour); bounds2 = {MinEValue, MaxEValue}. */
void ovlref_qed_hamiltonian(int n_b, double *H, double *bounds2) {
    Quiet q;
    QED::SetConstantMagneticField(n_b);
    OverlapQEDEigenfunctions::ConvertU1GaugeLinks(QED::U, EvolutionOperator::Ucc);
    Dynamics::Fermions::ComputeRitzEigenvalues();
    const DOUBLE lo = Dynamics::Fermions::MinEValue, hi = Dynamics::Fermions::MaxEValue;
    bounds2[0] = lo;
    bounds2[1] = hi;
    const INT V = Lattice::Volume, D = 4 * Nc * V;
    std::vector<wcf> in(V), out(V);
    COMPLEX *h = reinterpret_cast<COMPLEX *>(H);
    for (INT j = 0; j < D; j++) {
        std::memset(in.data(), 0, sizeof(wcf) * V);
        const INT site = j % V, spin = (j / V) % 4, colour = j / (4 * V);
        in[site].c[colour].f[spin] = COMPLEX(1.0, 0.0);
        EvolutionOperator::OverlapOperator::Compute(EvolutionOperator::Ucc, in.data(), out.data(), lo, hi);
        for (INT s = 0; s < V; s++)
            for (INT c = 0; c < Nc; c++)
                for (INT a = 0; a < 4; a++) h[(s + V * (a + 4 * c)) + (size_t)D * j] = COMPLEX(0.0, 1.0) * out[s].c[c].f[a];
    }
}
#endif

/* Observables::Bulk::Update: out[0..7] = T00, TXX, TYY, TZZ, E-part, B-part, and
 * the Gauss-law and unitarity max/avg violations (out[6..9]). */
void ovlref_bulk(double *out) {
    Dynamics::SetMetric();
    Observables::Bulk::Update(GLinks::U, EFields::E);
    out[0] = Observables::Bulk::T00();
    out[1] = Observables::Bulk::TXX();
    out[2] = Observables::Bulk::TYY();
    out[3] = Observables::Bulk::TZZ();
    out[4] = Observables::Bulk::ELECTRIC();
    out[5] = Observables::Bulk::MAGNETIC();
    Observables::GaussLaw::UpdateViolation(0, Lattice::N[0] - 1, 0, Lattice::N[1] - 1, 0, Lattice::N[2] - 1, GLinks::U, EFields::E);
    out[6] = Observables::GaussLaw::GlobalMaxViolation;
    out[7] = Observables::GaussLaw::GlobalAvgViolation;
    Observables::Unitarity::UpdateViolation(0, Lattice::N[0] - 1, 0, Lattice::N[1] - 1, 0, Lattice::N[2] - 1, GLinks::U);
    out[8] = Observables::Unitarity::GlobalMaxViolation;
    out[9] = Observables::Unitarity::GlobalAvgViolation;
}

/* IO::SaveConfiguration (IO/SaveConfiguration.cpp:3-62) of the current links
 * and E, as the reference runs it: files <dir>/<uname>ID<seed>.txt and
 * <dir>/<ename>ID<seed>.txt. */
void ovlref_save_configuration(const char *dir, long seed, const char *uname, const char *ename) {
    IO::OutputDirectory = std::string(dir) + "/";
    RandomNumberGenerator::MySEED = seed;
    IO::SaveConfiguration(uname, ename);
}

/* IO::LoadConfiguration (IO/LoadConfiguration.cpp:3-148) of <dir>/<ufile> and
 * <dir>/<efile> into the current links and E (the files must hold every link:
 * the reference exits otherwise). */
void ovlref_load_configuration(const char *dir, const char *ufile, const char *efile) {
    Dynamics::SetMetric();
    IO::InputDirectory = std::string(dir) + "/";
    IO::InputUFile = ufile;
    IO::InputEFile = efile;
    IO::LoadConfiguration(GLinks::U, EFields::E);
}

/* Gradient-flow cooling of the current links with the reference's own
 * routines: Cooling::Perform for the standard phase (CoolNSave's order: fields
 * set up, flow reset), then the calibration phase of Cooling::ContinueCooling
 * stepped here with GradientFlow::CalibrationUpdate, Observables::Bulk,
 * VacuumEstimator::NCS and Block, so that every log value is kept at full
 * precision (the reference prints them at the stream's default 6 digits).
 * log: rows {cooling time, magnetic, electric, DeltaNCsCooling, vacuum N_CS};
 * out = {DeltaNCsCooling, cooling time, blocking level}; cooled = the links
 * after the standard phase, cooledN their lattice. */
void ovlref_cool(int standard_steps, int standard_blocking, int calibration_steps, int calibration_blocking,
                 int block_frequency, double *log, int *rows, double *out, double *cooled, int *cooledN) {
    Dynamics::SetMetric();
    Cooling::BlockFrequency = block_frequency;
    Cooling::Allocate(GLinks::U);
    Cooling::DynamicFields::BlockingNumber = 0;
    Cooling::Setup(GLinks::U);
    GradientFlow::Reset();
    Cooling::Perform("ovlref_standard", standard_steps, standard_blocking, 0);
    GaugeLinks *U = Cooling::DynamicFields::U;
    for (int k = 0; k < 3; k++) cooledN[k] = U->N[k];
    std::memcpy(cooled, U->Get(0, 0, 0, 0), sizeof(double) * 4 * 3 * U->N[0] * U->N[1] * U->N[2]);
    // ContinueCooling from the cooled links (E zero), DeltaNCsCooling reset as Calibrate does
    ChernSimonsNumber::DeltaNCsCooling = 0.0;
    Cooling::DynamicFields::E->SetZero();
    int n = 0;
    auto row = [&]() {
        Observables::Bulk::Update(Cooling::DynamicFields::U, Cooling::DynamicFields::E);
        double *r = log + 5 * n++;
        r[0] = GradientFlow::CoolingTime();
        r[1] = Observables::Bulk::MAGNETIC();
        r[2] = Observables::Bulk::ELECTRIC();
        r[3] = ChernSimonsNumber::DeltaNCsCooling;
        r[4] = ChernSimonsNumber::VacuumEstimator::NCS(Cooling::DynamicFields::U);
    };
    row();
    const int total = standard_steps + calibration_steps;
    while (GradientFlow::CoolingSteps < total) {
        GradientFlow::CalibrationUpdate(Cooling::DynamicFields::U, Cooling::DynamicFields::E);
        row();
        if (GradientFlow::CoolingSteps % (Cooling::BlockFrequency * INT(std::pow(8, Cooling::DynamicFields::BlockingNumber))) == 0 &&
            Cooling::DynamicFields::BlockingNumber < calibration_blocking) {
            Block(&Cooling::DynamicFields::U);
            Block(&Cooling::DynamicFields::E);
            Cooling::DynamicFields::BlockingNumber++;
        }
    }
    *rows = n;
    out[0] = ChernSimonsNumber::DeltaNCsCooling;
    out[1] = GradientFlow::CoolingTime();
    out[2] = Cooling::DynamicFields::BlockingNumber;
    Cooling::Cleanup();
}

/* The reference driver's own calibration, unchanged (Simulation.cpp:425-431:
 * CoolingMethod::Init, Start, Calibrate) with the given schedule: the
 * reference writes <dir>/VacuumCoolingT0ID<seed>.log at 6 digits. */
void ovlref_cool_driver_log(const char *dir, long seed, int standard_steps, int standard_blocking,
                            int calibration_steps, int calibration_blocking, int block_frequency) {
    Dynamics::SetMetric();
    IO::OutputDirectory = std::string(dir) + "/";
    RandomNumberGenerator::MySEED = seed;
    Cooling::BlockFrequency = block_frequency;
    ChernSimonsNumber::CoolingMethod::StandardCoolingMaxSteps = standard_steps;
    ChernSimonsNumber::CoolingMethod::StandardBlockingLevel = standard_blocking;
    ChernSimonsNumber::CoolingMethod::CalibrationCoolingMaxSteps = calibration_steps;
    ChernSimonsNumber::CoolingMethod::CalibrationBlockingLevel = calibration_blocking;
    ChernSimonsNumber::CoolingMethod::Init();
    ChernSimonsNumber::CoolingMethod::Start();
    ChernSimonsNumber::CoolingMethod::Calibrate();
}

/* QED::SetConstantMagneticField (QED/QED.cpp:62-84); out = 2*N0*N1 complex. */
void ovlref_u1_flux(int nb, double *out) {
    QED::SetConstantMagneticField(nb);
    std::memcpy(out, QED::U, sizeof(COMPLEX) * 2 * Lattice::N[0] * Lattice::N[1]);
}

/* One application of the evolution operator -i h to a single mode in the
 * reference layout, with the current links: WilsonEvoOperator::Compute
 * (WilsonOperator.cpp:30-114) or OverlapOperator::Compute (OverlapOperator.cpp:25-65)
 * with the given spectral bounds. */
void ovlref_apply(const double *phi, double *out, double lambda_min, double lambda_max) {
    EvolutionOperator::Setup(GLinks::U);
#if FERMION_FLAG == WILSON_FLAG
    (void)lambda_min; (void)lambda_max;
    EvolutionOperator::WilsonEvoOperator::Compute(EvolutionOperator::Ucc, (wcf *)phi, (wcf *)out);
#else
    Quiet q;
    EvolutionOperator::OverlapOperator::Compute(EvolutionOperator::Ucc, (wcf *)phi, (wcf *)out, lambda_min, lambda_max);
#endif
}

#if FERMION_FLAG == OVERLAP_FLAG
/* Dynamics::Fermions::ComputeRitzEigenvalues (OverlapUpdate.cpp:61-97) on the
 * current links: out = {MinEValue, MaxEValue}. */
void ovlref_ritz_bounds(double *out) {
    Quiet q;
    EvolutionOperator::Setup(GLinks::U);
    Dynamics::Fermions::ComputeRitzEigenvalues();
    out[0] = Dynamics::Fermions::MinEValue;
    out[1] = Dynamics::Fermions::MaxEValue;
}

/* OverlapOperations::RitzSolver (RitzSolver.cpp:91-292) on the current links
 * with the reference's settings (OverlapUpdate.cpp:53-58), one eigenvalue, from
 * `start` given as one mode [V][Nc][4] complex (the solver's own order is
 * site + V (spin + 4 colour), RitzSolver.cpp:56-63). */
double ovlref_ritz_solve(const double *start, double sign) {
    Quiet q;
    EvolutionOperator::Setup(GLinks::U);
    const INT V = Lattice::N[0] * Lattice::N[1] * Lattice::N[2];
    const INT n = V * Nc * DiracAlgebra::SpinorComponents;
    std::vector<COMPLEX> v(n);
    for (INT i = 0; i < V; i++)
        for (INT j = 0; j < Nc; j++)
            for (INT k = 0; k < DiracAlgebra::SpinorComponents; k++) {
                const INT src = (i * Nc + j) * DiracAlgebra::SpinorComponents + k;
                v[i + V * (k + j * DiracAlgebra::SpinorComponents)] = COMPLEX(start[2 * src], start[2 * src + 1]);
            }
    return EvolutionOperator::OverlapOperations::RitzSolver(
        EvolutionOperator::Ucc, v.data(), Dynamics::Fermions::NumberOfEVals, Dynamics::Fermions::NormRatio,
        Dynamics::Fermions::MaximumIterations, sign, Dynamics::Fermions::NumberOfRestarts, n);
}

/* Zolotarev coefficients (ZolotarevCoefficients.cpp:71-175) with the reference's
 * tolerance and pole count (OverlapOperator.cpp:13-14): b[25], d[25]; returns eps. */
double ovlref_zolotarev(double lambda_min, double lambda_max, double *b, double *d) {
    return EvolutionOperator::OverlapOperations::ZolotarevCoefficients(
        lambda_min, lambda_max, EvolutionOperator::OverlapOperator::ZolotarevErrTol,
        EvolutionOperator::OverlapOperator::NumofZolotarevCoeffs, b, d);
}

/* (MinEValue, MaxEValue) last set by ComputeRitzEigenvalues, e.g. by the
 * ComputeCurrents call (OverlapCurrents.cpp:106-110). */
void ovlref_last_bounds(double *out) {
    out[0] = Dynamics::Fermions::MinEValue;
    out[1] = Dynamics::Fermions::MaxEValue;
}

/* Bounds recorded per half step by the leapfrog since the last call. */
int ovlref_take_bounds(double *out, int capacity) {
    int n = (int)Dynamics::harness_bounds.size();
    for (int i = 0; i < n && i < capacity; i++) out[i] = Dynamics::harness_bounds[i];
    Dynamics::harness_bounds.clear();
    return n;
}
#endif

long ovlref_rng_draws(void) { return (long)RandomNumberGenerator::Generator->draws; }

}  /* extern "C" */
