// Drop-in test program: the reference's own Simulation-style build with its
// fermion hot path replaced by include/ovl_dropin.hpp and its gauge routines
// (NCsDot, UpdateGaugeLinks, UpdateElectricFields) by include/ovl_dropin_gauge.hpp
// (the GPU path), the way a maintainer of the reference would include them.
// Built twice by tests/dropin/Makefile where the reference tree exists: with
// the Wilson fermions (ovl_dropin_test) and with OVL_TEST_OVERLAP defined, the
// overlap fermions (ovl_dropin_overlap_test).  Test infrastructure, run by
// tests/test_gpu_dropin.py, which compares the fermion results with the
// reference compiled from source.  The gauge routines are checked in this
// process: the reference's own definitions stay in the build under the names
// the renaming macros give them, and run on the same fields.
//
// usage: ovl_dropin_test N0 N1 N2 nranks rank m r mdw tsph dt steps in.bin out.bin
//   in.bin : links double[V*12] then efield double[V*9]
//   out.bin: psi, psimid (local modes, reference layout), links, the current
//            arrays of ComputeCurrents (captured at MPI_Reduce: six for Wilson,
//            jV and jA for overlap), then NCsDot (drop-in, reference), E after
//            UpdateElectricFields(dt) (drop-in, reference), U after
//            UpdateGaugeLinks(dt) (drop-in, reference), all on the input fields
#include <cstdio>
#include <sstream>
#include <vector>

#include "Definitions.cpp"
#define SU_Nc_FLAG SU2_FLAG
#define METRIC_FLAG MINKOWSKI_FLAG
#ifdef OVL_TEST_OVERLAP
#define FERMION_FLAG OVERLAP_FLAG
#else
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
DOUBLE Qs = 1.0;
DOUBLE tSphaleron = 6.0;
DOUBLE mFermion = 0.0;
DOUBLE rWilson = 1.0;
DOUBLE MDWHeight = 1.4;
INT BFlux = 1;
#include "CALC/ChernSimonsOperators.cpp"
#define NCsDot OVL_ReferenceNCsDot
#include "TOPOLOGY/ChernSimonsDerivative.cpp"
#undef NCsDot
#define UpdateGaugeLinks OVL_ReferenceUpdateGaugeLinks
#define UpdateElectricFields OVL_ReferenceUpdateElectricFields
#define Update OVL_ReferenceUpdate
#include "DYNAMICS/Dynamics.cpp"
#undef UpdateGaugeLinks
#undef UpdateElectricFields
#undef Update
namespace Dynamics {
DOUBLE harness_dt = 0.02;
DOUBLE harness_time() { return Qs * (tSteps * harness_dt); }
}
#define dTau harness_dt
#define Time harness_time
#include "ovl_dropin_gauge.hpp"  // NCsDot, UpdateGaugeLinks, UpdateElectricFields, Update on the GPU
#include "QED/QED.cpp"
#include "DiracAlgebra.cpp"
#include "FERMIONS/FermionField.cpp"
#include "ovl_dropin.hpp"  // in place of the fermion kind's EvolutionOperator, Update and Currents files
#include "INITIALCONDITIONS/FERMIONS/SetFreeFermions.cpp"

static std::vector<std::vector<double>> g_reduced;
static void capture(const double *d, int n) { g_reduced.emplace_back(d, d + n); }

int main(int argc, char **argv) {
    if (argc != 14) { std::fprintf(stderr, "bad arguments\n"); return 2; }
    const int N0 = std::atoi(argv[1]), N1 = std::atoi(argv[2]), N2 = std::atoi(argv[3]);
    Lattice::N[0] = N0; Lattice::N[1] = N1; Lattice::N[2] = N2;
    Lattice::Volume = N0 * N1 * N2;
    MPIBasic::NumberOfNodes = std::atoi(argv[4]);
    MPIBasic::ID = std::atoi(argv[5]);
    mFermion = std::atof(argv[6]); rWilson = std::atof(argv[7]); MDWHeight = std::atof(argv[8]);
    tSphaleron = std::atof(argv[9]); Dynamics::harness_dt = std::atof(argv[10]);
    const int steps = std::atoi(argv[11]);
    IO::OutputDirectory = "/dev/null/";
    RandomNumberGenerator::Init(1);
    Lattice::Init();
    QED::Init();
    Fermions::Init();
    EvolutionOperator::Init();
    Dynamics::Reset();
    const INT V = Lattice::Volume;
    FILE *in = std::fopen(argv[12], "rb");
    if (!in) return 3;
    if (std::fread(GLinks::U->U, sizeof(double), 12 * V, in) != (size_t)(12 * V)) return 3;
    if (std::fread(EFields::E->E, sizeof(double), 9 * V, in) != (size_t)(9 * V)) return 3;
    std::fclose(in);
    // the gauge routines, drop-in and reference, on the input fields
    const std::vector<double> U0(GLinks::U->U, GLinks::U->U + 12 * V), E0(EFields::E->E, EFields::E->E + 9 * V);
    const double dt = Dynamics::harness_dt;
    const double ncs[2] = {ChernSimonsNumber::NCsDot(GLinks::U, EFields::E),
                           ChernSimonsNumber::OVL_ReferenceNCsDot(GLinks::U, EFields::E)};
    std::vector<double> gauge_out[4];
    for (int k = 0; k < 2; k++) {  // E after UpdateElectricFields: drop-in, reference
        std::copy(E0.begin(), E0.end(), EFields::E->E);
        if (k == 0) Dynamics::UpdateElectricFields(0, N0 - 1, 0, N1 - 1, 0, N2 - 1, GLinks::U, EFields::E, dt);
        else Dynamics::OVL_ReferenceUpdateElectricFields(0, N0 - 1, 0, N1 - 1, 0, N2 - 1, GLinks::U, EFields::E, dt);
        gauge_out[k].assign(EFields::E->E, EFields::E->E + 9 * V);
    }
    std::copy(E0.begin(), E0.end(), EFields::E->E);
    for (int k = 0; k < 2; k++) {  // U after UpdateGaugeLinks: drop-in, reference
        std::copy(U0.begin(), U0.end(), GLinks::U->U);
        if (k == 0) Dynamics::UpdateGaugeLinks(0, N0 - 1, 0, N1 - 1, 0, N2 - 1, GLinks::U, EFields::E, dt);
        else Dynamics::OVL_ReferenceUpdateGaugeLinks(0, N0 - 1, 0, N1 - 1, 0, N2 - 1, GLinks::U, EFields::E, dt);
        gauge_out[2 + k].assign(GLinks::U->U, GLinks::U->U + 12 * V);
    }
    std::copy(U0.begin(), U0.end(), GLinks::U->U);
    std::ostringstream quiet;
    std::streambuf *err = std::cerr.rdbuf(quiet.rdbuf());
    InitialConditions::SetFreeFermions(Fermions::Psi, Fermions::PsiMid);
    for (int t = 0; t < steps; t++) Dynamics::Fermions::Update(GLinks::U, EFields::E, Fermions::Psi, Fermions::PsiMid);
    ovlref_reduce_hook = capture;
    Fermions::Observables::ComputeCurrents(GLinks::U, Fermions::Psi);
    ovlref_reduce_hook = nullptr;
    std::cerr.rdbuf(err);
    ovl_dropin::SyncModesToHost(Fermions::Psi, Fermions::PsiMid);
    FILE *out = std::fopen(argv[13], "wb");
    if (!out) return 4;
    for (INT s = 0; s < MPIModePartition::ModesPerNode; s++) std::fwrite(Fermions::Psi->GetMode(s), sizeof(double), 16 * V, out);
    for (INT s = 0; s < MPIModePartition::ModesPerNode; s++) std::fwrite(Fermions::PsiMid->GetMode(s), sizeof(double), 16 * V, out);
    std::fwrite(GLinks::U->U, sizeof(double), 12 * V, out);
    for (auto &a : g_reduced) std::fwrite(a.data(), sizeof(double), a.size(), out);
    std::fwrite(ncs, sizeof(double), 2, out);
    for (auto &a : gauge_out) std::fwrite(a.data(), sizeof(double), a.size(), out);
    std::fclose(out);
    std::printf("%d %d\n", MPIModePartition::FirstIndex, MPIModePartition::ModesPerNode);
    return 0;
}
