// ovl_dropin.hpp -- drop-in replacement, inside the reference's own build, of
// the Wilson fermion hot path of markmace/OVERLAP by the overlap_b200 GPU path.
//
// Include it in Simulation.cpp in place of
//     #include "FERMIONS/WILSON/EvolutionOperator.cpp"
//     #include "FERMIONS/WILSON/Update.cpp"
//     #include "FERMIONS/WILSON/Currents.cpp"
// (Simulation.cpp includes them through its FERMION_FLAG == WILSON_FLAG branch)
// and link with -lovl_b200.  It must come after the reference's lattice, field
// and Dynamics headers, exactly where those three files were included.  It
// defines, with the reference's signatures and meaning:
//
//   void Dynamics::Fermions::Update(GaugeLinks*, ElectricFields*, FermionField*, FermionField*)
//                                                        FERMIONS/WILSON/Update.cpp:48-79
//   void Fermions::Observables::ComputeCurrents(GaugeLinks*, FermionField*)
//                                                        FERMIONS/WILSON/Currents.cpp:396-400
//   namespace EvolutionOperator { Init, Setup }          FERMIONS/WILSON/EvolutionOperator.cpp:12-57
//
// State: the first Update creates one device context sized from Lattice::N,
// MPIModePartition (this rank's mode slice) and the globals mFermion, rWilson,
// MDWHeight, tSphaleron, Qs and Dynamics::dTau, and uploads Psi and PsiMid.
// From then on the modes live on the GPU; the host copies in Psi/PsiMid are
// stale until ovl_dropin::SyncModesToHost is called.  Every Update uploads the
// host links and E field, advances one leapfrog step on the GPU, downloads the
// links (the step moves them while Time() < tSphaleron) and increments
// Dynamics::tSteps, as the reference does.  ComputeCurrents evaluates the
// current maps on the GPU and writes the reference's text files.
// Errors print the C ABI message and exit, as the reference does on errors.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

#include "ovl.h"

namespace ovl_dropin {

inline ovl_ctx *&context() {
    static ovl_ctx *ctx = nullptr;
    return ctx;
}

inline void check(int rc, const char *what) {
    if (rc != OVL_OK) {
        std::cerr << "#ERROR overlap_b200 " << what << ": " << ovl_last_error(context()) << std::endl;
        std::exit(1);
    }
}

inline void UploadModes(FermionField *Psi, FermionField *PsiMid) {
    const INT V = Psi->Volume;
    std::vector<double> a((size_t)V * 16 * Psi->NumberOfSamples), b(a.size());
    for (INT s = 0; s < Psi->NumberOfSamples; s++) {
        std::memcpy(&a[(size_t)s * V * 16], Psi->GetMode(s), sizeof(double) * 16 * V);
        std::memcpy(&b[(size_t)s * V * 16], PsiMid->GetMode(s), sizeof(double) * 16 * V);
    }
    check(ovl_set_modes(context(), 0, Psi->NumberOfSamples, a.data(), b.data()), "ovl_set_modes");
}

// Copies the device modes back into the reference's FermionField objects.
inline void SyncModesToHost(FermionField *Psi, FermionField *PsiMid) {
    if (!context()) return;
    const INT V = Psi->Volume;
    std::vector<double> a((size_t)V * 16 * Psi->NumberOfSamples), b(a.size());
    check(ovl_get_modes(context(), 0, Psi->NumberOfSamples, a.data(), b.data()), "ovl_get_modes");
    for (INT s = 0; s < Psi->NumberOfSamples; s++) {
        std::memcpy(Psi->GetMode(s), &a[(size_t)s * V * 16], sizeof(double) * 16 * V);
        std::memcpy(PsiMid->GetMode(s), &b[(size_t)s * V * 16], sizeof(double) * 16 * V);
    }
}

inline void Create(FermionField *Psi, FermionField *PsiMid, int precision, int form) {
    ovl_params p;
    if (ovl_abi_version() != OVL_ABI_VERSION) {
        std::fprintf(stderr, "ovl_dropin: libovl_b200 ABI %d, header %d: rebuild\n", ovl_abi_version(), OVL_ABI_VERSION);
        std::exit(1);
    }
    ovl_params_init(&p);
    p.N[0] = Lattice::N[0];
    p.N[1] = Lattice::N[1];
    p.N[2] = Lattice::N[2];
    p.n_colours = Nc;
    p.n_modes = MPIModePartition::ModesPerNode;
    p.first_mode = MPIModePartition::FirstIndex;
    p.precision = precision;
    p.form = form;
    p.r_wilson = rWilson;
    p.m_fermion = mFermion;
    p.m_dw = MDWHeight;
    p.dt = Dynamics::dTau;
    p.qs = Qs;
    p.t_sphaleron = tSphaleron;
    p.device = 0;
    check(ovl_create(&p, &context()), "ovl_create");
    UploadModes(Psi, PsiMid);
}

// Precision and form of the context the first Update creates.
inline int &precision() { static int v = OVL_PREC_FP64; return v; }
inline int &form() { static int v = OVL_FORM_FUSED; return v; }

}  // namespace ovl_dropin

// The u_cc link copy of the reference (EvolutionOperator.cpp:12-57) is not
// needed: the GPU reads the 4-real links directly.
namespace EvolutionOperator {
inline void Init() {}
inline void Setup(GaugeLinks *) {}
}  // namespace EvolutionOperator

namespace Dynamics {
namespace Fermions {

inline void Update(GaugeLinks *U, ElectricFields *E, FermionField *Psi, FermionField *PsiMid) {
    using namespace ovl_dropin;
    if (!context()) Create(Psi, PsiMid, precision(), form());
    ovl_ctx *ctx = context();
    check(ovl_set_links(ctx, U->U), "ovl_set_links");
    check(ovl_set_efield(ctx, E->E), "ovl_set_efield");
    check(ovl_set_step_count(ctx, Dynamics::tSteps), "ovl_set_step_count");
    check(ovl_step(ctx, 1), "ovl_step");
    check(ovl_get_links(ctx, U->U), "ovl_get_links");
    tSteps++;
    MPI_Barrier(MPI_COMM_WORLD);
}

}  // namespace Fermions
}  // namespace Dynamics

namespace Fermions {
namespace Observables {

// Current maps on the GPU; output files as FERMIONS/WILSON/Currents.cpp:338-373.
inline void ComputeCurrents(GaugeLinks *U, FermionField *Psi) {
    using namespace ovl_dropin;
    const INT V = Psi->Volume;
    std::vector<double> jV(4 * V), jA(4 * V), jVw(4 * V), jAw(4 * V), PS(V), WA(V);
    if (!context()) Create(Psi, Fermions::PsiMid, precision(), form());
    check(ovl_set_links(context(), U->U), "ovl_set_links");
    check(ovl_currents(context(), jV.data(), jA.data(), jVw.data(), jAw.data(), PS.data(), WA.data()), "ovl_currents");
    std::vector<double> g[6];
    double *loc[6] = {jV.data(), jA.data(), jVw.data(), jAw.data(), PS.data(), WA.data()};
    const INT len[6] = {4 * V, 4 * V, 4 * V, 4 * V, V, V};
    for (int k = 0; k < 6; k++) {
        g[k].resize(len[k]);
        MPI_Reduce(loc[k], g[k].data(), len[k], MPI_DOUBLE, MPI_SUM, 0, MPI_COMM_WORLD);
    }
    if (MPIBasic::ID != 0) return;
    const DOUBLE t = Dynamics::Time();
    std::ofstream vec(StringManipulation::StringCast(IO::OutputDirectory, "VectorCurrentT", t, ".txt").c_str());
    std::ofstream ax(StringManipulation::StringCast(IO::OutputDirectory, "AxialCurrentT", t, ".txt").c_str());
    std::ofstream ps(StringManipulation::StringCast(IO::OutputDirectory, "PseudoScalarT", t, ".txt").c_str());
    std::ofstream wa(StringManipulation::StringCast(IO::OutputDirectory, "WilsonAnomalyT", t, ".txt").c_str());
    for (INT z = 0; z < Psi->N[2]; z++) {
        for (INT y = 0; y < Psi->N[1]; y++) {
            for (INT x = 0; x < Psi->N[0]; x++) {
                const INT s = Psi->Index3D(x, y, z);
                vec << t << " " << x << " " << y << " " << z;
                for (int mu = 0; mu < 4; mu++) vec << " " << g[0][mu + 4 * s];
                for (int mu = 0; mu < 4; mu++) vec << " " << g[2][mu + 4 * s];
                vec << std::endl;
                ax << t << " " << x << " " << y << " " << z;
                for (int mu = 0; mu < 4; mu++) ax << " " << g[1][mu + 4 * s];
                for (int mu = 0; mu < 4; mu++) ax << " " << g[3][mu + 4 * s];
                ax << std::endl;
                ps << t << " " << x << " " << y << " " << z << " " << g[4][s] << std::endl;
                wa << t << " " << x << " " << y << " " << z << " " << g[5][s] << std::endl;
            }
            vec << std::endl; ax << std::endl; ps << std::endl; wa << std::endl;
        }
        vec << std::endl; ax << std::endl; ps << std::endl; wa << std::endl;
    }
}

inline void ComputeCurrents(INT, INT, INT, INT, INT, INT, GaugeLinks *U, FermionField *Psi) { ComputeCurrents(U, Psi); }

}  // namespace Observables
}  // namespace Fermions
