// ovl_dropin.hpp -- drop-in replacement, inside the reference's own build, of
// the fermion hot path of markmace/OVERLAP by the overlap_b200 GPU path.  The
// reference's FERMION_FLAG selects which half this header defines.
//
// Wilson build (FERMION_FLAG == WILSON_FLAG): include it in Simulation.cpp in
// place of
//     #include "FERMIONS/WILSON/EvolutionOperator.cpp"
//     #include "FERMIONS/WILSON/Update.cpp"
//     #include "FERMIONS/WILSON/Currents.cpp"
// It defines, with the reference's signatures and meaning:
//   void Dynamics::Fermions::Update(GaugeLinks*, ElectricFields*, FermionField*, FermionField*)
//                                                        FERMIONS/WILSON/Update.cpp:48-79
//   void Fermions::Observables::ComputeCurrents(GaugeLinks*, FermionField*)
//                                                        FERMIONS/WILSON/Currents.cpp:396-400
//   namespace EvolutionOperator { Init, Setup }          FERMIONS/WILSON/EvolutionOperator.cpp:12-57
//
// Overlap build (FERMION_FLAG == OVERLAP_FLAG): include it in place of
//     #include "FERMIONS/OVERLAP/OverlapEvolutionOperator.cpp"
//     #include "FERMIONS/OVERLAP/OverlapUpdate.cpp"
//     #include "FERMIONS/OVERLAP/OverlapCurrents.cpp"
// It defines:
//   void Dynamics::Fermions::Update(GaugeLinks*, ElectricFields*, FermionField*, FermionField*)
//                                                        FERMIONS/OVERLAP/OverlapUpdate.cpp:99-135
//   void Dynamics::Fermions::ComputeRitzEigenvalues(), DOUBLE MinEValue, MaxEValue
//                                                        FERMIONS/OVERLAP/OverlapUpdate.cpp:61-97
//   void Fermions::Observables::ComputeCurrents(GaugeLinks*, FermionField*) and the
//        bounded overload                                FERMIONS/OVERLAP/OverlapCurrents.cpp:5-296
//   u_cc, EvolutionOperator::Ucc, Init, ConvertGaugeLinks, Setup
//                                                        FERMIONS/OVERLAP/OverlapEvolutionOperator.cpp:1-57
//   void EvolutionOperator::OverlapOperator::Compute(u_cc*, wcf*, wcf*, DOUBLE, DOUBLE)
//                                                        FERMIONS/OVERLAP/OPERATOR/OverlapOperator.cpp:25-65
// The overlap sign function is the reference's (25-pole Zolotarev rational
// function, multi-shift CG with its tolerances); the spectral bounds of every
// half step and current measurement come from the GPU's Ritz solver started
// from the context's own generator, so the reference's RNG is not drawn from
// (its bounds agree with the reference's to round-off, and the evolution to
// 1e-10).
//
// Either build must come after the reference's lattice, field and Dynamics
// headers, exactly where the replaced files were included, and links with
// -lovl_b200.  The gauge routines the fermion loop calls
// (Dynamics::UpdateGaugeLinks and the others) run on the host unless
// ovl_dropin_gauge.hpp replaces them too.
//
// State: the first Update (or ComputeCurrents) creates one device context sized
// from Lattice::N, MPIModePartition (this rank's mode slice) and the globals
// mFermion, rWilson, MDWHeight, tSphaleron, Qs and Dynamics::dTau, and uploads
// Psi and PsiMid.  From then on the modes live on the GPU; the host copies in
// Psi/PsiMid are stale until ovl_dropin::SyncModesToHost is called.  Every
// Update uploads the host links and E field, advances one leapfrog step on the
// GPU and, while Time() < tSphaleron (the only time the step moves them),
// downloads the links; it increments Dynamics::tSteps, as the reference does.
// ComputeCurrents evaluates the current maps on the GPU and writes the
// reference's text files.  Errors print the C ABI message and exit, as the
// reference does on errors.
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
    const bool overlap = FERMION_FLAG == OVERLAP_FLAG;
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
    if (overlap) {
        // the reference's sign function and its Ritz bounds before every
        // overlap application (OverlapOperator.cpp:13-18, OverlapUpdate.cpp:100-125)
        p.fermion = OVL_FERMION_OVERLAP;
        p.sign_method = OVL_SIGN_ZOLOTAREV;
        p.precision = OVL_PREC_FP64;
        p.ritz_auto = 1;
        p.ritz_seed = 20261203;
    }
    check(ovl_create(&p, &context()), "ovl_create");
    UploadModes(Psi, PsiMid);
}

// Links of the step: while Time() < tSphaleron the step moves them
// (Update.cpp:57-60, OverlapUpdate.cpp:111-113), afterwards they are unchanged
// and need not come back.
inline void StepOnce(GaugeLinks *U, ElectricFields *E) {
    ovl_ctx *ctx = context();
    const bool moves = Dynamics::Time() < tSphaleron;
    check(ovl_set_links(ctx, U->U), "ovl_set_links");
    check(ovl_set_efield(ctx, E->E), "ovl_set_efield");
    check(ovl_set_step_count(ctx, Dynamics::tSteps), "ovl_set_step_count");
    check(ovl_step(ctx, 1), "ovl_step");
    if (moves) check(ovl_get_links(ctx, U->U), "ovl_get_links");
}

// Precision and form of the context the first Update creates.
inline int &precision() { static int v = OVL_PREC_FP64; return v; }
inline int &form() { static int v = OVL_FORM_FUSED; return v; }

}  // namespace ovl_dropin

#if FERMION_FLAG == WILSON_FLAG

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
    StepOnce(U, E);
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

#endif  // FERMION_FLAG == WILSON_FLAG

#if FERMION_FLAG == OVERLAP_FLAG

#ifndef GAUGEF_H_GUARD
#define GAUGEF_H_GUARD
typedef struct { COMPLEX c[2]; } u_c;
typedef struct { u_c c[2]; } u_cc;
#endif

namespace ovl_dropin {

// Applications of OverlapOperator::Compute outside the leapfrog (the
// reference's initial conditions call it with links and bounds of their own):
// a context of its own whose bounds and links each call sets.
inline ovl_ctx *&operator_context() {
    static ovl_ctx *ctx = nullptr;
    return ctx;
}

inline void ucc_to_links(const u_cc *u, std::vector<double> &links) {
    // the inverse of ConvertGaugeLinks (OverlapEvolutionOperator.cpp:23-53) with
    // GetMatrix's convention (SUNc/SU2/GroupOperations.cpp:213-225):
    // c[0][0] = u3 + i u2, c[1][0] = -u1 + i u0
    const INT V = Lattice::N[0] * Lattice::N[1] * Lattice::N[2];
    links.resize((size_t)12 * V);
    for (INT s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            const u_cc &m = u[s + mu * V];
            double *q = &links[4 * (mu + 3 * (size_t)s)];
            q[0] = m.c[1].c[0].imag();
            q[1] = -m.c[1].c[0].real();
            q[2] = m.c[0].c[0].imag();
            q[3] = m.c[0].c[0].real();
        }
}

}  // namespace ovl_dropin

namespace EvolutionOperator {

// The reference's u_cc copy of the links (OverlapEvolutionOperator.cpp:9-57),
// kept for callers outside the leapfrog that pass it to OverlapOperator::Compute;
// the GPU leapfrog reads the 4-real links directly.
u_cc *Ucc = nullptr;

inline void Init() { Ucc = new u_cc[Lattice::N[0] * Lattice::N[1] * Lattice::N[2] * Lattice::Dimension]; }

inline void ConvertGaugeLinks(GaugeLinks *U, u_cc *UccLinks) {
    const INT V = U->N[0] * U->N[1] * U->N[2];
    for (INT s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            const double *q = &U->U[4 * (mu + 3 * (size_t)s)];
            u_cc &m = UccLinks[s + mu * V];
            m.c[0].c[0] = COMPLEX(q[3], q[2]);
            m.c[0].c[1] = COMPLEX(q[1], q[0]);
            m.c[1].c[0] = COMPLEX(-q[1], q[0]);
            m.c[1].c[1] = COMPLEX(q[3], -q[2]);
        }
}

inline void Setup(GaugeLinks *U) { ConvertGaugeLinks(U, Ucc); }

namespace OverlapOperator {

// psi = -i h_ov phi for one mode with links u and spectral bounds
// [LambdaMin, LambdaMax] of h_W^2 (the reference's Zolotarev coefficients and
// multi-shift CG), on the GPU.  Unlike the reference it draws nothing from the
// reference's RNG (the reference fills an unused random vector there).
inline void Compute(u_cc *u, wcf *phi, wcf *psi, DOUBLE LambdaMin, DOUBLE LambdaMax) {
    using namespace ovl_dropin;
    if (!operator_context()) {
        ovl_params p;
        ovl_params_init(&p);
        p.N[0] = Lattice::N[0];
        p.N[1] = Lattice::N[1];
        p.N[2] = Lattice::N[2];
        p.n_colours = Nc;
        p.n_modes = 1;
        p.fermion = OVL_FERMION_OVERLAP;
        p.sign_method = OVL_SIGN_ZOLOTAREV;
        p.precision = OVL_PREC_FP64;
        p.r_wilson = rWilson;
        p.m_fermion = mFermion;
        p.m_dw = MDWHeight;
        p.device = 0;
        if (ovl_create(&p, &operator_context()) != OVL_OK) {
            std::cerr << "#ERROR overlap_b200 ovl_create (overlap operator): " << ovl_last_error(nullptr) << std::endl;
            std::exit(1);
        }
    }
    ovl_ctx *ctx = operator_context();
    auto ok = [&](int rc, const char *what) {
        if (rc != OVL_OK) {
            std::cerr << "#ERROR overlap_b200 " << what << ": " << ovl_last_error(ctx) << std::endl;
            std::exit(1);
        }
    };
    std::vector<double> links;
    ucc_to_links(u, links);
    ok(ovl_set_links(ctx, links.data()), "ovl_set_links");
    const double bounds[2] = {LambdaMin, LambdaMax};
    ok(ovl_set_spectral_bounds(ctx, bounds, 1), "ovl_set_spectral_bounds");
    ok(ovl_apply(ctx, 1, reinterpret_cast<const double *>(phi), reinterpret_cast<double *>(psi)), "ovl_apply");
}

}  // namespace OverlapOperator
}  // namespace EvolutionOperator

namespace Dynamics {
namespace Fermions {

// The spectral bounds of the last ComputeRitzEigenvalues (the GPU leapfrog and
// currents compute their own before every overlap application).
DOUBLE MinEValue = 0.0, MaxEValue = 0.0;

// MinEValue = 0.95 lambda_min, MaxEValue = 1.05 lambda_max of h_W^2 on the
// current host links, by the reference's Ritz iteration on the GPU
// (ovl_ritz_bounds, from a start vector of the context's generator).
inline void ComputeRitzEigenvalues() {
    using namespace ovl_dropin;
    if (!context()) Create(::Fermions::Psi, ::Fermions::PsiMid, precision(), form());
    check(ovl_set_links(context(), GLinks::U->U), "ovl_set_links");
    double out[2];
    check(ovl_ritz_bounds(context(), nullptr, out, nullptr, nullptr), "ovl_ritz_bounds");
    MinEValue = out[0];
    MaxEValue = out[1];
}

inline void Update(GaugeLinks *U, ElectricFields *E, FermionField *Psi, FermionField *PsiMid) {
    using namespace ovl_dropin;
    if (!context()) Create(Psi, PsiMid, precision(), form());
    StepOnce(U, E);
    tSteps++;
    MPI_Barrier(MPI_COMM_WORLD);
}

}  // namespace Fermions
}  // namespace Dynamics

namespace Fermions {
namespace Observables {

// Overlap current maps jV, jA on the GPU (the local bilinears with the
// -i/2 g0 G g0 h_ov correction, OverlapCurrents.cpp:5-290), reduced over the
// MPI ranks and written as the reference writes them.
inline void ComputeCurrents(INT xLow, INT xHigh, INT yLow, INT yHigh, INT zLow, INT zHigh, GaugeLinks *U,
                            FermionField *Psi) {
    using namespace ovl_dropin;
    const INT V = Psi->Volume;
    std::vector<double> jV(4 * V), jA(4 * V);
    if (!context()) Create(Psi, ::Fermions::PsiMid, precision(), form());
    check(ovl_set_links(context(), U->U), "ovl_set_links");
    check(ovl_currents(context(), jV.data(), jA.data(), nullptr, nullptr, nullptr, nullptr), "ovl_currents");
    MPI_Barrier(MPI_COMM_WORLD);
    std::vector<double> gV(4 * V), gA(4 * V);
    MPI_Reduce(jV.data(), gV.data(), 4 * V, MPI_DOUBLE, MPI_SUM, 0, MPI_COMM_WORLD);
    MPI_Reduce(jA.data(), gA.data(), 4 * V, MPI_DOUBLE, MPI_SUM, 0, MPI_COMM_WORLD);
    if (MPIBasic::ID != 0) return;
    const DOUBLE t = Dynamics::Time();
    std::ofstream vec(StringManipulation::StringCast(IO::OutputDirectory, "VectorCurrentT", t, ".txt").c_str());
    std::ofstream ax(StringManipulation::StringCast(IO::OutputDirectory, "AxialCurrentT", t, ".txt").c_str());
    for (INT z = zLow; z <= zHigh; z++) {
        for (INT y = yLow; y <= yHigh; y++) {
            for (INT x = xLow; x <= xHigh; x++) {
                const INT s = Psi->Index3D(x, y, z);
                vec << t << " " << x << " " << y << " " << z;
                ax << t << " " << x << " " << y << " " << z;
                for (int mu = 0; mu < 4; mu++) {
                    vec << " " << gV[mu + 4 * s];
                    ax << " " << gA[mu + 4 * s];
                }
                vec << std::endl;
                ax << std::endl;
            }
            vec << std::endl;
            ax << std::endl;
        }
        vec << std::endl;
        ax << std::endl;
    }
}

inline void ComputeCurrents(GaugeLinks *U, FermionField *Psi) {
    ComputeCurrents(0, Psi->N[0] - 1, 0, Psi->N[1] - 1, 0, Psi->N[2] - 1, U, Psi);
}

}  // namespace Observables
}  // namespace Fermions

#endif  // FERMION_FLAG == OVERLAP_FLAG
