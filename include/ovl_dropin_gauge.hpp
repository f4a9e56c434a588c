// ovl_dropin_gauge.hpp -- drop-in replacement, inside the reference's own
// build, of the gauge-field routines of markmace/OVERLAP that the fermion loop
// and its observables call, by the overlap_b200 GPU path:
//
//   DOUBLE ChernSimonsNumber::NCsDot(GaugeLinks*, ElectricFields*)
//                                                  TOPOLOGY/ChernSimonsDerivative.cpp:31-49
//   void Dynamics::UpdateGaugeLinks(INT xLow, INT xHigh, INT yLow, INT yHigh, INT zLow, INT zHigh,
//                                   GaugeLinks*, ElectricFields*, DOUBLE dTauStep)
//                                                  DYNAMICS/Dynamics.cpp:97-138
//   void Dynamics::UpdateElectricFields(INT xLow, ..., GaugeLinks*, ElectricFields*, DOUBLE dTauStep)
//                                                  DYNAMICS/Dynamics.cpp:145-197
//   void Dynamics::Update(GaugeLinks*, ElectricFields*), void Dynamics::Update()
//                                                  DYNAMICS/Dynamics.cpp:204-224
//
// Those files define more than these routines, so they stay in the build and
// their definitions of the routines are renamed by macro while they are
// included; this header then defines the routines under the reference's names:
//
//   #define NCsDot OVL_ReferenceNCsDot
//   #include "TOPOLOGY/ChernSimonsDerivative.cpp"
//   #undef NCsDot
//   #define UpdateGaugeLinks OVL_ReferenceUpdateGaugeLinks
//   #define UpdateElectricFields OVL_ReferenceUpdateElectricFields
//   #define Update OVL_ReferenceUpdate
//   #include "DYNAMICS/Dynamics.cpp"
//   #undef UpdateGaugeLinks
//   #undef UpdateElectricFields
//   #undef Update
//   #include "ovl_dropin_gauge.hpp"
//
// (everything the reference includes after Dynamics.cpp -- the cooling-path
// N_CS, the fermion update -- then calls the GPU routines).  Link with
// -lovl_b200.
//
// Each call uploads the host links and E field to a small device context of
// its own, runs the routine on the GPU and downloads what it changed (links or
// E), so the host fields stay the canonical copies, as in the reference.  The
// GPU routines cover the whole lattice in the Minkowski metric with unit
// lattice spacings, which is how the reference's driver calls them; any other
// range, metric or spacing prints an error and exits, the reference's error
// convention.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "ovl.h"

namespace ovl_dropin {

inline ovl_ctx *&gauge_context() {
    static ovl_ctx *ctx = nullptr;
    return ctx;
}

inline void gauge_check(int rc, const char *what) {
    if (rc != OVL_OK) {
        std::cerr << "#ERROR overlap_b200 " << what << ": " << ovl_last_error(gauge_context()) << std::endl;
        std::exit(1);
    }
}

// The device context of the gauge routines (FP64 links and E; 32 modes it
// never steps).
inline ovl_ctx *gauge() {
    if (!gauge_context()) {
        if (ovl_abi_version() != OVL_ABI_VERSION) {
            std::fprintf(stderr, "ovl_dropin: libovl_b200 ABI %d, header %d: rebuild\n", ovl_abi_version(),
                         OVL_ABI_VERSION);
            std::exit(1);
        }
        ovl_params p;
        ovl_params_init(&p);
        p.N[0] = Lattice::N[0];
        p.N[1] = Lattice::N[1];
        p.N[2] = Lattice::N[2];
        p.n_colours = Nc;
        p.n_modes = 32;
        p.precision = OVL_PREC_FP64;
        p.form = OVL_FORM_FUSED;
        p.device = 0;
        gauge_check(ovl_create(&p, &gauge_context()), "ovl_create (gauge routines)");
    }
    return gauge_context();
}

// The whole lattice, the Minkowski metric and unit spacings, or exit.
inline void gauge_supported(INT xLow, INT xHigh, INT yLow, INT yHigh, INT zLow, INT zHigh, GaugeLinks *U,
                            const char *what) {
    const bool full = xLow == 0 && yLow == 0 && zLow == 0 && xHigh == U->N[0] - 1 && yHigh == U->N[1] - 1 &&
                      zHigh == U->N[2] - 1;
    bool flat = Dynamics::MetricDeterminant == 1.0;
    for (int mu = 0; mu < 3; mu++)
        flat = flat && Dynamics::gDownMetric[mu] == 1.0 && Dynamics::gUpMetric[mu] == 1.0 && U->a[mu] == 1.0;
    if (!full || !flat) {
        std::cerr << "#ERROR overlap_b200 " << what
                  << ": the GPU routine covers the whole lattice in the Minkowski metric with unit spacings"
                  << std::endl;
        std::exit(1);
    }
}

inline void upload_gauge(GaugeLinks *U, ElectricFields *E) {
    gauge_check(ovl_set_links(gauge(), U->U), "ovl_set_links");
    gauge_check(ovl_set_efield(gauge(), E->E), "ovl_set_efield");
}

}  // namespace ovl_dropin

namespace ChernSimonsNumber {

// Improved E.B / (8 pi^2) on the GPU (ovl_ncsdot).
inline DOUBLE NCsDot(GaugeLinks *U, ElectricFields *E) {
    using namespace ovl_dropin;
    upload_gauge(U, E);
    double out = 0.0;
    gauge_check(ovl_ncsdot(gauge(), &out), "ovl_ncsdot");
    return out;
}

}  // namespace ChernSimonsNumber

namespace Dynamics {

// U <- exp(i cU E) U with cU = -dTauStep (Minkowski, unit spacings), on the GPU.
inline void UpdateGaugeLinks(INT xLow, INT xHigh, INT yLow, INT yHigh, INT zLow, INT zHigh, GaugeLinks *U,
                             ElectricFields *E, DOUBLE dTauStep) {
    using namespace ovl_dropin;
    gauge_supported(xLow, xHigh, yLow, yHigh, zLow, zHigh, U, "Dynamics::UpdateGaugeLinks");
    upload_gauge(U, E);
    gauge_check(ovl_update_links(gauge(), dTauStep), "ovl_update_links");
    gauge_check(ovl_get_links(gauge(), U->U), "ovl_get_links");
}

// E += -2 dTauStep (staple force) on the GPU.
inline void UpdateElectricFields(INT xLow, INT xHigh, INT yLow, INT yHigh, INT zLow, INT zHigh, GaugeLinks *U,
                                 ElectricFields *E, DOUBLE dTauStep) {
    using namespace ovl_dropin;
    gauge_supported(xLow, xHigh, yLow, yHigh, zLow, zHigh, U, "Dynamics::UpdateElectricFields");
    upload_gauge(U, E);
    gauge_check(ovl_update_efield(gauge(), dTauStep), "ovl_update_efield");
    gauge_check(ovl_get_efield(gauge(), E->E), "ovl_get_efield");
}

// One gauge leapfrog step: E then U over the whole lattice, step counter + 1
// (one upload and one download of each field).
inline void Update(GaugeLinks *U, ElectricFields *E) {
    using namespace ovl_dropin;
    SetMetric();
    gauge_supported(0, U->N[0] - 1, 0, U->N[1] - 1, 0, U->N[2] - 1, U, "Dynamics::Update");
    upload_gauge(U, E);
    gauge_check(ovl_update_efield(gauge(), dTau), "ovl_update_efield");
    gauge_check(ovl_update_links(gauge(), dTau), "ovl_update_links");
    gauge_check(ovl_get_links(gauge(), U->U), "ovl_get_links");
    gauge_check(ovl_get_efield(gauge(), E->E), "ovl_get_efield");
    tSteps++;
}

inline void Update() { Update(GLinks::U, EFields::E); }

}  // namespace Dynamics
