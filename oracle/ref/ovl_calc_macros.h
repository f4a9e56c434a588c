/* Restated plaquette / colour-trace / Gauss-law macros for the reference
 * harness.  Test infrastructure only.
 *
 * The reference tree lacks CALC/Plaquettes.cpp, CALC/AvgFieldStrength.cpp and
 * CALC/GaussViolation.cpp, which its Simulation.cpp:52-62 includes.  These
 * macros are written from the physics their call sites require:
 *   DYNAMICS/Dynamics.cpp:237-264  (E update from staples),
 *   OBSERVABLES/BulkObservables.cpp:63-77 (4 ReTr(1-U_plaq) magnetic energy),
 *   GAUSSLAWFIXING/GaussRestore.cpp:90-102 (adjoint-transport convention of
 *   the Gauss-law constraint).
 * Plaquette names follow the call sites: U<mu><nu> is the elementary plaquette
 * U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+; an M marks the quadrant on the
 * negative side of that axis (see COMPUTE_NEIGHBORING_PLAQUETTES).
 * Parity of these macros with the (missing) originals is unpinned; they are
 * validated by Gauss-law preservation and energy conservation of the coupled
 * leapfrog (tests/test_oracle_gauge.py). */
#pragma once

#define SET_ELEMENTARY_PLAQUETTE_BUFFERS() \
    SU_Nc_FUNDAMENTAL_FORMAT Uxy[SUNcGroup::MatrixSize], Uyz[SUNcGroup::MatrixSize], Uzx[SUNcGroup::MatrixSize];

#define SET_NEIGHBORING_PLAQUETTE_BUFFERS() \
    SU_Nc_FUNDAMENTAL_FORMAT UxMy[SUNcGroup::MatrixSize], UMxy[SUNcGroup::MatrixSize], \
        UyMz[SUNcGroup::MatrixSize], UMyz[SUNcGroup::MatrixSize], UzMx[SUNcGroup::MatrixSize], UMzx[SUNcGroup::MatrixSize];

#define SET_ELEMENTARY_COLOR_TRACE_BUFFERS() \
    DOUBLE ReTrITaUxy[SUNcAlgebra::VectorSize], ReTrITaUyz[SUNcAlgebra::VectorSize], ReTrITaUzx[SUNcAlgebra::VectorSize];

#define SET_NEIGHBORING_COLOR_TRACE_BUFFERS() \
    DOUBLE ReTrITaUxMy[SUNcAlgebra::VectorSize], ReTrITaUMxy[SUNcAlgebra::VectorSize], \
        ReTrITaUyMz[SUNcAlgebra::VectorSize], ReTrITaUMyz[SUNcAlgebra::VectorSize], \
        ReTrITaUzMx[SUNcAlgebra::VectorSize], ReTrITaUMzx[SUNcAlgebra::VectorSize];

/* U_{mu nu}(x) = U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ */
#define COMPUTE_ELEMENTARY_PLAQUETTES(x, y, z) \
    SUNcGroup::AdvancedOperations::UUDD(U->Get((x), (y), (z), 0), U->Get((x) + 1, (y), (z), 1), U->Get((x), (y) + 1, (z), 0), U->Get((x), (y), (z), 1), Uxy); \
    SUNcGroup::AdvancedOperations::UUDD(U->Get((x), (y), (z), 1), U->Get((x), (y) + 1, (z), 2), U->Get((x), (y), (z) + 1, 1), U->Get((x), (y), (z), 2), Uyz); \
    SUNcGroup::AdvancedOperations::UUDD(U->Get((x), (y), (z), 2), U->Get((x), (y), (z) + 1, 0), U->Get((x) + 1, (y), (z), 2), U->Get((x), (y), (z), 0), Uzx);

#define COMPUTE_ELEMENTARY_COLOR_TRACES() \
    SUNcGroup::Operations::ReTrIGenU(Uxy, ReTrITaUxy); \
    SUNcGroup::Operations::ReTrIGenU(Uyz, ReTrITaUyz); \
    SUNcGroup::Operations::ReTrIGenU(Uzx, ReTrITaUzx);

/* The neighbouring plaquettes are, like the elementary ones, counter-clockwise
 * in their (mu, nu) plane and based at x, but lie in the quadrant the name
 * gives: U<mu>M<nu> in (+mu, -nu), UM<mu><nu> in (-mu, +nu) -- the naming of
 * the clover in CALC/ChernSimonsOperators.cpp:287-313 (UBoxXMY, UBoxMXY).
 * With this orientation each E-update row at Dynamics.cpp:262-264 sums the
 * colour traces of the two staples of U_mu(x) in each plane with one sign. */
#define COMPUTE_NEIGHBORING_PLAQUETTES(x, y, z) \
    SUNcGroup::AdvancedOperations::DUUD(U->Get((x), (y) - 1, (z), 1), U->Get((x), (y) - 1, (z), 0), U->Get((x) + 1, (y) - 1, (z), 1), U->Get((x), (y), (z), 0), UxMy); \
    SUNcGroup::AdvancedOperations::UDDU(U->Get((x), (y), (z), 1), U->Get((x) - 1, (y) + 1, (z), 0), U->Get((x) - 1, (y), (z), 1), U->Get((x) - 1, (y), (z), 0), UMxy); \
    SUNcGroup::AdvancedOperations::DUUD(U->Get((x), (y), (z) - 1, 2), U->Get((x), (y), (z) - 1, 1), U->Get((x), (y) + 1, (z) - 1, 2), U->Get((x), (y), (z), 1), UyMz); \
    SUNcGroup::AdvancedOperations::UDDU(U->Get((x), (y), (z), 2), U->Get((x), (y) - 1, (z) + 1, 1), U->Get((x), (y) - 1, (z), 2), U->Get((x), (y) - 1, (z), 1), UMyz); \
    SUNcGroup::AdvancedOperations::DUUD(U->Get((x) - 1, (y), (z), 0), U->Get((x) - 1, (y), (z), 2), U->Get((x) - 1, (y), (z) + 1, 0), U->Get((x), (y), (z), 2), UzMx); \
    SUNcGroup::AdvancedOperations::UDDU(U->Get((x), (y), (z), 0), U->Get((x) + 1, (y), (z) - 1, 2), U->Get((x), (y), (z) - 1, 0), U->Get((x), (y), (z) - 1, 2), UMzx);

#define COMPUTE_NEIGHBORING_COLOR_TRACES() \
    SUNcGroup::Operations::ReTrIGenU(UxMy, ReTrITaUxMy); \
    SUNcGroup::Operations::ReTrIGenU(UMxy, ReTrITaUMxy); \
    SUNcGroup::Operations::ReTrIGenU(UyMz, ReTrITaUyMz); \
    SUNcGroup::Operations::ReTrIGenU(UMyz, ReTrITaUMyz); \
    SUNcGroup::Operations::ReTrIGenU(UzMx, ReTrITaUzMx); \
    SUNcGroup::Operations::ReTrIGenU(UMzx, ReTrITaUMzx);

/* Gauss-law violation G^a(x) = sum_mu [E^a_mu(x) - (U_mu(x-mu)^+ E_mu(x-mu) U_mu(x-mu))^a];
 * the sign is the one for which the restoration step of
 * GAUSSLAWFIXING/GaussRestore.cpp:90-102 (E_mu(x) -= g (G(x) - U_mu(x) G(x+mu) U_mu(x)^+))
 * descends |G|^2. */
#define SET_GAUSS_LAW_BUFFERS() \
    SU_Nc_ALGEBRA_FORMAT GaussEXM[SUNcAlgebra::VectorSize], GaussEYM[SUNcAlgebra::VectorSize], GaussEZM[SUNcAlgebra::VectorSize];

#define COMPUTE_GAUSS_VIOLATION(Violation, x, y, z) \
    SUNcAlgebra::Operations::InverseAdjointMultiplication(U->Get((x) - 1, (y), (z), 0), E->Get((x) - 1, (y), (z), 0, 0), GaussEXM); \
    SUNcAlgebra::Operations::InverseAdjointMultiplication(U->Get((x), (y) - 1, (z), 1), E->Get((x), (y) - 1, (z), 1, 0), GaussEYM); \
    SUNcAlgebra::Operations::InverseAdjointMultiplication(U->Get((x), (y), (z) - 1, 2), E->Get((x), (y), (z) - 1, 2, 0), GaussEZM); \
    for (int gauss_a = 0; gauss_a < SUNcAlgebra::VectorSize; gauss_a++) { \
        (Violation)[gauss_a] = E->Get((x), (y), (z), 0, gauss_a)[0] - GaussEXM[gauss_a] \
                             + E->Get((x), (y), (z), 1, gauss_a)[0] - GaussEYM[gauss_a] \
                             + E->Get((x), (y), (z), 2, gauss_a)[0] - GaussEZM[gauss_a]; \
    }

/* The unimproved E.B of CALC/ChernSimonsOperators.cpp:1-112 is compiled but not
 * on the hot path (NCsDot uses the improved operator, ChernSimonsDerivative.cpp:44)
 * and the harness never calls it; its buffers are declared and zeroed. */
#define SET_AVG_FIELD_STRENGTH_BUFFERS() \
    DOUBLE E0Loc[SUNcAlgebra::VectorSize], E1Loc[SUNcAlgebra::VectorSize], E2Loc[SUNcAlgebra::VectorSize], \
        B0Loc[SUNcAlgebra::VectorSize], B1Loc[SUNcAlgebra::VectorSize], B2Loc[SUNcAlgebra::VectorSize];
#define COMPUTE_AVG_FIELD_STRENGTH(x, y, z) \
    for (int avg_a = 0; avg_a < SUNcAlgebra::VectorSize; avg_a++) { \
        E0Loc[avg_a] = E1Loc[avg_a] = E2Loc[avg_a] = B0Loc[avg_a] = B1Loc[avg_a] = B2Loc[avg_a] = 0.0; \
    }

/* CALC/GaugeTransformation.cpp (missing; used by
 * GAUGETRANSFORMATION/GaugeTransformation.cpp:112-160): the gauge transformation
 * of links and electric fields by G(x),
 *   U'_mu(x) = G(x) U_mu(x) G(x+mu)^+ ,   E'_mu(x) = G(x) E_mu(x) G(x)^+ ,
 * the convention under which the Gauss-law transport of
 * GAUSSLAWFIXING/GaussRestore.cpp:90-102 (U G(x+mu) U^+) is covariant; the
 * field rotation uses the reference's own AdjointMultiplication.  Parity with
 * the missing original is unpinned; the handmade sphaleron built with it has
 * the vacuum N_CS of its final links equal to the winding number of G
 * (tests/test_sphaleron.py). */
#define PERFORM_GAUGE_LINK_TRANSFORMATION(x, y, z)                                                                   \
    for (INT ovl_mu = 0; ovl_mu < Lattice::Dimension; ovl_mu++) {                                                   \
        SU_Nc_FUNDAMENTAL_FORMAT ovl_gu[SUNcGroup::MatrixSize];                                                     \
        SUNcGroup::Operations::UU(G->Get(x, y, z), UOld->Get(x, y, z, ovl_mu), ovl_gu);                             \
        SUNcGroup::Operations::UD(ovl_gu, G->Get((x) + (ovl_mu == 0), (y) + (ovl_mu == 1), (z) + (ovl_mu == 2)),    \
                                  UNew->Get(x, y, z, ovl_mu));                                                      \
    }

#define PERFORM_ELECTRIC_FIELD_TRANSFORMATION(x, y, z)                                                               \
    for (INT ovl_mu = 0; ovl_mu < Lattice::Dimension; ovl_mu++) {                                                   \
        SUNcAlgebra::Operations::AdjointMultiplication(G->Get(x, y, z), EOld->Get(x, y, z, ovl_mu, 0),              \
                                                       ENew->Get(x, y, z, ovl_mu, 0));                              \
    }
