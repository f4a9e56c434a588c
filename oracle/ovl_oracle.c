/* ovl_oracle.c -- plain-C CPU restatement of the OVERLAP hot path (SU(2)).
 *
 * TEST INFRASTRUCTURE ONLY (see ovl_oracle.h).  Written from the definitions the
 * reference implements, not from its code: quaternion algebra for SU(2), the
 * Wilson operator as mass term + spin-projected hops, Wilson loops as
 * path-ordered products anchored at a site.  Every function cites the reference
 * routine it restates; tests/test_oracle_pin.py checks each one against the
 * reference compiled from source.
 */
#define _DEFAULT_SOURCE
#include "ovl_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ---------------------------------------------------------------- lattice -- */

static int wrap(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

static int site_of(const orc_params *p, int x, int y, int z) {
    return wrap(x, p->N[0]) + p->N[0] * (wrap(y, p->N[1]) + p->N[1] * wrap(z, p->N[2]));
}

static void coords_of(const orc_params *p, int s, int c[3]) {
    c[0] = s % p->N[0];
    c[1] = (s / p->N[0]) % p->N[1];
    c[2] = s / (p->N[0] * p->N[1]);
}

static int shift(const orc_params *p, int s, int mu, int step) {
    int c[3];
    coords_of(p, s, c);
    c[mu] += step;
    return site_of(p, c[0], c[1], c[2]);
}

static int volume(const orc_params *p) { return p->N[0] * p->N[1] * p->N[2]; }

/* ------------------------------------------------------- SU(2) quaternions -- */
/* q = (v0, v1, v2, s) represents s*1 + i v_k sigma_k (GroupOperations.cpp:4-9). */

typedef struct { double v[4]; } quat;

static quat q_load(const double *U, int s, int mu) {
    quat q;
    memcpy(q.v, U + 4 * (mu + 3 * s), sizeof q.v);
    return q;
}

static quat q_unit(void) { quat q = {{0.0, 0.0, 0.0, 1.0}}; return q; }

static quat q_dag(quat a) { quat q = {{-a.v[0], -a.v[1], -a.v[2], a.v[3]}}; return q; }

/* (a3 + i a.s)(b3 + i b.s) = a3 b3 - a.b + i (a3 b + b3 a - a x b).s */
static quat q_mul(quat a, quat b) {
    quat c;
    c.v[3] = a.v[3] * b.v[3] - (a.v[0] * b.v[0] + a.v[1] * b.v[1] + a.v[2] * b.v[2]);
    c.v[0] = a.v[3] * b.v[0] + b.v[3] * a.v[0] - (a.v[1] * b.v[2] - a.v[2] * b.v[1]);
    c.v[1] = a.v[3] * b.v[1] + b.v[3] * a.v[1] - (a.v[2] * b.v[0] - a.v[0] * b.v[2]);
    c.v[2] = a.v[3] * b.v[2] + b.v[3] * a.v[2] - (a.v[0] * b.v[1] - a.v[1] * b.v[0]);
    return c;
}

/* 2x2 complex matrix of q, row-major m[i][j] (GetMatrix, GroupOperations.cpp:213-225). */
static void q_matrix(quat q, cplx m[2][2]) {
    m[0][0] = q.v[3] + I * q.v[2];
    m[0][1] = q.v[1] + I * q.v[0];
    m[1][0] = -q.v[1] + I * q.v[0];
    m[1][1] = q.v[3] - I * q.v[2];
}

/* Re tr(i t^a q), t^a = sigma_a / 2 (ReTrIGenU, GroupOperations.cpp:78-84). */
static double q_retr_ita(quat q, int a) { return -q.v[a]; }

/* exp(i c alpha^a t^a) (MatrixIExp, SU2/AlgebraOperations.cpp:37-56). */
static quat q_exp(double c, const double alpha[3]) {
    double d = sqrt((c * alpha[0]) * (c * alpha[0]) + (c * alpha[1]) * (c * alpha[1]) + (c * alpha[2]) * (c * alpha[2]));
    quat q;
    if (d == 0.0) return q_unit();
    double f = c * sin(0.5 * d) / d;
    q.v[0] = f * alpha[0];
    q.v[1] = f * alpha[1];
    q.v[2] = f * alpha[2];
    q.v[3] = cos(0.5 * d);
    return q;
}

/* Adjoint representation R_ab = 2 tr(t^a q t^b q^+), evaluated with matrices. */
static void q_adjoint(quat q, double R[3][3]) {
    static const cplx sig[3][2][2] = {
        {{0, 1}, {1, 0}},
        {{0, -I}, {I, 0}},
        {{1, 0}, {0, -1}},
    };
    cplx m[2][2], md[2][2];
    q_matrix(q, m);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) md[i][j] = conj(m[j][i]);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            cplx tr = 0;
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++)
                    for (int k = 0; k < 2; k++)
                        for (int l = 0; l < 2; l++)
                            tr += 0.5 * sig[a][i][j] * m[j][k] * 0.5 * sig[b][k][l] * md[l][i];
            R[a][b] = 2.0 * creal(tr);
        }
}

/* Path-ordered product of links along `nsteps` unit steps starting at site s:
 * step (mu, +1) multiplies by U_mu(x), step (mu, -1) by U_mu(x - mu)^+. */
typedef struct { int mu, dir, len; } leg;

static quat q_path(const orc_params *p, const double *U, int s, const leg *legs, int nlegs) {
    quat acc = q_unit();
    int x = s;
    for (int l = 0; l < nlegs; l++)
        for (int k = 0; k < legs[l].len; k++) {
            if (legs[l].dir > 0) {
                acc = q_mul(acc, q_load(U, x, legs[l].mu));
                x = shift(p, x, legs[l].mu, +1);
            } else {
                x = shift(p, x, legs[l].mu, -1);
                acc = q_mul(acc, q_dag(q_load(U, x, legs[l].mu)));
            }
        }
    return acc;
}

/* Counter-clockwise (first +mu, then +nu) lmu x lnu loop in the (mu, nu) plane
 * with site s at its corner in quadrant (smu, snu), holonomy based at s. */
static quat q_loop(const orc_params *p, const double *U, int s, int mu, int nu, int smu, int snu, int lmu, int lnu) {
    leg ccw[4] = {{mu, +1, lmu}, {nu, +1, lnu}, {mu, -1, lmu}, {nu, -1, lnu}};
    /* index of the leg that leaves the corner s when walking counter-clockwise */
    int start = (smu > 0 && snu > 0) ? 0 : (smu < 0 && snu > 0) ? 1 : (smu < 0 && snu < 0) ? 2 : 3;
    leg legs[4];
    for (int k = 0; k < 4; k++) legs[k] = ccw[(start + k) % 4];
    return q_path(p, U, s, legs, 4);
}

/* ------------------------------------------------------ U(1) background -- */
/* Phases multiplying the x and y links of the hopping term (the U(1)
 * background extension); NULL = none.  Layout of QED::U: mu + 2 (x + N0 y). */
static const double *g_u1 = NULL;

void orc_set_u1(const double *u1) { g_u1 = u1; }

static void dress(const orc_params *p, int s, int mu, cplx m[2][2]) {
    if (!g_u1 || mu >= 2) return;
    const int plane = s % (p->N[0] * p->N[1]);
    const cplx ph = g_u1[2 * (mu + 2 * plane)] + I * g_u1[2 * (mu + 2 * plane) + 1];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) m[i][j] *= ph;
}

/* ----------------------------------------------------------- Dirac algebra -- */
/* Dirac representation (DiracAlgebra.cpp:5-12). */
static const cplx G0[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, -1, 0}, {0, 0, 0, -1}};
static const cplx GX[4][4] = {{0, 0, 0, 1}, {0, 0, 1, 0}, {0, -1, 0, 0}, {-1, 0, 0, 0}};
static const cplx GY[4][4] = {{0, 0, 0, -I}, {0, 0, I, 0}, {0, I, 0, 0}, {-I, 0, 0, 0}};
static const cplx GZ[4][4] = {{0, 0, 1, 0}, {0, 0, 0, -1}, {-1, 0, 0, 0}, {0, 1, 0, 0}};
static const cplx G5[4][4] = {{0, 0, 1, 0}, {0, 0, 0, 1}, {1, 0, 0, 0}, {0, 1, 0, 0}};

static void mat4_mul(const cplx a[4][4], const cplx b[4][4], cplx c[4][4]) {
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            cplx t = 0;
            for (int k = 0; k < 4; k++) t += a[i][k] * b[k][j];
            c[i][j] = t;
        }
}

static void mat4_scale(cplx f, const cplx a[4][4], cplx c[4][4]) {
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) c[i][j] = f * a[i][j];
}

/* ------------------------------------------------------------ Wilson h_W -- */

#define NC 2
#define SPINOR (NC * 4)  /* complex numbers per site and mode */

static const cplx *site_spinor(const double *field, int s) { return (const cplx *)field + (size_t)SPINOR * s; }

void orc_wilson_apply(const orc_params *p, const double *U, const double *phi, double *out) {
    const int V = volume(p);
    /* Spin structure of the symmetric difference U phi(x+mu) - U^+ phi(x-mu):
     * the hop term is  -(1 - G_mu) a - (1 + G_mu) b  with a = U_mu(x) phi(x+mu),
     * b = U_mu(x-mu)^+ phi(x-mu) and G_mu = -i gamma_mu, hermitian with
     * G_mu^2 = 1 (WilsonOperator.cpp:79-98).  Mass term (6r + 2m - 2M) phi
     * (:39), overall factor -i gamma_0 / 2 (:100-109). */
    cplx G[3][4][4];
    mat4_scale(-I, GX, G[0]);
    mat4_scale(-I, GY, G[1]);
    mat4_scale(-I, GZ, G[2]);
    const double amass = 6.0 * p->r_wilson + 2.0 * p->m_fermion - 2.0 * p->m_dw;
    for (int s = 0; s < V; s++) {
        const cplx *f = site_spinor(phi, s);
        cplx acc[NC][4];
        for (int c = 0; c < NC; c++)
            for (int a = 0; a < 4; a++) acc[c][a] = amass * f[4 * c + a];
        for (int mu = 0; mu < 3; mu++) {
            cplx Mf[2][2], Mb[2][2];
            q_matrix(q_load(U, s, mu), Mf);
            dress(p, s, mu, Mf);
            int sb = shift(p, s, mu, -1);
            q_matrix(q_load(U, sb, mu), Mb);
            dress(p, sb, mu, Mb);
            const cplx *fp = site_spinor(phi, shift(p, s, mu, +1));
            const cplx *fm = site_spinor(phi, sb);
            cplx a[NC][4], b[NC][4];
            for (int i = 0; i < NC; i++)
                for (int al = 0; al < 4; al++) {
                    a[i][al] = 0;
                    b[i][al] = 0;
                    for (int j = 0; j < NC; j++) {
                        a[i][al] += Mf[i][j] * fp[4 * j + al];
                        b[i][al] += conj(Mb[j][i]) * fm[4 * j + al];
                    }
                }
            for (int i = 0; i < NC; i++)
                for (int al = 0; al < 4; al++) {
                    cplx g = 0;
                    for (int be = 0; be < 4; be++) g += G[mu][al][be] * (a[i][be] - b[i][be]);
                    acc[i][al] += -a[i][al] - b[i][al] + g;
                }
        }
        cplx *o = (cplx *)out + (size_t)SPINOR * s;
        for (int c = 0; c < NC; c++)
            for (int a = 0; a < 4; a++) o[4 * c + a] = (a < 2 ? -0.5 * I : 0.5 * I) * acc[c][a];
    }
}

/* ----------------------------------------------------------- gauge update -- */

void orc_update_links(const orc_params *p, double *U, const double *E, double dt_step) {
    const int V = volume(p);
    /* cU = -dt g_mumu a_mu^2 / (sqrt(-g) a^3) = -dt for Minkowski, a = 1 (Dynamics.cpp:102-104). */
    const double cU = -dt_step;
    for (int s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            quat e = q_exp(cU, E + 3 * (mu + 3 * s));
            quat u = q_mul(e, q_load(U, s, mu));
            memcpy(U + 4 * (mu + 3 * s), u.v, sizeof u.v);
        }
}

void orc_update_efield(const orc_params *p, const double *U, double *E, double dt_step) {
    const int V = volume(p);
    const double gamma = -2.0 * dt_step;  /* -2 dt sqrt(-g) a^3, Dynamics.cpp:150 */
    double *dE = malloc(sizeof(double) * 9 * (size_t)V);
    for (int s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++)
            for (int a = 0; a < 3; a++) {
                double f = 0.0;
                for (int nu = 0; nu < 3; nu++) {
                    if (nu == mu) continue;
                    /* the two staples of U_mu(x) in the (mu, nu) plane, both
                     * written to start with U_mu(x) */
                    leg up[4] = {{mu, +1, 1}, {nu, +1, 1}, {mu, -1, 1}, {nu, -1, 1}};
                    leg dn[4] = {{mu, +1, 1}, {nu, -1, 1}, {mu, -1, 1}, {nu, +1, 1}};
                    f += q_retr_ita(q_path(p, U, s, up, 4), a) + q_retr_ita(q_path(p, U, s, dn, 4), a);
                }
                dE[a + 3 * (mu + 3 * s)] = gamma * f;
            }
    for (size_t k = 0; k < 9 * (size_t)V; k++) E[k] += dE[k];
    free(dE);
}

/* --------------------------------------------------------------- leapfrog -- */

static void half_step(const orc_params *p, const double *U, const double *src, double *dst, int nmodes, double *work) {
    const int V = volume(p);
    const size_t per_mode = (size_t)2 * SPINOR * V;
    for (int m = 0; m < nmodes; m++) {
        orc_wilson_apply(p, U, src + per_mode * m, work);
        double *d = dst + per_mode * m;
        for (size_t k = 0; k < per_mode; k++) d[k] += p->dt * work[k];
    }
}

void orc_wilson_leapfrog(const orc_params *p, double *U, const double *E, double *psi, double *psimid,
                         int nmodes, int *tsteps, int nsteps) {
    double *work = malloc(sizeof(double) * 2 * SPINOR * (size_t)volume(p));
    for (int n = 0; n < nsteps; n++) {
        /* Update.cpp:48-79: psi += dt D(psimid); links 1/2; psimid += dt D(psi); links 1/2. */
        half_step(p, U, psimid, psi, nmodes, work);
        if (p->qs * (*tsteps * p->dt) < p->t_sphaleron) orc_update_links(p, U, E, 0.5 * p->dt);
        half_step(p, U, psi, psimid, nmodes, work);
        if (p->qs * (*tsteps * p->dt) < p->t_sphaleron) orc_update_links(p, U, E, 0.5 * p->dt);
        (*tsteps)++;
    }
    free(work);
}

/* ----------------------------------------------------- handmade sphaleron -- */

/* Lattice coordinate i of extent n -> angle on the torus: the arctangent map
 * centred on the lattice that concentrates the winding within a width r
 * (LocalizedLatticeMap, HandmadeSphaleron.cpp:7-18). */
static double torus_angle(int i, int n, double r) {
    const double b = 1.0 / r, h = n / 2.0;
    return 2.0 * M_PI * (atan(b * (i - h)) - atan(b * (-h))) / (atan(b * h) - atan(-b * h));
}

/* The site's element of SU(2) on S^3: torus angles -> R^3 by tan((t - pi) / 2)
 * (the point at infinity where an angle is 0 or 2 pi), then the inverse
 * stereographic projection (TorusProjection, InverseStereographicProjection,
 * HandmadeSphaleron.cpp:22-70). */
static quat sphaleron_g(const orc_params *p, int s, double r) {
    int c[3];
    coords_of(p, s, c);
    double t[3];
    int inf = 0;
    for (int k = 0; k < 3; k++) {
        t[k] = torus_angle(c[k], p->N[k], r);
        if (t[k] == 0.0 || t[k] == 2.0 * M_PI) inf = 1;
    }
    quat g = {{0.0, 0.0, 0.0, 1.0}};
    if (!inf) {
        const double x = tan(0.5 * (t[0] - M_PI)), y = tan(0.5 * (t[1] - M_PI)), z = tan(0.5 * (t[2] - M_PI));
        const double q = x * x + y * y + z * z, u = (q - 1.0) / (q + 1.0);
        g.v[0] = (1.0 - u) * x;
        g.v[1] = (1.0 - u) * y;
        g.v[2] = (1.0 - u) * z;
        g.v[3] = u;
    }
    return g;
}

void orc_handmade_sphaleron(const orc_params *p, double r_sph, double t_sph, double *U, double *E, double *Ufinal,
                            double *G) {
    const int V = volume(p);
    for (int s = 0; s < V; s++) {
        const quat g = sphaleron_g(p, s, r_sph);
        if (G) memcpy(G + 4 * s, g.v, sizeof g.v);
        for (int mu = 0; mu < 3; mu++) {
            /* the final link G(x) 1 G(x+mu)^+ and the algebra element A with
             * exp(-i A^a t^a) = final link (MatrixILog with C = -1,
             * SU2/AlgebraOperations.cpp:59-74), divided by the transition time */
            const quat b = q_mul(g, q_dag(sphaleron_g(p, shift(p, s, mu, 1), r_sph)));
            if (Ufinal) memcpy(Ufinal + 4 * (mu + 3 * s), b.v, sizeof b.v);
            const double d = sqrt(b.v[0] * b.v[0] + b.v[1] * b.v[1] + b.v[2] * b.v[2]);
            const double m = d != 0.0 ? 2.0 * atan2(d, b.v[3]) / (-d) : 0.0;
            for (int a = 0; a < 3; a++) E[a + 3 * (mu + 3 * s)] = (m * b.v[a]) * (1.0 / t_sph);
            const quat one = q_unit();
            memcpy(U + 4 * (mu + 3 * s), one.v, sizeof one.v);
        }
    }
}

/* ------------------------------------------------------------ plane waves -- */

/* Wilson spinors (GetWilsonDiracSpinor, FermionField.cpp:145-317) or, with
 * `overlap`, overlap spinors (GetOverlapDiracSpinor, :331-517): the same
 * helicity construction with p = M hp / s, meff = M (1 + hp5 / s),
 * hp = sin(2 pi n / N), hp5 = 3 - M - sum cos(2 pi n / N), s = |(hp, hp5)|. */
static int free_spinor_kind(const orc_params *p, const int k[3], int spin, int particle, int overlap, cplx u[4],
                            double *omega) {
    const double TWO_PI = 2.0 * M_PI;
    double pp[3], meff = p->m_fermion, p2 = 0.0;
    if (overlap) {
        double hp5 = 3.0 - p->m_dw, s2 = 0.0;
        for (int i = 0; i < 3; i++) {
            int n = particle == 0 ? k[i] : p->N[i] - k[i];
            pp[i] = sin(TWO_PI * n / (double)p->N[i]);
            hp5 -= cos(TWO_PI * n / (double)p->N[i]);
            s2 += pp[i] * pp[i];
        }
        double sabs = sqrt(s2 + hp5 * hp5);
        for (int i = 0; i < 3; i++) {
            pp[i] = p->m_dw * pp[i] / sabs;
            p2 += pp[i] * pp[i];
        }
        meff = p->m_dw * (1.0 + hp5 / sabs);
    } else {
        for (int i = 0; i < 3; i++) {
            int n = particle == 0 ? k[i] : p->N[i] - k[i];  /* antiparticles carry -p (FermionField.cpp:168-174) */
            pp[i] = sin(TWO_PI * n / (double)p->N[i]);
            double h = sin(M_PI * n / (double)p->N[i]);
            meff += 2.0 * p->r_wilson * h * h;
            p2 += pp[i] * pp[i];
        }
    }
    double pabs = sqrt(p2);
    double w = sqrt(p2 + meff * meff);
    *omega = particle == 0 ? w : -w;

    /* the axis cases test k == 0 or k == N/2 in integer division (FermionField.cpp:188,229):
     * for odd N the momentum index (N-1)/2 takes them too */
    int edge[3];
    for (int i = 0; i < 3; i++) edge[i] = (k[i] == 0 || k[i] == p->N[i] / 2);
    /* two-spinor of definite helicity (:185-226) */
    cplx phi[2];
    double hel;
    if (edge[0] && edge[1]) {
        if (spin == 0) { phi[0] = 1; phi[1] = 0; hel = pp[2] / fabs(pp[2]); }
        else { phi[0] = 0; phi[1] = 1; hel = -pp[2] / fabs(pp[2]); }
        if (edge[2]) hel = 0.0;
    } else {
        hel = spin == 0 ? 1.0 : -1.0;
        cplx q = -(pp[2] - hel * pabs) / (pp[0] - I * pp[1]);
        double d = sqrt(1.0 + creal(q) * creal(q) + cimag(q) * cimag(q));
        phi[0] = 1.0 / d;
        phi[1] = q / d;
    }
    /* four-spinor (:228-268) */
    if (edge[0] && edge[1] && edge[2]) {
        int upper = (particle == 0) == (meff >= 0);
        u[0] = upper ? phi[0] : 0; u[1] = upper ? phi[1] : 0;
        u[2] = upper ? 0 : phi[0]; u[3] = upper ? 0 : phi[1];
    } else {
        double norm = sqrt(2.0 * (*omega) * ((*omega) - meff) / p2);
        u[0] = phi[0] / norm;
        u[1] = phi[1] / norm;
        u[2] = hel * ((*omega) - meff) / pabs * (phi[0] / norm);
        u[3] = hel * ((*omega) - meff) / pabs * (phi[1] / norm);
    }
    /* eigen-residual and normalisation (:270-312) with H = gamma_0 (meff + p.gamma) */
    cplx H[4][4], t[4][4];
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) t[a][b] = meff * (a == b) + pp[0] * GX[a][b] + pp[1] * GY[a][b] + pp[2] * GZ[a][b];
    mat4_mul(G0, t, H);
    int bad = 0;
    for (int a = 0; a < 4; a++) {
        cplx hu = 0;
        for (int b = 0; b < 4; b++) hu += H[a][b] * u[b];
        if (cabs((*omega) * u[a] - hu) > 1e-6) bad = 1;
    }
    double n2 = 0;
    for (int a = 0; a < 4; a++) n2 += creal(u[a]) * creal(u[a]) + cimag(u[a]) * cimag(u[a]);
    if (fabs(n2 - 1.0) > 1e-6) bad = 1;
    return bad;
}

static int g_free_overlap = 0;  /* plane waves of orc_free_fermions / orc3_free_fermions: 1 = overlap spinors */
void orc_set_free_kind(int overlap) { g_free_overlap = overlap; }

int orc_free_fermions(const orc_params *p, int first, int nmodes, double *psi, double *psimid) {
    const int V = volume(p);
    int failures = 0;
    for (int m = 0; m < nmodes; m++) {
        /* mode index = particle + 2(colour + Nc(spin + 2(px + N0(py + N1 pz)))) (FermionField.cpp:38-60) */
        int g = first + m;
        int particle = g % 2; g /= 2;
        int colour = g % NC; g /= NC;
        int spin = g % 2; g /= 2;
        int k[3];
        k[0] = g % p->N[0]; g /= p->N[0];
        k[1] = g % p->N[1]; g /= p->N[1];
        k[2] = g % p->N[2];
        cplx u[4];
        double omega;
        failures += free_spinor_kind(p, k, spin, particle, g_free_overlap, u, &omega);
        cplx half = cexp(-0.5 * I * omega * p->dt);
        cplx *f = (cplx *)psi + (size_t)SPINOR * V * m;
        cplx *fm = (cplx *)psimid + (size_t)SPINOR * V * m;
        for (int s = 0; s < V; s++) {
            int c[3];
            coords_of(p, s, c);
            double arg = (k[0] * c[0]) / (double)p->N[0] + (k[1] * c[1]) / (double)p->N[1] + (k[2] * c[2]) / (double)p->N[2];
            double th = (particle == 0 ? 2.0 : -2.0) * M_PI * arg;
            cplx phase = cos(th) + I * sin(th);
            for (int cc = 0; cc < NC; cc++)
                for (int a = 0; a < 4; a++) {
                    cplx v = cc == colour ? phase * u[a] : 0;
                    f[SPINOR * s + 4 * cc + a] = v;
                    fm[SPINOR * s + 4 * cc + a] = cc == colour ? v * half : 0;
                }
        }
    }
    return failures;
}

/* --------------------------------------------------------------- currents -- */

/* sum_{colour i,j} sum_{alpha beta} g[alpha][beta] M[i][j] conj(f_alpha^i) h_beta^j */
static cplx bilinear(const cplx g[4][4], const cplx M[2][2], const cplx *f, const cplx *h) {
    cplx t = 0;
    for (int i = 0; i < NC; i++)
        for (int j = 0; j < NC; j++) {
            if (M[i][j] == 0) continue;
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++)
                    if (g[a][b] != 0) t += g[a][b] * M[i][j] * conj(f[4 * i + a]) * h[4 * j + b];
        }
    return t;
}

void orc_wilson_currents(const orc_params *p, const double *U, const double *psi, int nmodes, int first,
                         double *jV, double *jA, double *jVw, double *jAw, double *PS, double *WA) {
    const int V = volume(p);
    /* couplings (Currents.cpp:44-92) */
    const cplx (*Gmu[3])[4] = {GX, GY, GZ};
    cplx gV[4][4][4], gA[4][4][4], gPS[4][4], gVw[4][4], gAw[4][4], t[4][4];
    mat4_mul(G0, G0, gV[0]);
    for (int mu = 0; mu < 3; mu++) mat4_mul(G0, Gmu[mu], gV[mu + 1]);
    for (int mu = 0; mu < 4; mu++) mat4_mul(gV[mu], G5, gA[mu]);
    mat4_mul(G0, G5, t);
    mat4_scale(I, t, gPS);
    mat4_scale(-I * p->r_wilson, G0, gVw);
    mat4_scale(-I * p->r_wilson, t, gAw);
    const cplx one[2][2] = {{1, 0}, {0, 1}};

    double *out[6] = {jV, jA, jVw, jAw, PS, WA};
    size_t len[6] = {4 * (size_t)V, 4 * (size_t)V, 4 * (size_t)V, 4 * (size_t)V, (size_t)V, (size_t)V};
    for (int k = 0; k < 6; k++)
        if (out[k]) memset(out[k], 0, sizeof(double) * len[k]);
    const double pre = 1.0 / (2.0 * V);
    for (int m = 0; m < nmodes; m++) {
        const double w = ((first + m) % 2 == 0) ? 1.0 : -1.0;  /* CommutatorExpectationValue, FermionField.cpp:109-122 */
        const cplx *mode = (const cplx *)psi + (size_t)SPINOR * V * m;
        for (int s = 0; s < V; s++) {
            const cplx *f = mode + SPINOR * s;
            cplx jv[4], ja[4], wv[4] = {0, 0, 0, 0}, wa[4] = {0, 0, 0, 0};
            jv[0] = w * bilinear(gV[0], one, f, f);
            ja[0] = w * bilinear(gA[0], one, f, f);
            cplx ps = w * bilinear(gPS, one, f, f);
            cplx anomaly = -2.0 * 3.0 * w * bilinear(gAw, one, f, f);
            for (int mu = 0; mu < 3; mu++) {
                cplx Mf[2][2], Mb[2][2], Mbd[2][2];
                q_matrix(q_load(U, s, mu), Mf);
                dress(p, s, mu, Mf);
                int sb = shift(p, s, mu, -1);
                q_matrix(q_load(U, sb, mu), Mb);
                dress(p, sb, mu, Mb);
                for (int i = 0; i < 2; i++)
                    for (int j = 0; j < 2; j++) Mbd[i][j] = conj(Mb[j][i]);
                const cplx *fp = mode + SPINOR * shift(p, s, mu, +1);
                const cplx *fm = mode + SPINOR * sb;
                jv[mu + 1] = w * bilinear(gV[mu + 1], Mf, f, fp);
                ja[mu + 1] = w * bilinear(gA[mu + 1], Mf, f, fp);
                wv[mu + 1] = w * bilinear(gVw, Mf, f, fp);
                wa[mu + 1] = w * bilinear(gAw, Mf, f, fp);
                anomaly += wa[mu + 1] + w * bilinear(gAw, Mbd, f, fm);
            }
            for (int mu = 0; mu < 4; mu++) {
                if (jV) jV[mu + 4 * s] += pre * creal(jv[mu]);
                if (jA) jA[mu + 4 * s] += pre * creal(ja[mu]);
                if (jVw && mu > 0) jVw[mu + 4 * s] += pre * creal(wv[mu]);
                if (jAw && mu > 0) jAw[mu + 4 * s] += pre * creal(wa[mu]);
            }
            if (PS) PS[s] += pre * creal(ps);
            if (WA) WA[s] += pre * creal(anomaly);
        }
    }
}

/* -------------------------------------------------------------- E.B, NCs -- */

/* Improved colour-electric field on the mu link at s: weights -1/12, 7/12, 7/12,
 * -1/12 on E_mu at s+mu, s, s-mu, s-2mu, each transported to s in the adjoint
 * (ChernSimonsOperators.cpp:379-401). */
static void improved_e(const orc_params *p, const double *U, const double *E, int s, int mu, double out[3]) {
    const int sp = shift(p, s, mu, +1), sm = shift(p, s, mu, -1), smm = shift(p, s, mu, -2);
    double Rp[3][3], Rm[3][3], Rmm[3][3];
    q_adjoint(q_load(U, s, mu), Rp);                                 /* s+mu -> s */
    q_adjoint(q_dag(q_load(U, sm, mu)), Rm);                         /* s-mu -> s */
    q_adjoint(q_mul(q_dag(q_load(U, sm, mu)), q_dag(q_load(U, smm, mu))), Rmm);  /* s-2mu -> s */
    const double *ep = E + 3 * (mu + 3 * sp), *e0 = E + 3 * (mu + 3 * s);
    const double *em = E + 3 * (mu + 3 * sm), *emm = E + 3 * (mu + 3 * smm);
    for (int a = 0; a < 3; a++) {
        double t = (7.0 / 12.0) * e0[a];
        for (int b = 0; b < 3; b++)
            t += -(1.0 / 12.0) * Rp[a][b] * ep[b] + (7.0 / 12.0) * Rm[a][b] * em[b] - (1.0 / 12.0) * Rmm[a][b] * emm[b];
        out[a] = t;
    }
}

/* Improved colour-magnetic field B_k for the (mu, nu) plane: 5/12 of the four
 * plaquettes and -1/24 of the eight 2x1 rectangles with s at a corner, all
 * counter-clockwise and based at s; B^a = 2 Re tr(i t^a avg)
 * (ChernSimonsOperators.cpp:283-421). */
static void improved_b(const orc_params *p, const double *U, int s, int mu, int nu, double out[3]) {
    double avg[4] = {0, 0, 0, 0};
    const int sg[4][2] = {{+1, +1}, {-1, +1}, {-1, -1}, {+1, -1}};
    for (int q = 0; q < 4; q++) {
        quat box = q_loop(p, U, s, mu, nu, sg[q][0], sg[q][1], 1, 1);
        quat r1 = q_loop(p, U, s, mu, nu, sg[q][0], sg[q][1], 2, 1);
        quat r2 = q_loop(p, U, s, mu, nu, sg[q][0], sg[q][1], 1, 2);
        for (int k = 0; k < 4; k++) avg[k] += (5.0 / 12.0) * box.v[k] - (1.0 / 24.0) * (r1.v[k] + r2.v[k]);
    }
    quat a4 = {{avg[0], avg[1], avg[2], avg[3]}};
    for (int a = 0; a < 3; a++) out[a] = 2.0 * q_retr_ita(a4, a);
}

double orc_ncsdot(const orc_params *p, const double *U, const double *E) {
    const int V = volume(p);
    double edotb = 0.0;
    for (int s = 0; s < V; s++) {
        double e[3][3], b[3][3];
        for (int mu = 0; mu < 3; mu++) improved_e(p, U, E, s, mu, e[mu]);
        improved_b(p, U, s, 1, 2, b[0]);  /* B_x from the yz plane */
        improved_b(p, U, s, 2, 0, b[1]);  /* B_y from the zx plane */
        improved_b(p, U, s, 0, 1, b[2]);  /* B_z from the xy plane */
        for (int mu = 0; mu < 3; mu++) edotb += e[mu][0] * b[mu][0] + e[mu][1] * b[mu][1] + e[mu][2] * b[mu][2];
    }
    return 0.125 * edotb / (M_PI * M_PI);
}

/* -------------------------------------------------- energy, Gauss, unitarity -- */

void orc_bulk(const orc_params *p, const double *U, const double *E, double *out) {
    const int V = volume(p);
    double e2[3] = {0, 0, 0}, b2[3] = {0, 0, 0};
    double gmax = 0.0, gsum = 0.0, umax = 0.0, usum = 0.0;
    for (int s = 0; s < V; s++) {
        for (int mu = 0; mu < 3; mu++)
            for (int a = 0; a < 3; a++) e2[mu] += E[a + 3 * (mu + 3 * s)] * E[a + 3 * (mu + 3 * s)];
        /* B_k^2 from the plaquette orthogonal to k: 4 Re tr(1 - U_plaq) (BulkObservables.cpp:72-77) */
        const int planes[3][2] = {{1, 2}, {2, 0}, {0, 1}};
        for (int k = 0; k < 3; k++) {
            quat pl = q_loop(p, U, s, planes[k][0], planes[k][1], +1, +1, 1, 1);
            b2[k] += 4.0 * 2.0 * (1.0 - pl.v[3]);
        }
        /* G^a = sum_mu E_mu(s) - (U^+ E U)(s - mu) */
        double g[3] = {0, 0, 0};
        for (int mu = 0; mu < 3; mu++) {
            int sm = shift(p, s, mu, -1);
            double R[3][3];
            q_adjoint(q_dag(q_load(U, sm, mu)), R);
            for (int a = 0; a < 3; a++) {
                double t = E[a + 3 * (mu + 3 * s)];
                for (int b = 0; b < 3; b++) t -= R[a][b] * E[b + 3 * (mu + 3 * sm)];
                g[a] += t;
            }
        }
        for (int a = 0; a < 3; a++) {
            if (g[a] > gmax) gmax = g[a];  /* signed maximum, as GaussLawViolation.cpp:44 */
            gsum += g[a] * g[a];
        }
        for (int mu = 0; mu < 3; mu++) {
            quat u = q_load(U, s, mu);
            double dev = fabs(u.v[0] * u.v[0] + u.v[1] * u.v[1] + u.v[2] * u.v[2] + u.v[3] * u.v[3] - 1.0);
            if (dev > umax) umax = dev;
            usum += dev * dev;
        }
    }
    for (int k = 0; k < 3; k++) { e2[k] /= V; b2[k] /= V; }
    out[0] = 0.5 * (e2[0] + e2[1] + e2[2] + b2[0] + b2[1] + b2[2]);
    out[1] = 0.5 * ((e2[1] + e2[2] + b2[1] + b2[2]) - (e2[0] + b2[0]));
    out[2] = 0.5 * ((e2[0] + e2[2] + b2[0] + b2[2]) - (e2[1] + b2[1]));
    out[3] = 0.5 * ((e2[0] + e2[1] + b2[0] + b2[1]) - (e2[2] + b2[2]));
    out[4] = 0.5 * (e2[0] + e2[1] + e2[2]);
    out[5] = 0.5 * (b2[0] + b2[1] + b2[2]);
    out[6] = gmax;
    out[7] = sqrt(gsum / (3.0 * V));
    out[8] = umax;
    out[9] = sqrt(usum / (3.0 * V));
}

void orc_u1_flux(const orc_params *p, int nb, double *out) {
    const int N0 = p->N[0], N1 = p->N[1];
    cplx *u = (cplx *)out;
    for (int y = 0; y < N1; y++)
        for (int x = 0; x < N0; x++) {
            /* U_y = exp(-2 pi i nb x / (N0 N1)); U_x = 1 except the x = N0-1 column,
             * which carries exp(2 pi i nb y N0 / (N0 N1)) (QED.cpp:62-84) */
            double ty = -2.0 * M_PI * (double)(nb * x) / (double)(N0 * N1);
            u[1 + 2 * (x + N0 * y)] = cos(ty) + I * sin(ty);
            if (x == N0 - 1) {
                double tx = 2.0 * M_PI * (double)(nb * y * N0) / (double)(N0 * N1);
                u[0 + 2 * (x + N0 * y)] = cos(tx) + I * sin(tx);
            } else {
                u[0 + 2 * (x + N0 * y)] = 1.0;
            }
        }
}

/* ------------------------------------------------------------ back-reaction -- */
/* Fermion back-reaction: an extension without reference counterpart (the
 * reference never updates E from the fermions, FERMIONS/WILSON/Update.cpp:48-79).
 * With U_mu(x) -> exp(i theta^a t^a) U_mu(x) and the fermion energy
 *   H_F = (1/2V) sum_m w_m Re <psi_m, h_W psi_m>,  h_W = i D,
 * the hop terms of h_W that contain U_mu(x) give
 *   dH_F/dtheta^a_mu(x) = -(1/2V) sum_m w_m Re[psi_m(x)^+ g0 (1 - G_mu) i t^a U_mu(x) psi_m(x+mu)],
 * G_mu = -i gamma_mu.  The coupled equations are dE/dt = dH/dtheta with
 * H = H_gauge + g^2 H_F, the gauge part being the staple force of
 * orc_update_efield, so H_gauge + g^2 H_F is conserved. */
void orc_color_force(const orc_params *p, const double *U, const double *psi, int nmodes, int first, double *out) {
    const int V = volume(p);
    cplx G[3][4][4], gp[3][4][4];
    mat4_scale(-I, GX, G[0]);
    mat4_scale(-I, GY, G[1]);
    mat4_scale(-I, GZ, G[2]);
    for (int mu = 0; mu < 3; mu++) {
        cplx t[4][4];
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) t[a][b] = (a == b) - G[mu][a][b];
        mat4_mul(G0, t, gp[mu]);  /* g0 (1 - G_mu) */
    }
    static const cplx sig[3][2][2] = {{{0, 1}, {1, 0}}, {{0, -I}, {I, 0}}, {{1, 0}, {0, -1}}};
    memset(out, 0, sizeof(double) * 9 * (size_t)V);
    const double pre = 1.0 / (2.0 * V);
    for (int m = 0; m < nmodes; m++) {
        const double w = ((first + m) % 2 == 0) ? 1.0 : -1.0;
        const cplx *mode = (const cplx *)psi + (size_t)SPINOR * V * m;
        for (int s = 0; s < V; s++) {
            const cplx *f = mode + SPINOR * s;
            for (int mu = 0; mu < 3; mu++) {
                cplx M[2][2];
                q_matrix(q_load(U, s, mu), M);
                dress(p, s, mu, M);
                const cplx *h = mode + SPINOR * shift(p, s, mu, +1);
                for (int a = 0; a < 3; a++) {
                    /* colour matrix i t^a M */
                    cplx A[2][2];
                    for (int i = 0; i < 2; i++)
                        for (int j = 0; j < 2; j++) {
                            A[i][j] = 0;
                            for (int k = 0; k < 2; k++) A[i][j] += I * 0.5 * sig[a][i][k] * M[k][j];
                        }
                    cplx b = 0;
                    for (int i = 0; i < NC; i++)
                        for (int j = 0; j < NC; j++)
                            for (int al = 0; al < 4; al++)
                                for (int be = 0; be < 4; be++)
                                    if (gp[mu][al][be] != 0) b += conj(f[4 * i + al]) * gp[mu][al][be] * A[i][j] * h[4 * j + be];
                    out[a + 3 * (mu + 3 * s)] += -pre * w * creal(b);
                }
            }
        }
    }
}

/* (1/2V) sum_m w_m Re <psi_m, i D psi_m>: the fermion energy H_F. */
double orc_fermion_energy(const orc_params *p, const double *U, const double *psi, int nmodes, int first) {
    const int V = volume(p);
    const size_t per_mode = (size_t)2 * SPINOR * V;
    double *work = malloc(sizeof(double) * per_mode);
    double e = 0.0;
    for (int m = 0; m < nmodes; m++) {
        const double w = ((first + m) % 2 == 0) ? 1.0 : -1.0;
        orc_wilson_apply(p, U, psi + per_mode * m, work);
        const cplx *f = (const cplx *)(psi + per_mode * m), *d = (const cplx *)work;
        cplx t = 0;
        for (int k = 0; k < SPINOR * V; k++) t += conj(f[k]) * I * d[k];
        e += w * creal(t);
    }
    free(work);
    return e / (2.0 * V);
}

/* Coupled leapfrog: the reference step (orc_wilson_leapfrog, links moving every
 * half step) followed by E += dt (gauge ? staple force : 0) + dt g2 dH_F/dtheta
 * from the integer-time modes and links. */
void orc_coupled_leapfrog(const orc_params *p, double *U, double *E, double *psi, double *psimid, int nmodes, int first,
                          int *tsteps, int nsteps, double g2, int gauge) {
    const int V = volume(p);
    double *force = malloc(sizeof(double) * 9 * (size_t)V);
    for (int n = 0; n < nsteps; n++) {
        orc_wilson_leapfrog(p, U, E, psi, psimid, nmodes, tsteps, 1);
        if (gauge) orc_update_efield(p, U, E, p->dt);
        if (g2 != 0.0) {
            orc_color_force(p, U, psi, nmodes, first, force);
            for (size_t k = 0; k < 9 * (size_t)V; k++) E[k] += p->dt * g2 * force[k];
        }
    }
    free(force);
}

/* ------------------------------------------------------------------- Ritz -- */
/* OverlapOperations::RitzSolver with one eigenvalue (FERMIONS/OVERLAP/OPERATOR/
 * RitzSolver.cpp:91-292; orthog is then a no-op): a conjugate-gradient
 * minimisation of the Rayleigh quotient of sign * A, A = -D^2 = h_W^2
 * (WilsonUU, :48-88), from `start` (one mode, [V][Nc][4] complex).  Returns the
 * extreme Rayleigh quotient (the smallest eigenvalue of sign * A); *iters = the
 * reference's ittot.  Vectors are kept in the mode layout; only the start
 * vector's layout matters for the result. */
static cplx vdot(const cplx *a, const cplx *b, size_t n) {
    cplx t = 0;
    for (size_t i = 0; i < n; i++) t += b[i] * conj(a[i]);
    return t;
}

static void apply_a(const orc_params *p, const double *U, double sign, const cplx *in, cplx *out, cplx *tmp) {
    const size_t n = (size_t)SPINOR * volume(p);
    orc_wilson_apply(p, U, (const double *)in, (double *)tmp);
    orc_wilson_apply(p, U, (const double *)tmp, (double *)out);
    for (size_t i = 0; i < n; i++) out[i] = -sign * out[i];
}

double orc_ritz(const orc_params *p, const double *U, const double *start, double sign, int max_iter, int nrestart,
                double delitr, int *iters) {
    const size_t n = (size_t)SPINOR * volume(p);
    cplx *x = malloc(sizeof(cplx) * n), *y = malloc(sizeof(cplx) * n), *z = malloc(sizeof(cplx) * n);
    cplx *g = malloc(sizeof(cplx) * n), *pv = malloc(sizeof(cplx) * n), *tmp = malloc(sizeof(cplx) * n);
    memcpy(x, start, sizeof(cplx) * n);
    double xn = 1.0 / sqrt(creal(vdot(x, x, n)));
    for (size_t i = 0; i < n; i++) x[i] *= xn;
    int ittot = 0, done = 0;
    cplx xy = 0;
    while (!done) {
        apply_a(p, U, sign, x, y, tmp);
        xy = vdot(x, y, n);
        for (size_t i = 0; i < n; i++) g[i] = pv[i] = y[i] - xy * x[i];
        double gnormim = creal(vdot(g, g, n));
        double pnorm = sqrt(gnormim);
        for (size_t i = 0; i < n; i++) pv[i] /= pnorm;
        for (int itt = 1; itt <= nrestart; itt++) {
            ittot++;
            apply_a(p, U, sign, pv, z, tmp);
            const cplx amb = xy - creal(vdot(pv, z, n));
            const double ccc = creal(vdot(x, z, n));
            const double cox = 2.0 * ccc / creal(amb);
            const double sig1 = -copysign(1.0, creal(amb));
            const double sig2 = copysign(1.0, cox) * sig1;
            const double c2 = cox * cox;
            double ct, st;
            if (c2 <= 1.0e-3) {
                /* the reference's series for the rotation (:197-200), constants as there */
                const double sqp = 1.0 - 0.125 * c2 + 0.0859375 * c2 * c2 - 0.0673828125 * c2 * c2 * c2 +
                                   0.0562439 * c2 * c2 * c2 * c2 + 0.0487 * c2 * c2 * c2 * c2 * c2;
                const double sqm = 0.5 * sig1 * sig2 * cox *
                                   (1.0 - 0.375 * c2 + 0.2421875 * c2 * c2 - 0.182617875 * c2 * c2 * c2 +
                                    0.1482849 * c2 * c2 * c2 * c2 - 0.12575 * c2 * c2 * c2 * c2 * c2 +
                                    0.1097 * c2 * c2 * c2 * c2 * c2 * c2);
                if (sig1 < 0.0) { ct = sqm; st = sig2 * sqp; }
                else { ct = sqp; st = sig2 * sqm; }
            } else {
                const double sox = sig1 / sqrt(1.0 + c2);
                ct = sqrt((1.0 + sox) * 0.5);
                st = sqrt((1.0 - sox) * 0.5) * sig2;
            }
            for (size_t i = 0; i < n; i++) {
                x[i] = x[i] * ct + pv[i] * st;
                y[i] = y[i] * ct + z[i] * st;
            }
            double xnorm = creal(vdot(x, x, n));
            const cplx oxy = xy;
            xy = vdot(x, y, n);
            xnorm = 1.0 / sqrt(xnorm);
            xy = xy * xnorm;
            for (size_t i = 0; i < n; i++) {
                x[i] = x[i] * xnorm;
                g[i] = y[i] - xy * x[i];
            }
            const double gnorm = creal(vdot(g, g, n));
            const cplx xp = vdot(x, pv, n);
            if (creal(xy) > creal(oxy)) { done = 1; break; }
            if (gnorm < delitr * sign * creal(xy)) { done = 1; break; }
            const double beta = gnorm / gnormim * pnorm;
            for (size_t i = 0; i < n; i++) pv[i] = g[i] + beta * (pv[i] - x[i] * xp);
            pnorm = sqrt(creal(vdot(pv, pv, n)));
            for (size_t i = 0; i < n; i++) pv[i] /= pnorm;
            gnormim = gnorm;
            if (ittot >= max_iter) { done = 1; break; }
        }
    }
    free(x); free(y); free(z); free(g); free(pv); free(tmp);
    if (iters) *iters = ittot;
    return creal(xy);
}

/* ------------------------------------------------------- Gauss restoration -- */
/* GaussLawRestoration (GAUSSLAWFIXING/GaussRestore.cpp:13-168): G^a(x) =
 * sum_mu E_mu(x) - U_mu(x-mu)^+ E_mu(x-mu) U_mu(x-mu) (the violation of
 * orc_bulk), then E_mu(x) -= gamma (G(x) - U_mu(x) G(x+mu) U_mu(x)^+) with
 * gamma = 7/24, 7/48, 7/72 per iteration, until the signed maximum of G
 * (:46-49) is at most 1e-14 (10^(1 - digits10), :152) or 10000 iterations.
 * Returns the iterations; out2 = {max, avg} of the last violation. */
static double gauss_violation(const orc_params *p, const double *U, const double *E, double *G, double *avg) {
    const int V = volume(p);
    double mx = 0.0, sq = 0.0;
    for (int s = 0; s < V; s++) {
        double g[3] = {0, 0, 0};
        for (int mu = 0; mu < 3; mu++) {
            int sm = shift(p, s, mu, -1);
            double R[3][3];
            q_adjoint(q_dag(q_load(U, sm, mu)), R);
            for (int a = 0; a < 3; a++) {
                double t = E[a + 3 * (mu + 3 * s)];
                for (int b = 0; b < 3; b++) t -= R[a][b] * E[b + 3 * (mu + 3 * sm)];
                g[a] += t;
            }
        }
        for (int a = 0; a < 3; a++) {
            G[a + 3 * s] = g[a];
            if (g[a] > mx) mx = g[a];
            sq += g[a] * g[a];
        }
    }
    *avg = sqrt(sq / (3.0 * V));
    return mx;
}

static void gauss_update(const orc_params *p, const double *U, const double *G, double *E, double gamma) {
    const int V = volume(p);
    for (int s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            double R[3][3];
            q_adjoint(q_load(U, s, mu), R);
            const double *gp = G + 3 * shift(p, s, mu, +1);
            for (int a = 0; a < 3; a++) {
                double up = 0.0;
                for (int b = 0; b < 3; b++) up += R[a][b] * gp[b];
                E[a + 3 * (mu + 3 * s)] -= gamma * (G[a + 3 * s] - up);
            }
        }
}

int orc_gauss_restore(const orc_params *p, const double *U, double *E, int max_iter, double tol, double *out2) {
    const int V = volume(p);
    double *G = malloc(sizeof(double) * 3 * (size_t)V);
    double avg = 0.0;
    double mx = gauss_violation(p, U, E, G, &avg);
    int n = 0;
    static const double gammas[3] = {7.0 / 24.0, 7.0 / 48.0, 7.0 / 72.0};
    while (n < max_iter && mx > tol) {
        for (int k = 0; k < 3; k++) {
            mx = gauss_violation(p, U, E, G, &avg);
            gauss_update(p, U, G, E, gammas[k]);
        }
        n++;
    }
    free(G);
    if (out2) { out2[0] = mx; out2[1] = avg; }
    return n;
}

/* ======================================================================== */
/* SU(3): the same operators for three colours.                             */
/*                                                                          */
/* The reference's fermion code is written for two colours                  */
/* (FermionField.cpp:8-9, WilsonOperator.cpp:45-46) and its SU(3) group      */
/* code does not build (LATTICE/GaugeLinks.cpp:46 returns the links as       */
/* DOUBLE*, SUNc/SU3/AlgebraOperations.cpp:197 calls an undeclared           */
/* ComplexEigensystem), so these functions restate the operators above from  */
/* their definitions for Nc = 3:                                             */
/*   links: 9 complex numbers per link, U_ij at i + 3j                       */
/*          (SUNc/SU3/GroupOperations.cpp:4-12), link (site, mu) at          */
/*          18 (mu + 3 site) doubles;                                        */
/*   E:     8 components per link, generators t^a = lambda^a / 2             */
/*          (SU3/AlgebraOperations.cpp:6), E[a + 8 (mu + 3 site)];           */
/*   modes: [mode][site][colour 3][spin 4] complex.                          */
/* With SU(2) embedded in the upper-left block (sigma_k -> lambda_k, a < 3)  */
/* every function reproduces its SU(2) counterpart above, which is pinned to */
/* the reference.                                                            */
/* ======================================================================== */

#define SPINOR3 12

typedef struct { cplx m[3][3]; } m3;

static m3 m3_load(const double *U, int s, int mu) {
    m3 a;
    const double *p = U + 18 * (size_t)(mu + 3 * s);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a.m[i][j] = p[2 * (i + 3 * j)] + I * p[2 * (i + 3 * j) + 1];
    return a;
}

static void m3_store(double *U, int s, int mu, const m3 *a) {
    double *p = U + 18 * (size_t)(mu + 3 * s);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            p[2 * (i + 3 * j)] = creal(a->m[i][j]);
            p[2 * (i + 3 * j) + 1] = cimag(a->m[i][j]);
        }
}

static m3 m3_unit(void) {
    m3 a;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a.m[i][j] = i == j ? 1.0 : 0.0;
    return a;
}

static m3 m3_mul(const m3 *a, const m3 *b) {
    m3 c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            cplx t = 0;
            for (int k = 0; k < 3; k++) t += a->m[i][k] * b->m[k][j];
            c.m[i][j] = t;
        }
    return c;
}

static m3 m3_dag(const m3 *a) {
    m3 c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c.m[i][j] = conj(a->m[j][i]);
    return c;
}

/* t^a alpha^a (MatrixForm, SU3/AlgebraOperations.cpp:89-105) */
static m3 su3_matrix_form(const double al[8]) {
    const double r3 = 1.0 / sqrt(3.0);
    m3 A;
    A.m[0][0] = 0.5 * (al[2] + al[7] * r3);
    A.m[1][1] = -0.5 * (al[2] - al[7] * r3);
    A.m[2][2] = -al[7] * r3;
    A.m[1][0] = 0.5 * (al[0] + I * al[1]);
    A.m[2][0] = 0.5 * (al[3] + I * al[4]);
    A.m[2][1] = 0.5 * (al[5] + I * al[6]);
    A.m[0][1] = conj(A.m[1][0]);
    A.m[0][2] = conj(A.m[2][0]);
    A.m[1][2] = conj(A.m[2][1]);
    return A;
}

static m3 su3_generator(int a) {
    double al[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    al[a] = 1.0;
    return su3_matrix_form(al);
}

/* 2 tr(t^a V), the algebra components of a hermitian traceless V */
static void su3_components(const m3 *V, double out[8]) {
    for (int a = 0; a < 8; a++) {
        m3 t = su3_generator(a);
        cplx s = 0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) s += t.m[i][j] * V->m[j][i];
        out[a] = 2.0 * creal(s);
    }
}

/* Re tr(i t^a V) (ReTrIGenU, SU3/GroupOperations.cpp:108-119) */
static double su3_retr_ita(const m3 *V, int a) {
    m3 t = su3_generator(a);
    cplx s = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) s += t.m[i][j] * V->m[j][i];
    return -cimag(s);
}

/* R_ab = 2 tr(t^a V t^b V^+) (GetAdjoint's definition, SU3/GroupOperations.cpp:213) */
static void su3_adjoint(const m3 *V, double R[8][8]) {
    m3 Vd = m3_dag(V), T[8];
    for (int a = 0; a < 8; a++) T[a] = su3_generator(a);
    for (int b = 0; b < 8; b++) {
        m3 x = m3_mul(V, &T[b]);
        m3 y = m3_mul(&x, &Vd);
        for (int a = 0; a < 8; a++) {
            cplx s = 0;
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) s += T[a].m[i][j] * y.m[j][i];
            R[a][b] = 2.0 * creal(s);
        }
    }
}

/* Eigensystem of a hermitian 3x3 matrix by cyclic Jacobi rotations:
 * A = Vec diag(lam) Vec^+.  Each rotation J = diag(1, e^{-i phi}) R(theta) on
 * the (p, q) pair, a_pq = r e^{i phi}, tan 2 theta = 2 r / (a_qq - a_pp). */
static void herm3_eigen(m3 A, double lam[3], m3 *Vec) {
    m3 Vm = m3_unit();
    for (int sweep = 0; sweep < 64; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < 3; i++) {
            diag += creal(A.m[i][i]) * creal(A.m[i][i]);
            for (int j = i + 1; j < 3; j++) off += creal(A.m[i][j] * conj(A.m[i][j]));
        }
        if (off <= 1e-34 * diag || off < 1e-300) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                const double r = cabs(A.m[p][q]);
                if (r == 0.0) continue;
                const cplx ph = A.m[p][q] / r;
                const double th = 0.5 * atan2(2.0 * r, creal(A.m[q][q]) - creal(A.m[p][p]));
                const double c = cos(th), s = sin(th);
                m3 J = m3_unit();
                J.m[p][p] = c;
                J.m[p][q] = s;
                J.m[q][p] = -s * conj(ph);
                J.m[q][q] = c * conj(ph);
                m3 Jd = m3_dag(&J);
                m3 t = m3_mul(&A, &J);
                A = m3_mul(&Jd, &t);
                Vm = m3_mul(&Vm, &J);
            }
    }
    for (int i = 0; i < 3; i++) lam[i] = creal(A.m[i][i]);
    *Vec = Vm;
}

/* exp(i c t^a alpha^a) through the eigensystem of t^a alpha^a, the method of
 * MatrixIExp (SU3/AlgebraOperations.cpp:141-183) with a Jacobi eigensolver. */
void orc3_exp(double c, const double alpha[8], double out[18]) {
    m3 A = su3_matrix_form(alpha), Vec, R;
    double lam[3];
    herm3_eigen(A, lam, &Vec);
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            cplx t = 0;
            for (int j = 0; j < 3; j++) t += Vec.m[i][j] * cexp(I * c * lam[j]) * conj(Vec.m[k][j]);
            R.m[i][k] = t;
        }
    m3_store(out, 0, 0, &R);
}

/* A^a with exp(-i A^a t^a) = W for unitary W of unit determinant (MatrixILog
 * with C = -1, SU3/AlgebraOperations.cpp:186-234): the eigenvectors of the
 * hermitian H = (W + W^+)/2 + (W - W^+)/2i are those of W while no two of
 * W's eigenphases add up to pi/2 (geodesics between nearby links); the
 * phases theta_j = arg(v_j^+ W v_j) are made to sum to zero. */
static void su3_log(const m3 *W, double out[8]) {
    m3 Wd = m3_dag(W), H, Vec;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) H.m[i][j] = 0.5 * (W->m[i][j] + Wd.m[i][j]) - 0.5 * I * (W->m[i][j] - Wd.m[i][j]);
    double lam[3], th[3], sum = 0.0;
    herm3_eigen(H, lam, &Vec);
    for (int j = 0; j < 3; j++) {
        cplx e = 0;
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++) e += conj(Vec.m[i][j]) * W->m[i][k] * Vec.m[k][j];
        th[j] = carg(e);
        sum += th[j];
    }
    if (fabs(sum) > M_PI) {  /* one phase on the other branch */
        int big = 0;
        for (int j = 1; j < 3; j++)
            if (fabs(th[j]) > fabs(th[big])) big = j;
        th[big] -= sum > 0 ? 2.0 * M_PI : -2.0 * M_PI;
        sum = th[0] + th[1] + th[2];
    }
    for (int j = 0; j < 3; j++) th[j] -= sum / 3.0;
    m3 G;  /* generator of W = exp(i G); A^a t^a = -G */
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            cplx t = 0;
            for (int j = 0; j < 3; j++) t += Vec.m[i][j] * th[j] * conj(Vec.m[k][j]);
            G.m[i][k] = -t;
        }
    su3_components(&G, out);
}

static void dress3(const orc_params *p, int s, int mu, m3 *m) {
    if (!g_u1 || mu >= 2) return;
    const int plane = s % (p->N[0] * p->N[1]);
    const cplx ph = g_u1[2 * (mu + 2 * plane)] + I * g_u1[2 * (mu + 2 * plane) + 1];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m->m[i][j] *= ph;
}

/* out = -i h_W phi for one three-colour mode (orc_wilson_apply with 3x3 links). */
void orc3_wilson_apply(const orc_params *p, const double *U, const double *phi, double *out) {
    const int V = volume(p);
    cplx G[3][4][4];
    mat4_scale(-I, GX, G[0]);
    mat4_scale(-I, GY, G[1]);
    mat4_scale(-I, GZ, G[2]);
    const double amass = 6.0 * p->r_wilson + 2.0 * p->m_fermion - 2.0 * p->m_dw;
    const cplx *fld = (const cplx *)phi;
    for (int s = 0; s < V; s++) {
        const cplx *f = fld + (size_t)SPINOR3 * s;
        cplx acc[3][4];
        for (int c = 0; c < 3; c++)
            for (int a = 0; a < 4; a++) acc[c][a] = amass * f[4 * c + a];
        for (int mu = 0; mu < 3; mu++) {
            const int sb = shift(p, s, mu, -1);
            m3 Mf = m3_load(U, s, mu), Mb = m3_load(U, sb, mu);
            dress3(p, s, mu, &Mf);
            dress3(p, sb, mu, &Mb);
            const cplx *fp = fld + (size_t)SPINOR3 * shift(p, s, mu, +1);
            const cplx *fm = fld + (size_t)SPINOR3 * sb;
            cplx a[3][4], b[3][4];
            for (int i = 0; i < 3; i++)
                for (int al = 0; al < 4; al++) {
                    a[i][al] = 0;
                    b[i][al] = 0;
                    for (int j = 0; j < 3; j++) {
                        a[i][al] += Mf.m[i][j] * fp[4 * j + al];
                        b[i][al] += conj(Mb.m[j][i]) * fm[4 * j + al];
                    }
                }
            for (int i = 0; i < 3; i++)
                for (int al = 0; al < 4; al++) {
                    cplx g = 0;
                    for (int be = 0; be < 4; be++) g += G[mu][al][be] * (a[i][be] - b[i][be]);
                    acc[i][al] += -a[i][al] - b[i][al] + g;
                }
        }
        cplx *o = (cplx *)out + (size_t)SPINOR3 * s;
        for (int c = 0; c < 3; c++)
            for (int a = 0; a < 4; a++) o[4 * c + a] = (a < 2 ? -0.5 * I : 0.5 * I) * acc[c][a];
    }
}

/* U <- exp(i cU t^a E^a) U, cU = -dt_step (Dynamics.cpp:97-138). */
void orc3_update_links(const orc_params *p, double *U, const double *E, double dt_step) {
    const int V = volume(p);
    for (int s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            double g[18];
            orc3_exp(-dt_step, E + 8 * (mu + 3 * s), g);
            m3 G = m3_load(g, 0, 0), u = m3_load(U, s, mu);
            m3 n = m3_mul(&G, &u);
            m3_store(U, s, mu, &n);
        }
}

static m3 m3_path(const orc_params *p, const double *U, int s, const leg *legs, int nlegs) {
    m3 acc = m3_unit();
    int cur = s;
    for (int k = 0; k < nlegs; k++)
        for (int n = 0; n < legs[k].len; n++) {
            if (legs[k].dir > 0) {
                m3 u = m3_load(U, cur, legs[k].mu);
                acc = m3_mul(&acc, &u);
                cur = shift(p, cur, legs[k].mu, +1);
            } else {
                cur = shift(p, cur, legs[k].mu, -1);
                m3 u = m3_load(U, cur, legs[k].mu), ud = m3_dag(&u);
                acc = m3_mul(&acc, &ud);
            }
        }
    return acc;
}

static m3 m3_loop(const orc_params *p, const double *U, int s, int mu, int nu, int smu, int snu, int lmu, int lnu) {
    /* the leg order of q_loop: counter-clockwise from the corner in quadrant (smu, snu) */
    leg L4[4] = {{mu, +1, lmu}, {nu, +1, lnu}, {mu, -1, lmu}, {nu, -1, lnu}};
    const int start = (smu > 0 && snu > 0) ? 0 : (smu < 0 && snu > 0) ? 1 : (smu < 0 && snu < 0) ? 2 : 3;
    leg legs[4];
    for (int k = 0; k < 4; k++) legs[k] = L4[(start + k) & 3];
    return m3_path(p, U, s, legs, 4);
}

/* Staple force, the SU(3) form of orc_update_efield (Dynamics.cpp:145-197). */
void orc3_update_efield(const orc_params *p, const double *U, double *E, double dt_step) {
    const int V = volume(p);
    const double gamma = -2.0 * dt_step;
    double *dE = malloc(sizeof(double) * 24 * (size_t)V);
    for (int s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            double f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int nu = 0; nu < 3; nu++) {
                if (nu == mu) continue;
                leg up[4] = {{mu, +1, 1}, {nu, +1, 1}, {mu, -1, 1}, {nu, -1, 1}};
                leg dn[4] = {{mu, +1, 1}, {nu, -1, 1}, {mu, -1, 1}, {nu, +1, 1}};
                m3 a = m3_path(p, U, s, up, 4), b = m3_path(p, U, s, dn, 4);
                for (int k = 0; k < 8; k++) f[k] += su3_retr_ita(&a, k) + su3_retr_ita(&b, k);
            }
            for (int k = 0; k < 8; k++) dE[k + 8 * (mu + 3 * s)] = gamma * f[k];
        }
    for (size_t k = 0; k < 24 * (size_t)V; k++) E[k] += dE[k];
    free(dE);
}

static void half_step3(const orc_params *p, const double *U, const double *src, double *dst, int nmodes,
                       double *work) {
    const size_t per_mode = (size_t)2 * SPINOR3 * volume(p);
    for (int m = 0; m < nmodes; m++) {
        orc3_wilson_apply(p, U, src + per_mode * m, work);
        double *d = dst + per_mode * m;
        for (size_t k = 0; k < per_mode; k++) d[k] += p->dt * work[k];
    }
}

/* The Wilson leapfrog (Update.cpp:48-79) for three colours. */
void orc3_wilson_leapfrog(const orc_params *p, double *U, const double *E, double *psi, double *psimid, int nmodes,
                          int *tsteps, int nsteps) {
    double *work = malloc(sizeof(double) * 2 * SPINOR3 * (size_t)volume(p));
    for (int n = 0; n < nsteps; n++) {
        half_step3(p, U, psimid, psi, nmodes, work);
        if (p->qs * (*tsteps * p->dt) < p->t_sphaleron) orc3_update_links(p, U, E, 0.5 * p->dt);
        half_step3(p, U, psi, psimid, nmodes, work);
        if (p->qs * (*tsteps * p->dt) < p->t_sphaleron) orc3_update_links(p, U, E, 0.5 * p->dt);
        (*tsteps)++;
    }
    free(work);
}

/* Plane waves for three colours (SetFreeFermions.cpp:3-56 with Nc = 3). */
int orc3_free_fermions(const orc_params *p, int first, int nmodes, double *psi, double *psimid) {
    const int V = volume(p);
    int failures = 0;
    for (int m = 0; m < nmodes; m++) {
        int g = first + m;
        int particle = g % 2; g /= 2;
        int colour = g % 3; g /= 3;
        int spin = g % 2; g /= 2;
        int k[3];
        k[0] = g % p->N[0]; g /= p->N[0];
        k[1] = g % p->N[1]; g /= p->N[1];
        k[2] = g % p->N[2];
        cplx u[4];
        double omega;
        failures += free_spinor_kind(p, k, spin, particle, g_free_overlap, u, &omega);
        cplx half = cexp(-0.5 * I * omega * p->dt);
        cplx *f = (cplx *)psi + (size_t)SPINOR3 * V * m;
        cplx *fm = (cplx *)psimid + (size_t)SPINOR3 * V * m;
        for (int s = 0; s < V; s++) {
            int c[3];
            coords_of(p, s, c);
            double arg = (k[0] * c[0]) / (double)p->N[0] + (k[1] * c[1]) / (double)p->N[1] + (k[2] * c[2]) / (double)p->N[2];
            double th = (particle == 0 ? 2.0 : -2.0) * M_PI * arg;
            cplx phase = cos(th) + I * sin(th);
            for (int cc = 0; cc < 3; cc++)
                for (int a = 0; a < 4; a++) {
                    cplx v = cc == colour ? phase * u[a] : 0;
                    f[SPINOR3 * s + 4 * cc + a] = v;
                    fm[SPINOR3 * s + 4 * cc + a] = cc == colour ? v * half : 0;
                }
        }
    }
    return failures;
}

static cplx bilinear3(const cplx g[4][4], const m3 *M, const cplx *f, const cplx *h) {
    cplx t = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const cplx mij = M ? M->m[i][j] : (i == j ? 1.0 : 0.0);
            if (mij == 0) continue;
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++)
                    if (g[a][b] != 0) t += g[a][b] * mij * conj(f[4 * i + a]) * h[4 * j + b];
        }
    return t;
}

/* Lattice sums of the Wilson currents (Currents.cpp:7-394 for three colours):
 * out = {sum jV^0, N_5 = sum jA^0, sum PS, sum WA}. */
void orc3_charges(const orc_params *p, const double *U, const double *psi, int nmodes, int first, double out[4]) {
    const int V = volume(p);
    cplx gV0[4][4], gA0[4][4], gPS[4][4], gAw[4][4], t[4][4];
    mat4_mul(G0, G0, gV0);
    mat4_mul(gV0, G5, gA0);
    mat4_mul(G0, G5, t);
    mat4_scale(I, t, gPS);
    mat4_scale(-I * p->r_wilson, t, gAw);
    double acc[4] = {0, 0, 0, 0};
    for (int m = 0; m < nmodes; m++) {
        const double w = ((first + m) % 2 == 0) ? 1.0 : -1.0;
        const cplx *mode = (const cplx *)psi + (size_t)SPINOR3 * V * m;
        for (int s = 0; s < V; s++) {
            const cplx *f = mode + SPINOR3 * s;
            acc[0] += w * creal(bilinear3(gV0, NULL, f, f));
            acc[1] += w * creal(bilinear3(gA0, NULL, f, f));
            acc[2] += w * creal(bilinear3(gPS, NULL, f, f));
            cplx anomaly = -2.0 * 3.0 * bilinear3(gAw, NULL, f, f);
            for (int mu = 0; mu < 3; mu++) {
                const int sb = shift(p, s, mu, -1);
                m3 Mf = m3_load(U, s, mu), Mb = m3_load(U, sb, mu);
                dress3(p, s, mu, &Mf);
                dress3(p, sb, mu, &Mb);
                m3 Mbd = m3_dag(&Mb);
                anomaly += bilinear3(gAw, &Mf, f, mode + SPINOR3 * shift(p, s, mu, +1)) +
                           bilinear3(gAw, &Mbd, f, mode + SPINOR3 * sb);
            }
            acc[3] += w * creal(anomaly);
        }
    }
    for (int k = 0; k < 4; k++) out[k] = acc[k] / (2.0 * V);
}

/* Improved E and B for three colours (ChernSimonsOperators.cpp:128-439, as
 * improved_e / improved_b above). */
static void improved_e3(const orc_params *p, const double *U, const double *E, int s, int mu, double out[8]) {
    const int sp = shift(p, s, mu, +1), sm = shift(p, s, mu, -1), smm = shift(p, s, mu, -2);
    double Rp[8][8], Rm[8][8], Rmm[8][8];
    m3 u0 = m3_load(U, s, mu), um = m3_load(U, sm, mu), umm = m3_load(U, smm, mu);
    m3 umd = m3_dag(&um), ummd = m3_dag(&umm), t = m3_mul(&umd, &ummd);
    su3_adjoint(&u0, Rp);
    su3_adjoint(&umd, Rm);
    su3_adjoint(&t, Rmm);
    const double *ep = E + 8 * (mu + 3 * sp), *e0 = E + 8 * (mu + 3 * s);
    const double *em = E + 8 * (mu + 3 * sm), *emm = E + 8 * (mu + 3 * smm);
    for (int a = 0; a < 8; a++) {
        double v = (7.0 / 12.0) * e0[a];
        for (int b = 0; b < 8; b++)
            v += -(1.0 / 12.0) * Rp[a][b] * ep[b] + (7.0 / 12.0) * Rm[a][b] * em[b] - (1.0 / 12.0) * Rmm[a][b] * emm[b];
        out[a] = v;
    }
}

static void improved_b3(const orc_params *p, const double *U, int s, int mu, int nu, double out[8]) {
    m3 avg;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) avg.m[i][j] = 0;
    const int sg[4][2] = {{+1, +1}, {-1, +1}, {-1, -1}, {+1, -1}};
    for (int q = 0; q < 4; q++) {
        m3 box = m3_loop(p, U, s, mu, nu, sg[q][0], sg[q][1], 1, 1);
        m3 r1 = m3_loop(p, U, s, mu, nu, sg[q][0], sg[q][1], 2, 1);
        m3 r2 = m3_loop(p, U, s, mu, nu, sg[q][0], sg[q][1], 1, 2);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                avg.m[i][j] += (5.0 / 12.0) * box.m[i][j] - (1.0 / 24.0) * (r1.m[i][j] + r2.m[i][j]);
    }
    for (int a = 0; a < 8; a++) out[a] = 2.0 * su3_retr_ita(&avg, a);
}

double orc3_ncsdot(const orc_params *p, const double *U, const double *E) {
    const int V = volume(p);
    const int plane[3][2] = {{1, 2}, {2, 0}, {0, 1}};
    double edotb = 0.0;
    for (int s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            double e[8], b[8];
            improved_e3(p, U, E, s, mu, e);
            improved_b3(p, U, s, plane[mu][0], plane[mu][1], b);
            for (int a = 0; a < 8; a++) edotb += e[a] * b[a];
        }
    return 0.125 * edotb / (M_PI * M_PI);
}

/* Geodesic interpolation between two link sets and Delta N_CS along it with
 * Simpson weights 1, 4, 1 (CoolingMethod.cpp:80-125, as ovl_ncs_update). */
double orc3_delta_ncs(const orc_params *p, const double *Uold, const double *Unew) {
    const int V = volume(p);
    double *Umid = malloc(sizeof(double) * 54 * (size_t)V), *Emid = malloc(sizeof(double) * 24 * (size_t)V);
    for (int s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            m3 uo = m3_load(Uold, s, mu), un = m3_load(Unew, s, mu), uod = m3_dag(&uo);
            m3 W = m3_mul(&un, &uod);
            double *e = Emid + 8 * (mu + 3 * s), g[18];
            su3_log(&W, e);
            orc3_exp(-0.5, e, g);  /* exp(-i c E_mid t), c = 1/2 */
            m3 G = m3_load(g, 0, 0), um = m3_mul(&G, &uo);
            m3_store(Umid, s, mu, &um);
        }
    const double d = (4.0 * orc3_ncsdot(p, Umid, Emid) + orc3_ncsdot(p, Uold, Emid) + orc3_ncsdot(p, Unew, Emid)) / 6.0;
    free(Umid);
    free(Emid);
    return d;
}

/* {T00, TXX, TYY, TZZ, E part, B part, gauss max, gauss rms, unit max, unit rms}
 * for three colours (BulkObservables.cpp:17-152, GaussLawViolation.cpp:13-67,
 * UnitarityViolation.cpp:13-51): B^2 = 4 Re tr(1 - U_plaq). */
void orc3_bulk(const orc_params *p, const double *U, const double *E, double *out) {
    const int V = volume(p);
    const int plane[3][2] = {{1, 2}, {2, 0}, {0, 1}};
    double e2[3] = {0, 0, 0}, b2[3] = {0, 0, 0}, gmax = 0.0, gsum = 0.0, umax = 0.0, usum = 0.0;
    for (int s = 0; s < V; s++) {
        for (int mu = 0; mu < 3; mu++)
            for (int a = 0; a < 8; a++) e2[mu] += E[a + 8 * (mu + 3 * s)] * E[a + 8 * (mu + 3 * s)];
        for (int k = 0; k < 3; k++) {
            m3 pl = m3_loop(p, U, s, plane[k][0], plane[k][1], +1, +1, 1, 1);
            b2[k] += 4.0 * (3.0 - creal(pl.m[0][0] + pl.m[1][1] + pl.m[2][2]));
        }
        double g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int mu = 0; mu < 3; mu++) {
            const int sm = shift(p, s, mu, -1);
            m3 um = m3_load(U, sm, mu), umd = m3_dag(&um);
            double R[8][8];
            su3_adjoint(&umd, R);
            for (int a = 0; a < 8; a++) {
                double t = E[a + 8 * (mu + 3 * s)];
                for (int b = 0; b < 8; b++) t -= R[a][b] * E[b + 8 * (mu + 3 * sm)];
                g[a] += t;
            }
        }
        for (int a = 0; a < 8; a++) {
            gmax = fmax(gmax, g[a]);
            gsum += g[a] * g[a];
        }
        for (int mu = 0; mu < 3; mu++) {
            m3 u = m3_load(U, s, mu), ud = m3_dag(&u), c = m3_mul(&u, &ud);
            double n = 0.0;
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    cplx d = c.m[i][j] - (i == j ? 1.0 : 0.0);
                    n += creal(d * conj(d));
                }
            n = sqrt(n);
            umax = fmax(umax, n);
            usum += n * n;
        }
    }
    for (int k = 0; k < 3; k++) { e2[k] /= V; b2[k] /= V; }
    out[0] = 0.5 * (e2[0] + e2[1] + e2[2] + b2[0] + b2[1] + b2[2]);
    out[1] = 0.5 * ((e2[1] + e2[2] + b2[1] + b2[2]) - (e2[0] + b2[0]));
    out[2] = 0.5 * ((e2[0] + e2[2] + b2[0] + b2[2]) - (e2[1] + b2[1]));
    out[3] = 0.5 * ((e2[0] + e2[1] + b2[0] + b2[1]) - (e2[2] + b2[2]));
    out[4] = 0.5 * (e2[0] + e2[1] + e2[2]);
    out[5] = 0.5 * (b2[0] + b2[1] + b2[2]);
    out[6] = gmax;
    out[7] = sqrt(gsum / (8.0 * V));  /* over the Nc^2 - 1 components (GaussLawViolation.cpp:64) */
    out[8] = umax;
    out[9] = sqrt(usum / (3.0 * V));
}

/* Gauss violation G^a(x) = sum_mu E_mu(x) - R(U_mu(x-mu)^+) E_mu(x-mu) into G
 * (8 per site); returns the signed maximum (from 0), *avg the rms over the 8 V
 * components. */
static double gauss_violation3(const orc_params *p, const double *U, const double *E, double *G, double *avg) {
    const int V = volume(p);
    double mx = 0.0, sum = 0.0;
    for (int s = 0; s < V; s++) {
        double g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int mu = 0; mu < 3; mu++) {
            const int sm = shift(p, s, mu, -1);
            m3 um = m3_load(U, sm, mu), umd = m3_dag(&um);
            double R[8][8];
            su3_adjoint(&umd, R);
            for (int a = 0; a < 8; a++) {
                double t = E[a + 8 * (mu + 3 * s)];
                for (int b = 0; b < 8; b++) t -= R[a][b] * E[b + 8 * (mu + 3 * sm)];
                g[a] += t;
            }
        }
        for (int a = 0; a < 8; a++) {
            G[a + 8 * s] = g[a];
            mx = fmax(mx, g[a]);
            sum += g[a] * g[a];
        }
    }
    *avg = sqrt(sum / (8.0 * V));
    return mx;
}

/* E_mu(x) -= gamma (G(x) - R(U_mu(x)) G(x + mu)) (GaussRestore.cpp:72-118, three colours) */
static void gauss_update3(const orc_params *p, const double *U, const double *G, double *E, double gamma) {
    const int V = volume(p);
    for (int s = 0; s < V; s++)
        for (int mu = 0; mu < 3; mu++) {
            const int sp = shift(p, s, mu, +1);
            m3 u = m3_load(U, s, mu);
            double R[8][8];
            su3_adjoint(&u, R);
            for (int a = 0; a < 8; a++) {
                double up = 0.0;
                for (int b = 0; b < 8; b++) up += R[a][b] * G[b + 8 * sp];
                E[a + 8 * (mu + 3 * s)] -= gamma * (G[a + 8 * s] - up);
            }
        }
}

/* GaussLawRestoration::Restore (GaussRestore.cpp:132-168) for three colours. */
int orc3_gauss_restore(const orc_params *p, const double *U, double *E, int max_iter, double tol, double *out2) {
    const int V = volume(p);
    double *G = malloc(sizeof(double) * 8 * (size_t)V);
    double avg = 0.0;
    double mx = gauss_violation3(p, U, E, G, &avg);
    int n = 0;
    static const double gammas[3] = {7.0 / 24.0, 7.0 / 48.0, 7.0 / 72.0};
    while (n < max_iter && mx > tol) {
        for (int k = 0; k < 3; k++) {
            mx = gauss_violation3(p, U, E, G, &avg);
            gauss_update3(p, U, G, E, gammas[k]);
        }
        n++;
    }
    free(G);
    if (out2) { out2[0] = mx; out2[1] = avg; }
    return n;
}

/* dH_F/dtheta^a_mu(x) for three colours (orc_color_force with 3x3 links and
 * t^a = lambda^a / 2): -(1/2V) sum_m w_m Re[psi(x)^+ g0 (1 - G_mu) i t^a U_mu(x) psi(x+mu)],
 * out[a + 8 (mu + 3 site)]. */
void orc3_color_force(const orc_params *p, const double *U, const double *psi, int nmodes, int first, double *out) {
    const int V = volume(p);
    cplx G[3][4][4], gp[3][4][4];
    mat4_scale(-I, GX, G[0]);
    mat4_scale(-I, GY, G[1]);
    mat4_scale(-I, GZ, G[2]);
    for (int mu = 0; mu < 3; mu++) {
        cplx t[4][4];
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) t[a][b] = (a == b) - G[mu][a][b];
        mat4_mul(G0, t, gp[mu]);
    }
    m3 T[8];
    for (int a = 0; a < 8; a++) T[a] = su3_generator(a);
    memset(out, 0, sizeof(double) * 24 * (size_t)V);
    const double pre = 1.0 / (2.0 * V);
    for (int m = 0; m < nmodes; m++) {
        const double w = ((first + m) % 2 == 0) ? 1.0 : -1.0;
        const cplx *mode = (const cplx *)psi + (size_t)SPINOR3 * V * m;
        for (int s = 0; s < V; s++) {
            const cplx *f = mode + SPINOR3 * s;
            for (int mu = 0; mu < 3; mu++) {
                m3 M = m3_load(U, s, mu);
                dress3(p, s, mu, &M);
                const cplx *h = mode + SPINOR3 * shift(p, s, mu, +1);
                for (int a = 0; a < 8; a++) {
                    m3 A = m3_mul(&T[a], &M);  /* i t^a M */
                    cplx b = 0;
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++)
                            for (int al = 0; al < 4; al++)
                                for (int be = 0; be < 4; be++)
                                    if (gp[mu][al][be] != 0)
                                        b += conj(f[4 * i + al]) * gp[mu][al][be] * I * A.m[i][j] * h[4 * j + be];
                    out[a + 8 * (mu + 3 * s)] += -pre * w * creal(b);
                }
            }
        }
    }
}

double orc3_fermion_energy(const orc_params *p, const double *U, const double *psi, int nmodes, int first) {
    const int V = volume(p);
    const size_t per_mode = (size_t)2 * SPINOR3 * V;
    double *work = malloc(sizeof(double) * per_mode);
    double e = 0.0;
    for (int m = 0; m < nmodes; m++) {
        const double w = ((first + m) % 2 == 0) ? 1.0 : -1.0;
        orc3_wilson_apply(p, U, psi + per_mode * m, work);
        const cplx *f = (const cplx *)(psi + per_mode * m), *d = (const cplx *)work;
        cplx t = 0;
        for (int k = 0; k < SPINOR3 * V; k++) t += conj(f[k]) * I * d[k];
        e += w * creal(t);
    }
    free(work);
    return e / (2.0 * V);
}

/* The coupled leapfrog (orc_coupled_leapfrog) for three colours. */
void orc3_coupled_leapfrog(const orc_params *p, double *U, double *E, double *psi, double *psimid, int nmodes,
                           int first, int *tsteps, int nsteps, double g2, int gauge) {
    const int V = volume(p);
    double *force = malloc(sizeof(double) * 24 * (size_t)V);
    for (int n = 0; n < nsteps; n++) {
        orc3_wilson_leapfrog(p, U, E, psi, psimid, nmodes, tsteps, 1);
        if (gauge) orc3_update_efield(p, U, E, p->dt);
        if (g2 != 0.0) {
            orc3_color_force(p, U, psi, nmodes, first, force);
            for (size_t k = 0; k < 24 * (size_t)V; k++) E[k] += p->dt * g2 * force[k];
        }
    }
    free(force);
}

/* Chebyshev coefficients of x^(-1/2) on [eps, 1] (c_0 with weight 1/2), by
 * Chebyshev-Gauss quadrature on max(4K, 256) nodes. */
void orc_chebyshev_coeffs(int K, double eps, double *c) {
    const int M = 4 * K > 256 ? 4 * K : 256;
    for (int k = 0; k <= K; k++) {
        double s = 0.0;
        for (int j = 0; j < M; j++) {
            const double th = M_PI * (j + 0.5) / M;
            const double x = 0.5 * (1.0 + eps) + 0.5 * (1.0 - eps) * cos(th);
            s += cos(k * th) / sqrt(x);
        }
        c[k] = 2.0 * s / M;
    }
}

/* The overlap evolution operator with the Chebyshev inverse square root, for
 * three colours:  out = M [ -i g0 (1 + m/2) phi + (1 - m/2) D chi ],
 * chi = lambda_max^(-1/2) [c_0/2 + sum_k c_k T_k(t)] phi,
 * t = (2 h^2 / lambda_max - 1 - eps) / (1 - eps),  h^2 = -D^2  (OverlapU.cpp:188-202
 * with the series in place of the Zolotarev solve). */
void orc3_overlap_apply(const orc_params *p, const double *U, const double *phi, double *out, int K, double eps,
                        double lambda_max) {
    const size_t n = (size_t)SPINOR3 * volume(p);
    cplx *b0 = calloc(n, sizeof(cplx)), *b1 = calloc(n, sizeof(cplx)), *b2 = calloc(n, sizeof(cplx));
    cplx *w = malloc(n * sizeof(cplx)), *x = malloc(n * sizeof(cplx));
    double *c = malloc(sizeof(double) * (K + 1));
    orc_chebyshev_coeffs(K, eps, c);
    const double a = 2.0 / ((1.0 - eps) * lambda_max), beta = -(1.0 + eps) / (1.0 - eps);
    const double scale = 1.0 / sqrt(lambda_max);
    const cplx *f = (const cplx *)phi;
    for (int k = K; k >= 0; k--) {
        /* x = t(X) b1 = a (-D^2 b1) + beta b1 */
        orc3_wilson_apply(p, U, (const double *)b1, (double *)w);
        orc3_wilson_apply(p, U, (const double *)w, (double *)x);
        const double factor = k > 0 ? 2.0 : 1.0, ck = (k > 0 ? c[k] : 0.5 * c[0]) * scale;
        for (size_t e = 0; e < n; e++) b0[e] = factor * (-a * x[e] + beta * b1[e]) - b2[e] + ck * f[e];
        cplx *t = b2;
        b2 = b1;
        b1 = b0;
        b0 = t;
    }
    /* chi = b1; D chi */
    orc3_wilson_apply(p, U, (const double *)b1, (double *)w);
    const double cp = 1.0 + 0.5 * p->m_fermion, cm = 1.0 - 0.5 * p->m_fermion;
    cplx *o = (cplx *)out;
    for (size_t e = 0; e < n; e++) {
        const int spin = (int)(e % 4);
        const cplx g = (spin < 2 ? -I : I) * cp * f[e];
        o[e] = p->m_dw * (g + cm * w[e]);
    }
    free(b0); free(b1); free(b2); free(w); free(x); free(c);
}

/* The overlap leapfrog (OverlapUpdate.cpp:99-135) for three colours with the
 * Chebyshev operator and a fixed lambda_max. */
void orc3_overlap_leapfrog(const orc_params *p, double *U, const double *E, double *psi, double *psimid, int nmodes,
                           int *tsteps, int nsteps, int K, double eps, double lambda_max) {
    const size_t per_mode = (size_t)2 * SPINOR3 * volume(p);
    double *work = malloc(sizeof(double) * per_mode);
    for (int n = 0; n < nsteps; n++) {
        for (int h = 0; h < 2; h++) {
            const double *src = h == 0 ? psimid : psi;
            double *dst = h == 0 ? psi : psimid;
            for (int m = 0; m < nmodes; m++) {
                orc3_overlap_apply(p, U, src + per_mode * m, work, K, eps, lambda_max);
                for (size_t k = 0; k < per_mode; k++) dst[per_mode * m + k] += p->dt * work[k];
            }
            if (p->qs * (*tsteps * p->dt) < p->t_sphaleron) orc3_update_links(p, U, E, 0.5 * p->dt);
        }
        (*tsteps)++;
    }
    free(work);
}

/* ------------------------------------------------------------ cooling -- */
/* Gradient-flow cooling and the Chern-Simons calibration, both colours
 * (GRADIENTFLOW/GradientFlow.cpp:35-190, GRADIENTFLOW/Cooling.cpp:71-201,
 * TOPOLOGY/CoolingMethod.cpp:168-196, TOPOLOGY/VacuumEstimator.cpp:7-85,
 * LATTICE/GaugeLinks.cpp:126-153), Minkowski metric, aScale 1, spacing
 * a = 2^level in every direction. */

/* f(a,b,c) as the vacuum estimator reads it: the Levi-Civita symbol for two
 * colours; for three, the reference's table written for labels 1..8 called
 * with components 0..7 (SU3/AlgebraOperations.cpp:28-76), so only the
 * entries with all labels <= 7 are reached. */
static double cool_f(int nc, int a, int b, int c) {
    const int prod = (a - b) * (a - c) * (c - b);
    if (prod == 0) return 0.0;
    if (nc == 2) return 0.5 * prod;
    int t[3] = {a, b, c};
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++)
            if (t[j] < t[i]) { int x = t[i]; t[i] = t[j]; t[j] = x; }
    const int key = 100 * t[0] + 10 * t[1] + t[2];
    double base = 0.0;
    if (key == 123) base = 1.0;
    else if (key == 147 || key == 246 || key == 257 || key == 345) base = 0.5;
    else if (key == 156 || key == 367) base = -0.5;
    return prod > 0 ? base : -base;
}

/* ReTrIGenU(2, U_mu(s)): 2 Re tr(i t^a U). */
static void cool_algebra(const orc_params *p, int nc, const double *U, int s, int mu, double *A) {
    (void)p;
    if (nc == 2) {
        quat q = q_load(U, s, mu);
        for (int a = 0; a < 3; a++) A[a] = 2.0 * q_retr_ita(q, a);
    } else {
        m3 V = m3_load(U, s, mu);
        for (int a = 0; a < 8; a++) A[a] = 2.0 * su3_retr_ita(&V, a);
    }
}

double orc_vacuum_ncs(const orc_params *p, int nc, const double *U) {
    const int V = volume(p), na = nc * nc - 1;
    double sum = 0.0;
    for (int s = 0; s < V; s++) {
        double A[3][8];
        for (int mu = 0; mu < 3; mu++) {
            double ap[8], am[8];
            cool_algebra(p, nc, U, s, mu, ap);
            cool_algebra(p, nc, U, shift(p, s, mu, -1), mu, am);
            for (int a = 0; a < na; a++) A[mu][a] = 0.5 * (ap[a] + am[a]);
        }
        for (int a = 0; a < na; a++)
            for (int b = 0; b < na; b++)
                for (int c = 0; c < na; c++) {
                    const double f = cool_f(nc, a, b, c);
                    if (f != 0.0) sum += 1.0 / (16.0 * M_PI * M_PI) * f * A[0][a] * A[1][b] * A[2][c];
                }
    }
    return sum;
}

void orc_block_links(const orc_params *p, int nc, const double *U, double *Uout) {
    orc_params q = *p;
    for (int k = 0; k < 3; k++) q.N[k] = p->N[k] / 2;
    const int Vb = volume(&q);
    for (int s = 0; s < Vb; s++) {
        int c[3];
        coords_of(&q, s, c);
        for (int mu = 0; mu < 3; mu++) {
            int f[3] = {2 * c[0], 2 * c[1], 2 * c[2]};
            const int s0 = site_of(p, f[0], f[1], f[2]);
            f[mu] += 1;
            const int s1 = site_of(p, f[0], f[1], f[2]);
            if (nc == 2) {
                quat u = q_mul(q_load(U, s0, mu), q_load(U, s1, mu));
                memcpy(Uout + 4 * (mu + 3 * s), u.v, sizeof u.v);
            } else {
                m3 a = m3_load(U, s0, mu), b = m3_load(U, s1, mu);
                m3 u = m3_mul(&a, &b);
                m3_store(Uout, s, mu, &u);
            }
        }
    }
}

typedef struct {
    orc_params q;  /* the current lattice */
    int nc;
    double *U, *Ub, *E;
    double a, aCube, tau, dncs;
    int steps, blocking;
    double *log;
    int rows, max_rows;
} cool_state;

static size_t cool_link_doubles(int nc) { return nc == 3 ? 18 : 4; }

static void cool_row(cool_state *st) {
    const int nc = st->nc;
    double b[10];
    if (nc == 2) orc_bulk(&st->q, st->U, st->E, b);
    else orc3_bulk(&st->q, st->U, st->E, b);
    const double c = (st->a / st->aCube) * (st->a / st->aCube);  /* Bulk::SetConstants */
    if (st->log && st->rows < st->max_rows) {
        double *r = st->log + 5 * (size_t)st->rows;
        r[0] = st->tau;
        r[1] = c * b[5];
        r[2] = c * b[4];
        r[3] = st->dncs;
        r[4] = orc_vacuum_ncs(&st->q, nc, st->U);
    }
    st->rows++;
}

static void cool_step(cool_state *st, int calibrate) {
    const int nc = st->nc, V = volume(&st->q);
    const double s = 0.5 / M_SQRT2, pw = pow(st->aCube, 2.0 / 3.0);
    const double DcTau = s * s * pw;
    const double gamma = -2.0 * st->aCube, cE = 1.0 / (st->a * st->a);
    const double cU = -1.0 * (st->a * st->a * (s * s * pw)) / st->aCube;
    const double cS = st->a * st->a / st->aCube;
    memset(st->E, 0, sizeof(double) * (size_t)(nc * nc - 1) * 3 * V);
    /* E = gamma cE^2 (staple sum): the staple routine adds -2 dt (staple sum) */
    if (nc == 2) orc_update_efield(&st->q, st->U, st->E, -0.5 * gamma * cE * cE);
    else orc3_update_efield(&st->q, st->U, st->E, -0.5 * gamma * cE * cE);
    if (calibrate) st->dncs += 0.5 * DcTau * (cS * (nc == 2 ? orc_ncsdot(&st->q, st->U, st->E) : orc3_ncsdot(&st->q, st->U, st->E)));
    if (nc == 2) orc_update_links(&st->q, st->U, st->E, -cU);
    else orc3_update_links(&st->q, st->U, st->E, -cU);
    if (calibrate) st->dncs += 0.5 * DcTau * (cS * (nc == 2 ? orc_ncsdot(&st->q, st->U, st->E) : orc3_ncsdot(&st->q, st->U, st->E)));
    st->steps++;
    st->tau += DcTau;
}

static void cool_perform(cool_state *st, int max_steps, int max_blocking, int block_frequency, int calibrate) {
    if (calibrate) cool_row(st);
    while (st->steps < max_steps) {
        cool_step(st, calibrate);
        if (calibrate) cool_row(st);
        long long period = block_frequency;
        for (int k = 0; k < st->blocking; k++) period *= 8;
        if (st->steps % period == 0 && st->blocking < max_blocking) {
            orc_block_links(&st->q, st->nc, st->U, st->Ub);
            double *t = st->U; st->U = st->Ub; st->Ub = t;
            for (int k = 0; k < 3; k++) st->q.N[k] /= 2;
            st->a *= 2.0;
            st->aCube = st->a * st->a * st->a;
            memset(st->E, 0, sizeof(double) * (size_t)(st->nc * st->nc - 1) * 3 * volume(&st->q));
            st->blocking++;
        }
    }
}

int orc_cool(const orc_params *p, int nc, const double *U0, int standard_steps, int standard_blocking,
             int calibration_steps, int calibration_blocking, int block_frequency, double *log, int *rows,
             double out[3], double *cooled, int cooled_N[3]) {
    const int V = volume(p);
    const size_t nl = cool_link_doubles(nc) * 3 * (size_t)V, ne = (size_t)(nc * nc - 1) * 3 * V;
    cool_state st;
    memset(&st, 0, sizeof st);
    st.q = *p;
    st.nc = nc;
    st.U = malloc(sizeof(double) * nl);
    st.Ub = malloc(sizeof(double) * nl);
    st.E = calloc(ne, sizeof(double));
    memcpy(st.U, U0, sizeof(double) * nl);
    st.a = 1.0;
    st.aCube = 1.0;
    /* CoolNSave */
    cool_perform(&st, standard_steps, standard_blocking, block_frequency, 0);
    if (cooled_N) for (int k = 0; k < 3; k++) cooled_N[k] = st.q.N[k];
    if (cooled) memcpy(cooled, st.U, sizeof(double) * cool_link_doubles(nc) * 3 * (size_t)volume(&st.q));
    /* Calibrate: DeltaNCsCooling = 0, E zero, counters continue */
    st.dncs = 0.0;
    memset(st.E, 0, sizeof(double) * ne);
    st.log = log;
    st.max_rows = calibration_steps + 1;
    cool_perform(&st, standard_steps + calibration_steps, calibration_blocking, block_frequency, 1);
    if (rows) *rows = st.rows;
    if (out) { out[0] = st.dncs; out[1] = st.tau; out[2] = st.blocking; }
    free(st.U); free(st.Ub); free(st.E);
    return 0;
}
