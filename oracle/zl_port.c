/*
 * ORACLE — test infrastructure only (see zl_port.h).  Plain-C restatement of
 * the reference's single-level LBM step in the reference's own arithmetic
 * order, so that with strict IEEE flags (-O2 -fno-fast-math -ffp-contract=off)
 * it reproduces the reference's doubles bit for bit.
 *
 * Reference functions restated here (paths inside the reference project):
 *   lattice tables      lbm_project/d2q9_model/lbm_d2q9.h:53-92, d3q19_model/lbm_d3q19.h:18-167
 *   macros              lbm_project/lbm_solver_interface.cpp:477-592
 *   feq                 lbm_project/lbm_solver_interface.cpp:374-435
 *   Guo forcing term    lbm_project/lbm_solver_interface.cpp:443-470
 *   collision dispatch  lbm_project/lbm_solver_interface.cpp:266-323
 *   SRT                 lbm_project/collision_model/lbm_collision_model_srt.cpp:20-39
 *   MRT                 lbm_project/collision_model/lbm_collision_model_mrt.cpp:46-143
 *   tau per level       lbm_project/collision_model/lbm_collision_models.cpp:105-118
 *   pull stream         lbm_project/d3q19_model/lbm_d3q19_solver.cpp:20-136 (d2q9 analogue)
 *   BC order            lbm_project/lbm_grid_interface.cpp:225-314
 *   bounce back         lbm_project/boundary_conditions/lbm_bounce_back.cpp:28-91
 *   periodic            lbm_project/boundary_conditions/lbm_periodic.cpp:22-133
 *   NEQ extrapolation   lbm_project/boundary_conditions/lbm_noneq_extrapolation.cpp:27-144
 *   Smagorinsky         lbm_project/les_models/lbm_les_smagorinsky.cpp:22-94, with the
 *                       relaxation time used as tau0 + tau_sgs (the reference passes
 *                       tau_sgs alone, lbm_solver_interface.cpp:291-295; documented deviation)
 */
#include "zl_port.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- lattice tables (same direction order as the reference) ---- */
static const double kCx9[9] = {0., 1., 0., -1., 0., 1., -1., -1., 1.};
static const double kCy9[9] = {0., 0., 1., 0., -1., 1., 1., -1., -1.};
static const double kCz9[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
static const double kW9[9] = {4. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 36., 1. / 36., 1. / 36., 1. / 36.};
/* directions entering through a min face of an axis (c_axis > 0) and their inverses */
static const int kPos9[2][3] = {{1, 8, 5}, {2, 5, 6}};
static const int kNeg9[2][3] = {{3, 7, 6}, {4, 7, 8}};

static const double kCx19[19] = {0., 1., -1., 0., 0., 0., 0., 1., -1., 1., -1., 1., -1., 1., -1., 0., 0., 0., 0.};
static const double kCy19[19] = {0., 0., 0., 1., -1., 0., 0., 1., 1., -1., -1., 0., 0., 0., 0., 1., -1., 1., -1.};
static const double kCz19[19] = {0., 0., 0., 0., 0., 1., -1., 0., 0., 0., 0., 1., 1., -1., -1., 1., 1., -1., -1.};
static const double kW19[19] = {1. / 3., 1. / 18., 1. / 18., 1. / 18., 1. / 18., 1. / 18., 1. / 18.,
                                1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36.,
                                1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36.};
static const int kPos19[3][5] = {{1, 7, 9, 11, 13}, {3, 7, 8, 15, 17}, {5, 11, 12, 15, 16}};
static const int kNeg19[3][5] = {{2, 10, 8, 14, 12}, {4, 10, 9, 18, 16}, {6, 14, 13, 18, 17}};

/* MRT moment matrices (Lallemand-Luo D2Q9, d'Humieres D3Q19) in the reference's row order */
static const double kM9[9][9] = {
    {1., 1., 1., 1., 1., 1., 1., 1., 1.},     {-4., -1., -1., -1., -1., 2., 2., 2., 2.},
    {4., -2., -2., -2., -2., 1., 1., 1., 1.}, {0., 1., 0., -1., 0., 1., -1., -1., 1.},
    {0., -2., 0., 2., 0., 1., -1., -1., 1.},  {0., 0., 1., 0., -1., 1., 1., -1., -1.},
    {0., 0., -2., 0., 2., 1., 1., -1., -1.},  {0., 1., -1., 1., -1., 0., 0., 0., 0.},
    {0., 0., 0., 0., 0., 1., -1., 1., -1.}};
static const double kIm9[9][9] = {
    {1. / 9., -1. / 9., 1. / 9., 0., 0., 0., 0., 0., 0.},
    {1. / 9., -1. / 36., -1. / 18., 1. / 6., -1. / 6., 0., 0., 1. / 4., 0.},
    {1. / 9., -1. / 36., -1. / 18., 0., 0., 1. / 6., -1. / 6., -1. / 4., 0.},
    {1. / 9., -1. / 36., -1. / 18., -1. / 6., 1. / 6., 0., 0., 1. / 4., 0.},
    {1. / 9., -1. / 36., -1. / 18., 0., 0., -1. / 6., 1. / 6., -1. / 4., 0.},
    {1. / 9., 1. / 18., 1. / 36., 1. / 6., 1. / 12., 1. / 6., 1. / 12., 0., 1. / 4.},
    {1. / 9., 1. / 18., 1. / 36., -1. / 6., -1. / 12., 1. / 6., 1. / 12., 0., -1. / 4.},
    {1. / 9., 1. / 18., 1. / 36., -1. / 6., -1. / 12., -1. / 6., -1. / 12., 0., 1. / 4.},
    {1. / 9., 1. / 18., 1. / 36., 1. / 6., 1. / 12., -1. / 6., -1. / 12., 0., -1. / 4.}};
static const double kS9[9] = {0., 1.4, 1.4, 0., 1.2, 0., 1.2, 0., 0.};
static const int kTauRows9[2] = {7, 8};

static const double kM19[19][19] = {
    {1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1.},
    {-30., -11., -11., -11., -11., -11., -11., 8., 8., 8., 8., 8., 8., 8., 8., 8., 8., 8., 8.},
    {12., -4., -4., -4., -4., -4., -4., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1., 1.},
    {0., 1., -1., 0., 0., 0., 0., 1., -1., 1., -1., 1., -1., 1., -1., 0., 0., 0., 0.},
    {0., -4., 4., 0., 0., 0., 0., 1., -1., 1., -1., 1., -1., 1., -1., 0., 0., 0., 0.},
    {0., 0., 0., 1., -1., 0., 0., 1., 1., -1., -1., 0., 0., 0., 0., 1., -1., 1., -1.},
    {0., 0., 0., -4., 4., 0., 0., 1., 1., -1., -1., 0., 0., 0., 0., 1., -1., 1., -1.},
    {0., 0., 0., 0., 0., 1., -1., 0., 0., 0., 0., 1., 1., -1., -1., 1., 1., -1., -1.},
    {0., 0., 0., 0., 0., -4., 4., 0., 0., 0., 0., 1., 1., -1., -1., 1., 1., -1., -1.},
    {0., 2., 2., -1., -1., -1., -1., 1., 1., 1., 1., 1., 1., 1., 1., -2., -2., -2., -2.},
    {0., -4., -4., 2., 2., 2., 2., 1., 1., 1., 1., 1., 1., 1., 1., -2., -2., -2., -2.},
    {0., 0., 0., 1., 1., -1., -1., 1., 1., 1., 1., -1., -1., -1., -1., 0., 0., 0., 0.},
    {0., 0., 0., -2., -2., 2., 2., 1., 1., 1., 1., -1., -1., -1., -1., 0., 0., 0., 0.},
    {0., 0., 0., 0., 0., 0., 0., 1., -1., -1., 1., 0., 0., 0., 0., 0., 0., 0., 0.},
    {0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 1., -1., -1., 1.},
    {0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 1., -1., -1., 1., 0., 0., 0., 0.},
    {0., 0., 0., 0., 0., 0., 0., 1., -1., 1., -1., -1., 1., -1., 1., 0., 0., 0., 0.},
    {0., 0., 0., 0., 0., 0., 0., -1., -1., 1., 1., 0., 0., 0., 0., 1., -1., 1., -1.},
    {0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 1., 1., -1., -1., -1., -1., 1., 1.}};
#define I19 (1. / 19)
#define A (-11. / 2394)
#define B (-1. / 63)
#define C4 (4. / 1197)
#define D (1. / 252)
static const double kIm19[19][19] = {
    {I19, -5. / 399, 1. / 21, 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0.},
    {I19, A, B, 0.1, -0.1, 0., 0., 0., 0., 1. / 18, -1. / 18, 0., 0., 0., 0., 0., 0., 0., 0.},
    {I19, A, B, -0.1, 0.1, 0., 0., 0., 0., 1. / 18, -1. / 18, 0., 0., 0., 0., 0., 0., 0., 0.},
    {I19, A, B, 0., 0., 0.1, -0.1, 0., 0., -1. / 36, 1. / 36, 1. / 12, -1. / 12, 0., 0., 0., 0., 0., 0.},
    {I19, A, B, 0., 0., -0.1, 0.1, 0., 0., -1. / 36, 1. / 36, 1. / 12, -1. / 12, 0., 0., 0., 0., 0., 0.},
    {I19, A, B, 0., 0., 0., 0., 0.1, -0.1, -1. / 36, 1. / 36, -1. / 12, 1. / 12, 0., 0., 0., 0., 0., 0.},
    {I19, A, B, 0., 0., 0., 0., -0.1, 0.1, -1. / 36, 1. / 36, -1. / 12, 1. / 12, 0., 0., 0., 0., 0., 0.},
    {I19, C4, D, 0.1, 0.025, 0.1, 0.025, 0., 0., 1. / 36, 1. / 72, 1. / 12, 1. / 24, 0.25, 0., 0., 0.125, -0.125, 0.},
    {I19, C4, D, -0.1, -0.025, 0.1, 0.025, 0., 0., 1. / 36, 1. / 72, 1. / 12, 1. / 24, -0.25, 0., 0., -0.125, -0.125, 0.},
    {I19, C4, D, 0.1, 0.025, -0.1, -0.025, 0., 0., 1. / 36, 1. / 72, 1. / 12, 1. / 24, -0.25, 0., 0., 0.125, 0.125, 0.},
    {I19, C4, D, -0.1, -0.025, -0.1, -0.025, 0., 0., 1. / 36, 1. / 72, 1. / 12, 1. / 24, 0.25, 0., 0., -0.125, 0.125, 0.},
    {I19, C4, D, 0.1, 0.025, 0., 0., 0.1, 0.025, 1. / 36, 1. / 72, -1. / 12, -1. / 24, 0., 0., 0.25, -0.125, 0., 0.125},
    {I19, C4, D, -0.1, -0.025, 0., 0., 0.1, 0.025, 1. / 36, 1. / 72, -1. / 12, -1. / 24, 0., 0., -0.25, 0.125, 0., 0.125},
    {I19, C4, D, 0.1, 0.025, 0., 0., -0.1, -0.025, 1. / 36, 1. / 72, -1. / 12, -1. / 24, 0., 0., -0.25, -0.125, 0., -0.125},
    {I19, C4, D, -0.1, -0.025, 0., 0., -0.1, -0.025, 1. / 36, 1. / 72, -1. / 12, -1. / 24, 0., 0., 0.25, 0.125, 0., -0.125},
    {I19, C4, D, 0., 0., 0.1, 0.025, 0.1, 0.025, -1. / 18, -1. / 36, 0., 0., 0., 0.25, 0., 0., 0.125, -0.125},
    {I19, C4, D, 0., 0., -0.1, -0.025, 0.1, 0.025, -1. / 18, -1. / 36, 0., 0., 0., -0.25, 0., 0., -0.125, -0.125},
    {I19, C4, D, 0., 0., 0.1, 0.025, -0.1, -0.025, -1. / 18, -1. / 36, 0., 0., 0., -0.25, 0., 0., 0.125, 0.125},
    {I19, C4, D, 0., 0., -0.1, -0.025, -0.1, -0.025, -1. / 18, -1. / 36, 0., 0., 0., 0.25, 0., 0., -0.125, 0.125}};
#undef I19
#undef A
#undef B
#undef C4
#undef D
static const double kS19[19] = {0., 1.5, 1.4, 0., 1.2, 0., 1.2, 0., 1.2, 0., 1.4, 0., 1.4, 0., 0., 0., 1.98, 1.98, 1.98};
static const int kTauRows19[5] = {9, 11, 13, 14, 15};

typedef struct lattice {
    int q, dims, nface_q;
    const double *cx, *cy, *cz, *w;
} lattice;

static lattice lattice_of(int dims) {
    lattice l;
    if (dims == 2) {
        l.q = 9; l.dims = 2; l.nface_q = 3;
        l.cx = kCx9; l.cy = kCy9; l.cz = kCz9; l.w = kW9;
    } else {
        l.q = 19; l.dims = 3; l.nface_q = 5;
        l.cx = kCx19; l.cy = kCy19; l.cz = kCz19; l.w = kW19;
    }
    return l;
}

double zlp_tau(double nu, int level) {
    const double dt = 1. / (double)(1u << level);
    return nu * 3. / dt + 0.5;
}

void zlp_feq(int dims, double rho, const double* u, double* feq) {
    const lattice l = lattice_of(dims);
    if (dims == 2) {
        const double uv_sq = u[0] * u[0] + u[1] * u[1];
        for (int iq = 0; iq < l.q; ++iq) {
            const double c_uv = u[0] * l.cx[iq] + u[1] * l.cy[iq];
            feq[iq] = l.w[iq] * rho * (1. + 3. * c_uv + 4.5 * c_uv * c_uv - 1.5 * uv_sq);
        }
    } else {
        const double uv_sq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        for (int iq = 0; iq < l.q; ++iq) {
            const double c_uv = u[0] * l.cx[iq] + u[1] * l.cy[iq] + u[2] * l.cz[iq];
            feq[iq] = l.w[iq] * rho * (1. + 3. * c_uv + 4.5 * c_uv * c_uv - 1.5 * uv_sq);
        }
    }
}

/* density and momentum sums in direction order, then divide by rho (compressible default) */
static void macro_sums(const lattice* l, const double* f, double* rho, double* u) {
    *rho = f[0];
    u[0] = 0.; u[1] = 0.; u[2] = 0.;
    for (int iq = 1; iq < l->q; ++iq) {
        *rho += f[iq];
        u[0] += l->cx[iq] * f[iq];
        u[1] += l->cy[iq] * f[iq];
        if (l->dims == 3) u[2] += l->cz[iq] * f[iq];
    }
}

static void macro(const lattice* l, const zlp_level* c, double dt, const double* f, double* rho, double* u) {
    macro_sums(l, f, rho, u);
    if (c->has_force) {
        u[0] += 0.5 * c->force[0] * dt;
        u[1] += 0.5 * c->force[1] * dt;
        if (l->dims == 3) u[2] += 0.5 * c->force[2] * dt;
    }
    u[0] /= *rho;
    u[1] /= *rho;
    if (l->dims == 3) u[2] /= *rho;
}

static void diag_times(int q, const double* s, const double* mat, double* out) {
    /* out = S * mat with S diagonal, accumulated over k like the reference's triple loop */
    for (int j = 0; j < q; ++j)
        for (int i = 0; i < q; ++i) {
            double acc = 0.;
            for (int k = 0; k < q; ++k) acc = acc + (i == k ? s[i] : 0.) * mat[k * q + j];
            out[i * q + j] = acc;
        }
}

static void mrt_build(int dims, double relax, int d_matrix, double* out) {
    const int q = dims == 2 ? 9 : 19;
    double s[19], m[19 * 19], im[19 * 19], sm[19 * 19];
    for (int i = 0; i < q; ++i) {
        s[i] = dims == 2 ? kS9[i] : kS19[i];
        for (int j = 0; j < q; ++j) {
            m[i * q + j] = dims == 2 ? kM9[i][j] : kM19[i][j];
            im[i * q + j] = dims == 2 ? kIm9[i][j] : kIm19[i][j];
        }
    }
    const int ntau = dims == 2 ? 2 : 5;
    for (int t = 0; t < ntau; ++t) s[dims == 2 ? kTauRows9[t] : kTauRows19[t]] = relax;
    if (d_matrix)
        for (int i = 0; i < q; ++i) s[i] = 1. - 0.5 * s[i];
    diag_times(q, s, m, sm);
    for (int j = 0; j < q; ++j)
        for (int i = 0; i < q; ++i) {
            double acc = 0.;
            for (int k = 0; k < q; ++k) acc = acc + im[i * q + k] * sm[k * q + j];
            out[i * q + j] = acc;
        }
}

void zlp_mrt_matrix(int dims, double tau, double* out) { mrt_build(dims, 1. / tau, 0, out); }

/* Smagorinsky subgrid relaxation increment, reference arithmetic (les_models/lbm_les_smagorinsky.cpp) */
static double smag_tau_sgs(const lattice* l, const zlp_level* c, double dt, double tau0, const double* f,
                           const double* feq, const double* u) {
    double pxx = 0., pxy = 0., pyy = 0., pzz = 0., pxz = 0., pyz = 0.;
    for (int iq = 1; iq < l->q; ++iq) {
        const double d = f[iq] - feq[iq];
        pxx += l->cx[iq] * l->cx[iq] * d;
        pxy += l->cx[iq] * l->cy[iq] * d;
        pyy += l->cy[iq] * l->cy[iq] * d;
        if (l->dims == 3) {
            pzz += l->cz[iq] * l->cz[iq] * d;
            pxz += l->cx[iq] * l->cz[iq] * d;
            pyz += l->cy[iq] * l->cz[iq] * d;
        }
    }
    if (c->has_force) {
        const double* F = c->force;
        pxx += dt * F[0] * u[0];
        pyy += dt * F[1] * u[1];
        pxy += 0.5 * dt * (F[0] * u[0] + F[1] * u[1]);
        if (l->dims == 3) {
            pzz += dt * F[2] * u[2];
            pxz += 0.5 * dt * (F[0] * u[0] + F[2] * u[2]);
            pyz += 0.5 * dt * (F[1] * u[1] + F[2] * u[2]);
        }
    }
    const double pi2 = pxx * pxx + pyy * pyy + pzz * pzz + 2. * (pxy * pxy + pxz * pxz + pyz * pyz);
    const double cs = 18. * c->les_cs * c->les_cs;
    return 0.5 * (sqrt(tau0 * tau0 + cs * sqrt(2. * pi2)) - tau0);
}

double zlp_smag_tau_sgs(int dims, const double* f, const double* feq, double tau0, double dt, double cs,
                        int has_force, const double* force, const double* u) {
    const lattice l = lattice_of(dims);
    zlp_level c;
    memset(&c, 0, sizeof(c));
    c.dims = dims;
    c.les_cs = cs;
    c.has_force = has_force;
    for (int a = 0; a < 3; ++a) c.force[a] = force ? force[a] : 0.;
    return smag_tau_sgs(&l, &c, dt, tau0, f, feq, u);
}

static void forcing_term(const lattice* l, const double* u, const double* F, double* out) {
    for (int iq = 0; iq < l->q; ++iq) {
        if (l->dims == 2) {
            out[iq] = l->w[iq] * (3. * ((l->cx[iq] - u[0]) * F[0] + (l->cy[iq] - u[1]) * F[1])
                                  + 9. * (u[0] * l->cx[iq] + u[1] * l->cy[iq]) * (l->cx[iq] * F[0] + l->cy[iq] * F[1]));
        } else {
            out[iq] = l->w[iq] * (3. * ((l->cx[iq] - u[0]) * F[0] + (l->cy[iq] - u[1]) * F[1]
                                        + (l->cz[iq] - u[2]) * F[2])
                                  + 9. * (u[0] * l->cx[iq] + u[1] * l->cy[iq] + u[2] * l->cz[iq])
                                        * (l->cx[iq] * F[0] + l->cy[iq] * F[1] + l->cz[iq] * F[2]));
        }
    }
}

static void collide_node(const lattice* l, const zlp_level* c, double dt, double tau0, const double* mrt_s,
                         const double* mrt_d, const double* f, double* fc) {
    double rho, u[3], feq[19], fterm[19];
    macro(l, c, dt, f, &rho, u);
    zlp_feq(l->dims, rho, u, feq);
    if (c->has_force) forcing_term(l, u, c->force, fterm);
    double tau = tau0;
    double s_local[19 * 19], d_local[19 * 19];
    if (c->les == ZLP_LES_SMAGORINSKY) {
        tau = tau0 + smag_tau_sgs(l, c, dt, tau0, f, feq, u);
        if (c->collision == ZLP_MRT) {
            mrt_build(l->dims, 1. / tau, 0, s_local);
            mrt_s = s_local;
            if (c->has_force) {
                mrt_build(l->dims, 1. / tau, 1, d_local);
                mrt_d = d_local;
            }
        }
    }
    const int q = l->q;
    if (c->collision == ZLP_SRT) {
        for (int iq = 0; iq < q; ++iq) {
            if (c->has_force)
                fc[iq] = f[iq] - (f[iq] - feq[iq]) / tau + (1. - 0.5 / tau) * fterm[iq] * dt;
            else
                fc[iq] = f[iq] - (f[iq] - feq[iq]) / tau;
        }
    } else {
        for (int iq = 0; iq < q; ++iq) {
            double acc = 0.;
            for (int is = 0; is < q; ++is) {
                if (c->has_force)
                    acc += mrt_s[iq * q + is] * (f[is] - feq[is]) - mrt_d[iq * q + is] * fterm[is] * dt;
                else
                    acc += mrt_s[iq * q + is] * (f[is] - feq[is]);
            }
            fc[iq] = f[iq] - acc;
        }
    }
}

static long node_index(const zlp_level* c, int x, int y, int z) {
    return ((long)z * c->n[1] + y) * c->n[0] + x;
}

static int face_axis(int face) { return face >> 1; }
static int face_is_max(int face) { return face & 1; }

static void apply_face(const lattice* l, const zlp_level* c, double dt, int face, double* f, const double* fc) {
    const int kind = c->bc_kind[face];
    if (kind == ZLP_BC_NONE) return;
    const int axis = face_axis(face), is_max = face_is_max(face), q = l->q;
    const int* in_dirs = is_max ? (l->dims == 2 ? kNeg9[axis] : kNeg19[axis]) : (l->dims == 2 ? kPos9[axis] : kPos19[axis]);
    const int* inv_dirs = is_max ? (l->dims == 2 ? kPos9[axis] : kPos19[axis]) : (l->dims == 2 ? kNeg9[axis] : kNeg19[axis]);
    const int plane = is_max ? c->n[axis] - 1 : 0;
    const int other = is_max ? 0 : c->n[axis] - 1;
    const int inner = is_max ? plane - 1 : plane + 1;
    const double* uw = c->bc_vel[face];
    double feq_b[19];
    if (kind == ZLP_BC_NONEQ_EXTRAP) zlp_feq(l->dims, c->rho0, uw, feq_b);
    for (int z = 0; z < c->n[2]; ++z)
        for (int y = 0; y < c->n[1]; ++y)
            for (int x = 0; x < c->n[0]; ++x) {
                int p[3] = {x, y, z};
                if (p[axis] != plane) continue;
                double* fn = f + node_index(c, x, y, z) * q;
                if (kind == ZLP_BC_BOUNCE_BACK) {
                    const double* fcn = fc + node_index(c, x, y, z) * q;
                    for (int i = 0; i < l->nface_q; ++i) {
                        const int o = inv_dirs[i];
                        const double cu = l->dims == 2 ? l->cx[o] * uw[0] + l->cy[o] * uw[1]
                                                       : l->cx[o] * uw[0] + l->cy[o] * uw[1] + l->cz[o] * uw[2];
                        fn[in_dirs[i]] = fcn[o] - 6 * c->rho0 * l->w[o] * cu;
                    }
                } else if (kind == ZLP_BC_PERIODIC) {
                    int pc[3] = {x, y, z};
                    pc[axis] = other;
                    const double* fo = f + node_index(c, pc[0], pc[1], pc[2]) * q;
                    for (int i = 0; i < l->nface_q; ++i) fn[in_dirs[i]] = fo[in_dirs[i]];
                } else if (kind == ZLP_BC_NONEQ_EXTRAP) {
                    int pi[3] = {x, y, z};
                    pi[axis] = inner;
                    const double* fi = f + node_index(c, pi[0], pi[1], pi[2]) * q;
                    double rho_i, u_i[3], feq_i[19];
                    macro(l, c, dt, fi, &rho_i, u_i);
                    zlp_feq(l->dims, rho_i, u_i, feq_i);
                    for (int iq = 0; iq < q; ++iq) fn[iq] = feq_b[iq] + fi[iq] - feq_i[iq];
                } else if (kind == ZLP_BC_CONVECTIVE) {
                    /* convective outflow (not in the reference): the populations entering across
                       the face, f = (f_old + U f_inner) / (1 + U), U = |velocity . n| of the face */
                    int pi[3] = {x, y, z};
                    pi[axis] = inner;
                    const double* fi = f + node_index(c, pi[0], pi[1], pi[2]) * q;
                    const double u = fabs(uw[axis]);
                    for (int i = 0; i < l->nface_q; ++i) {
                        const int d = in_dirs[i];
                        fn[d] = (fn[d] + u * fi[d]) / (1. + u);
                    }
                }
            }
}

int zlp_run(const zlp_level* c, double* f, double* fc, int steps) {
    if (!c || !f || !fc || (c->dims != 2 && c->dims != 3)) return -1;
    const lattice l = lattice_of(c->dims);
    const int q = l.q;
    const double dt = 1. / (double)(1u << c->level);
    const double tau0 = zlp_tau(c->nu, c->level);
    double mrt_s[19 * 19], mrt_d[19 * 19];
    mrt_build(c->dims, 1. / tau0, 0, mrt_s);
    mrt_build(c->dims, 1. / tau0, 1, mrt_d);
    const int nz = c->dims == 3 ? c->n[2] : 1;
    const long nn = (long)c->n[0] * c->n[1] * nz;
    for (int step = 0; step < steps; ++step) {
        for (long i = 0; i < nn; ++i) {
            if (c->node_force) {
                zlp_level cn = *c;
                cn.has_force = 1;
                for (int a = 0; a < 3; ++a) cn.force[a] = (c->has_force ? c->force[a] : 0.) + c->node_force[i * 3 + a];
                collide_node(&l, &cn, dt, tau0, mrt_s, mrt_d, f + i * q, fc + i * q);
            } else {
                collide_node(&l, c, dt, tau0, mrt_s, mrt_d, f + i * q, fc + i * q);
            }
        }
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < c->n[1]; ++y)
                for (int x = 0; x < c->n[0]; ++x) {
                    double* fn = f + node_index(c, x, y, z) * q;
                    fn[0] = fc[node_index(c, x, y, z) * q];
                    for (int iq = 1; iq < q; ++iq) {
                        const int sx = x - (int)l.cx[iq], sy = y - (int)l.cy[iq], sz = z - (int)l.cz[iq];
                        if (sx < 0 || sy < 0 || sz < 0 || sx >= c->n[0] || sy >= c->n[1] || sz >= nz) continue;
                        fn[iq] = fc[node_index(c, sx, sy, sz) * q + iq];
                    }
                }
        for (int axis = 0; axis < c->dims; ++axis) apply_face(&l, c, dt, 2 * axis, f, fc);
        for (int axis = 0; axis < c->dims; ++axis) apply_face(&l, c, dt, 2 * axis + 1, f, fc);
    }
    return 0;
}

int zlp_macros(const zlp_level* c, const double* f, double* rho, double* u) {
    if (!c || !f || !rho || !u) return -1;
    const lattice l = lattice_of(c->dims);
    const double dt = 1. / (double)(1u << c->level);
    const int nz = c->dims == 3 ? c->n[2] : 1;
    const long nn = (long)c->n[0] * c->n[1] * nz;
    for (long i = 0; i < nn; ++i) {
        double uu[3];
        macro(&l, c, dt, f + i * l.q, rho + i, uu);
        for (int d = 0; d < c->dims; ++d) u[i * c->dims + d] = uu[d];
    }
    return 0;
}
