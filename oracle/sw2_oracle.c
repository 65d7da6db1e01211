/* sw2_oracle.c -- CPU restatement of AdH's SW2 Newton step.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the B200 library: tests, the smoke check and the
 * CPU-baseline leg of bench.py load it through ctypes.  It is never linked into,
 * called by or shipped with the product library.  It restates, in plain serial
 * C and in the reference's order of operations, the units of the reference path:
 *
 *   element residual        fe_sw2_body_resid        src/fe/sw2/fe_sw2_body_resid.c:45-1267
 *   temporal term           fe_sw2_temporal          src/fe/sw2/fe_sw2_body_resid.c:1288-1354
 *   wet/dry clipping        fe_sw2_wet_dry_wrapper   src/fe/fe_sw2_wet_dry_wrapper.c:106-306
 *                           fe_sw2_wet_dry_factor    src/fe/fe_sw2_wet_dry_wrapper.c:31-73
 *   wet/dry integrands      fe_sw2_wd_*              src/fe/sw2/fe_sw2_wet_dry_integrations.c:42-704
 *   boundary residual       fe_sw2_boundary_resid    src/fe/sw2/fe_sw2_boundary_resid.c:72-510
 *   residual assembly       fe_sw2_resid             src/fe/sw2/fe_sw2_resid.c:29-216
 *   FD Jacobian             fe_sw2_load              src/fe/sw2/fe_sw2_load.c:34-483
 *   Newton driver           fe_newton                src/fe/fe_newton.c:40-912
 *   scaling + Krylov        spv_jacobi, solv_bcgstab src/solver/spv_jacobi.c:222-317,
 *                                                    src/solver/solv_bcgstab.c:39-301
 *
 * Parity is pinned by running the reference executable built from its own sources
 * (oracle/ref/build_ref.py) on the same inputs; see tests/golden/.
 *
 * Supported scope: triangles; EVS/EEV eddy viscosity; log-law drag from Manning n;
 * Coriolis; temporal alpha; water source; NB VEL, NB OTW, NB OF and NB OVH edges;
 * PRS/VEL/VEL_PRS Dirichlet node strings; the grid mass diagnostics and the transport
 * side output elem_rhs_dacont_extra_terms.  Lid node strings are rejected at create
 * time; wind, waves, baroclinic terms, vorticity and quadrilaterals have no input
 * fields here (the generated workloads use none).
 *
 * The 2D transport of general constituents carried by the flow (fe_transport,
 * src/fe/transport/) is restated at the end of the file: fe_2d_transport_body_resid,
 * fe_2d_transport_boundary_resid, fe_transport_resid / _load / _init / _inc and the
 * transport branches of fe_newton.
 */
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include "../include/sw2gpu.h"

#define ORC_SMALL DBL_EPSILON            /* define.h:27 */
#define ORC_NQS   FLT_EPSILON            /* define.h:28 NOT_QUITE_SMALL */
#define ORC_UNSET_FLT (-9999999.9)
#define ORC_PI 3.141592653589793238462643383279502884197169399375105820974944592308
#define ORC_EARTH_ROTAT 7.2722E-5
#define ONE_3  0.333333333333333333333333
#define ONE_6  0.166666666666666666666667
#define ONE_12 0.083333333333333333333333
#define ONE_30 0.033333333333333333333333
#define ONE_60 0.016666666666666666666667
#define MAXD(a, b) ((a) > (b) ? (a) : (b))
#define MIND(a, b) ((a) < (b) ? (a) : (b))

enum { P_NONE = -1, P_U = 1, P_V = 2, P_H = 5 };

typedef struct { double c, x, y; } dof3;       /* c_eq, x_eq, y_eq */
typedef struct { double x, y; } v2;

typedef struct orc_ctx {
    int V, T, E, S, M, NS;
    double *x, *y, *z;
    int *node_string, *tri, *tri_mat, *edges, *edge_string, *edge_parent;
    int *str_bc, *str_isigma, *str_ivx, *str_ivy, *str_iu0;
    double *str_rough;
    int *mat_eev_mode;
    double *mat_ev, *mat_eev_coef, *mat_cor;
    sw2gpu_params p;
    /* geometry */
    double *djac, *grad;      /* grad[6*e]: (gx0, gy0, gx1, gy1, gx2, gy2) */
    double *edjac, *enrml;
    /* state: level 0 current, 1 old, 2 older */
    double *h[3], *u[3], *v[3];
    int *wd;
    double *dacont;            /* [3T] elem_rhs_dacont_extra_terms of the last body_resid call per element */
    double dt;
    double *series;
    double *wsx, *wsy;         /* [T] element wind stress (orc_set_wind), or NULL: no wind */
    double *wvx, *wvy;         /* [T] element wave radiation stress (orc_set_waves), or NULL: none */
    /* BCSR pattern (sorted columns, diagonal included) */
    int *rowptr, *col, nnzb;
    int *blk_of_pair;          /* [9*T] value block of (i, j) pair of each element */
    int *eblk_of_pair;         /* [4*E] */
    double *val, *resid, *sol;
    int *include;
    int bandwidth_nodes;
    int *perm, *iperm;         /* node order for the banded LU */
    int nblock;
    /* constituent transport (orc_trn_setup) */
    int ntrn;
    double *trn_refc;          /* [ntrn] property[0] */
    double *trn_dm;            /* [ntrn * M] MP DF d_m */
    int *trn_bc, *trn_ser;     /* [ntrn * S] trans[itrn].bc_flag, its series (iu_0 / isigma) */
    double *conc;              /* [ntrn][3][V] concentration levels */
    int *bcmask;               /* [V] mod->bc_mask of the last fe_transport_init */
    double *tval, *tres, *tsol;/* scalar Jacobian over the pattern [nnzb], residual, increment [V] */
} orc_ctx;

/* ------------------------------------------------------------------------------ */
/* closed-form P1 integrals (src/fe/fe_elem2d_integrations.c, fe_elem1d_integrations.c) */

static void tri_phi_f(double djac, double c, const double *f, double *I) {          /* :196 */
    double fs = f[0] + f[1] + f[2], t1 = djac * c * ONE_12;
    I[0] += t1 * (fs + f[0]); I[1] += t1 * (fs + f[1]); I[2] += t1 * (fs + f[2]);
}
static void tri_phi_f_lump(double djac, double c, const double *f, double *I) {     /* :250 */
    double t1 = djac * c * ONE_3;
    I[0] += t1 * f[0]; I[1] += t1 * f[1]; I[2] += t1 * f[2];
}
static void tri_phi(double djac, double c, double *I) {                            /* :159 */
    double t1 = c * djac * ONE_3;
    I[0] += t1; I[1] += t1; I[2] += t1;
}
static void tri_phi_f_g(double djac, double c, const double *f, const double *g, double *I) { /* :281 */
    double gs = 2 * (g[0] + g[1] + g[2]), t1 = c * djac * ONE_60;
    I[0] += t1 * (f[0] * (gs + 4 * g[0]) + f[1] * (gs - g[2]) + f[2] * (gs - g[1]));
    I[1] += t1 * (f[1] * (gs + 4 * g[1]) + f[2] * (gs - g[0]) + f[0] * (gs - g[2]));
    I[2] += t1 * (f[2] * (gs + 4 * g[2]) + f[1] * (gs - g[0]) + f[0] * (gs - g[1]));
}
static double tri_f_f(double djac, double c, const double *f) {
    return c * ONE_6 * djac * (f[0] * f[0] + f[0] * f[1] + f[1] * f[1] + f[0] * f[2] + f[1] * f[2] + f[2] * f[2]);
}
static void tri_gradphi_dot_vbar(const v2 *g, double djac, double c, v2 vb, double *I) { /* :422 */
    double t1 = c * djac;
    I[0] += t1 * (vb.x * g[0].x + vb.y * g[0].y);
    I[1] += t1 * (vb.x * g[1].x + vb.y * g[1].y);
    I[2] += t1 * (vb.x * g[2].x + vb.y * g[2].y);
}
static void tri_gradphi_dot_f_v(const v2 *g, double djac, double c, const double *f, const v2 *v, double *I) {
    double p1 = 2 * f[0] + f[1] + f[2], p2 = f[0] + 2 * f[1] + f[2], p3 = f[0] + f[1] + 2 * f[2];
    double tx = p1 * v[0].x + p2 * v[1].x + p3 * v[2].x;
    double ty = p1 * v[0].y + p2 * v[1].y + p3 * v[2].y;
    double con = djac * ONE_12 * c;
    I[0] += con * (g[0].x * tx + g[0].y * ty);
    I[1] += con * (g[1].x * tx + g[1].y * ty);
    I[2] += con * (g[2].x * tx + g[2].y * ty);
}
static void tri_dphi_f_g_h(const v2 *gr, double djac, double c, const double *f, const double *g,
                           const double *h, double *Ix, double *Iy) {             /* :832 */
    double ff1 = 3 * f[0] + f[1] + f[2], ff2 = 2 * f[0] + 2 * f[1] + f[2], ff3 = 2 * f[0] + f[1] + 2 * f[2];
    double ff4 = f[0] + 3 * f[1] + f[2], ff5 = f[0] + 2 * f[1] + 2 * f[2], ff6 = f[0] + f[1] + 3 * f[2];
    double gg1 = 2 * ff1 * g[0] + ff2 * g[1] + ff3 * g[2];
    double gg2 = ff2 * g[0] + 2 * ff4 * g[1] + ff5 * g[2];
    double gg3 = ff3 * g[0] + ff5 * g[1] + 2 * ff6 * g[2];
    double con = djac * ONE_60 * c * (gg1 * h[0] + gg2 * h[1] + gg3 * h[2]);
    int i;
    for (i = 0; i < 3; i++) { Ix[i] += con * gr[i].x; Iy[i] += con * gr[i].y; }
}
static void tri_dphi_f_f_h(const v2 *gr, double djac, double c, const double *f, const double *h,
                           double *Ix, double *Iy) {                               /* :864 */
    double f1 = f[0] * f[0], f2 = f[1] * f[1], f3 = f[2] * f[2];
    double p1 = 3 * f1 + 2 * f[0] * f[1] + f2 + (2 * f[0] + f[1]) * f[2] + f3;
    double p2 = f1 + 2 * f[0] * f[1] + 3 * f2 + (f[0] + 2 * f[1]) * f[2] + f3;
    double p3 = f1 + f[0] * f[1] + f2 + 2 * (f[0] + f[1]) * f[2] + 3 * f3;
    double con = djac * ONE_30 * c * (p1 * h[0] + p2 * h[1] + p3 * h[2]);
    int i;
    if (Ix) for (i = 0; i < 3; i++) Ix[i] += con * gr[i].x;
    if (Iy) for (i = 0; i < 3; i++) Iy[i] += con * gr[i].y;
}
static void tri_phi_h_df(double djac, double c, const double *h, v2 df, double *Ix, double *Iy) { /* :1016 */
    double sh = h[0] + h[1] + h[2], con;
    int i;
    con = djac * ONE_12 * c * df.x;
    for (i = 0; i < 3; i++) Ix[i] += con * (sh + h[i]);
    con = djac * ONE_12 * c * df.y;
    for (i = 0; i < 3; i++) Iy[i] += con * (sh + h[i]);
}
static void line_phi_h_h(double djac, double c, double h1, double h2, double *I) { /* elem1d:45 */
    double t1 = djac * ONE_12 * c;
    I[0] += t1 * (3 * h1 * h1 + 2 * h1 * h2 + h2 * h2);
    I[1] += t1 * (h1 * h1 + 2 * h1 * h2 + 3 * h2 * h2);
}
static void line_phi(double djac, double c, double *I) { double t1 = 0.5 * djac * c; I[0] += t1; I[1] += t1; }
static void line_phi_f(double djac, double c, const double *f, double *I) {
    double t1 = ONE_6 * djac * c;
    I[0] += t1 * (2 * f[0] + f[1]); I[1] += t1 * (f[0] + 2 * f[1]);
}
static void line_phi_h_v_dot_n(double djac, double c, const double *h, const v2 *v, v2 n, double *I) {
    double t1 = djac * ONE_12 * c;
    I[0] += t1 * (n.x * ((3 * h[0] + h[1]) * v[0].x + (h[0] + h[1]) * v[1].x) + n.y * ((3 * h[0] + h[1]) * v[0].y + (h[0] + h[1]) * v[1].y));
    I[1] += t1 * (n.x * ((h[0] + h[1]) * v[0].x + (h[0] + 3 * h[1]) * v[1].x) + n.y * ((h[0] + h[1]) * v[0].y + (h[0] + 3 * h[1]) * v[1].y));
}
static void line_phi_f_g_h(double djac, double c, double f1, double f2, double g1, double g2, double h1, double h2, double *I) {
    double t1 = ONE_60 * djac * c;
    I[0] += t1 * ((3 * (4 * f1 + f2) * g1 + (3 * f1 + 2 * f2) * g2) * h1 + ((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h2);
    I[1] += t1 * (((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h1 + ((2 * f1 + 3 * f2) * g1 + 3 * (f1 + 4 * f2) * g2) * h2);
}

/* ------------------------------------------------------------------------------ */
/* closures */

static double drag_coef(double depth, double ks) {       /* src/friction/fr_bedshstr_drag_coef.c:18-40 */
    double rh, bta, phi;
    depth = MAXD(depth, 1.E-8);
    ks = MAXD(ks, 1.E-8);
    if (ks > 29.7 * depth) rh = 1. / 29.7; else rh = depth / ks;
    bta = 29.7 * rh;
    phi = pow((.4 * bta) / ((bta + 1) * (log(bta + 1) - 1) + 1), 2.);
    return 2. * phi;
}
static double roughness(const orc_ctx *C, int str, double depth) {   /* fe_sw2_get_roughness.c:28-52 */
    double ks = C->str_rough[str];
    return ks > ORC_SMALL ? drag_coef(depth, ks) : 0.0;
}

/* ------------------------------------------------------------------------------ */
/* wet/dry wrapper (fe_sw2_wet_dry_wrapper.c:106-306) with the integrands as an enum */

enum { WD_AVG, WD_CONT_TEMPORAL, WD_CONVECTION, WD_GLS_CONVECTION, WD_PRESSURE, WD_BODYFORCE, WD_BPRESSURE,
       WD_TRN_TEMPORAL, WD_TRN_CONVECTION };

static void tri_gradphi_dot_f_g_v(const v2 *g, double djac, double c, const double *f, const double *gg,
                                  const v2 *v, double *I) {          /* fe_elem2d_integrations.c:571-587 */
    double b[3] = {0., 0., 0.};
    tri_phi_f_g(djac, c, f, gg, b);
    double ix = v[0].x * b[0] + v[1].x * b[1] + v[2].x * b[2];
    double iy = v[0].y * b[0] + v[1].y * b[1] + v[2].y * b[2];
    I[0] += ix * g[0].x + iy * g[0].y;
    I[1] += ix * g[1].x + iy * g[1].y;
    I[2] += ix * g[2].x + iy * g[2].y;
}

typedef struct {
    const v2 *x;          /* node coordinates */
    const double *h;      /* depth (clipping function) */
    const v2 *grad;       /* shape gradients (may be NULL) */
    const v2 *v;          /* unclipped vector (bodyForce: &grad_z) */
    const v2 *vwd;        /* clipped vector (may be NULL) */
    const double *fwd;    /* clipped scalar (may be NULL) */
    double djac;
    double a, b;          /* vars[0], vars[1] */
} wd_args;

static void wd_func(int kind, const v2 *x, const double *h, const v2 *g, const v2 *v, const v2 *vwd,
                    const double *fwd, double djac, double a, double b, dof3 *rhs) {
    int i;
    switch (kind) {
    case WD_AVG: {                            /* fe_sw2_wd_integrate_triangle_f :42 */
        double t1 = (h[0] + h[1] + h[2]) / 3.0, t2 = 0.0, t3 = 0.0;
        if (vwd) { t2 = (vwd[0].x + vwd[1].x + vwd[2].x) / 3.0; t3 = (vwd[0].y + vwd[1].y + vwd[2].y) / 3.0; }
        rhs[0].c += djac * t1; rhs[0].x += djac * t2; rhs[0].y += djac * t3;
        break; }
    case WD_CONT_TEMPORAL: {                  /* fe_sw2_wd_continuity_temporal_triangle */
        double rc[3] = {0, 0, 0};
        tri_phi_f(djac, b, h, rc);
        for (i = 0; i < 3; i++) rhs[i].c += rc[i];
        break; }
    case WD_CONVECTION: {                     /* fe_sw2_wd_convection_triangle */
        double c = b * a, rc[3] = {0, 0, 0}, rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0}, uu[3], vv[3];
        for (i = 0; i < 3; i++) { uu[i] = vwd[i].x; vv[i] = vwd[i].y; }
        tri_gradphi_dot_f_v(g, djac, c, h, vwd, rc);
        tri_dphi_f_g_h(g, djac, c, uu, vv, h, ry, rx);
        tri_dphi_f_f_h(g, djac, c, uu, h, rx, NULL);
        tri_dphi_f_f_h(g, djac, c, vv, h, NULL, ry);
        for (i = 0; i < 3; i++) { rhs[i].c += rc[i]; rhs[i].x += rx[i]; rhs[i].y += ry[i]; }
        break; }
    case WD_GLS_CONVECTION: {                 /* fe_sw2_wd_gls_convection_triangle */
        double ha = ONE_3 * (fwd[0] + fwd[1] + fwd[2]);
        double ua = ONE_3 * (vwd[0].x + vwd[1].x + vwd[2].x);
        double va = ONE_3 * (vwd[0].y + vwd[1].y + vwd[2].y);
        double dhdx = g[0].x * fwd[0] + g[1].x * fwd[1] + g[2].x * fwd[2];
        double dhdy = g[0].y * fwd[0] + g[1].y * fwd[1] + g[2].y * fwd[2];
        double dudx = g[0].x * vwd[0].x + g[1].x * vwd[1].x + g[2].x * vwd[2].x;
        double dudy = g[0].y * vwd[0].x + g[1].y * vwd[1].x + g[2].y * vwd[2].x;
        double dvdx = g[0].x * vwd[0].y + g[1].x * vwd[1].y + g[2].x * vwd[2].y;
        double dvdy = g[0].y * vwd[0].y + g[1].y * vwd[1].y + g[2].y * vwd[2].y;
        rhs[0].c += djac * a * b * (ua * dhdx + ha * dudx + va * dhdy + ha * dvdy);
        rhs[0].x += djac * a * b * (ua * dudx + va * dudy);
        rhs[0].y += djac * a * b * (ua * dvdx + va * dvdy);
        break; }
    case WD_PRESSURE: {                       /* fe_sw2_wd_pressure_triangle */
        double ff = tri_f_f(djac, b, h);
        for (i = 0; i < 3; i++) { rhs[i].x += g[i].x * ff; rhs[i].y += g[i].y * ff; }
        break; }
    case WD_BODYFORCE: {                      /* fe_sw2_wd_bodyForce_triangle */
        double rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
        tri_phi_h_df(djac, b, h, *v, rx, ry);
        for (i = 0; i < 3; i++) { rhs[i].x += rx[i]; rhs[i].y += ry[i]; }
        break; }
    case WD_TRN_TEMPORAL: {                   /* fe_2d_transport_wd_temporal_triangle
                                                 (fe_2d_transport_wet_dry_integrations.c:86-99) */
        double rc[3] = {0, 0, 0};
        tri_phi_f_g(djac, a * b, h, fwd, rc);
        for (i = 0; i < 3; i++) rhs[i].c += rc[i];
        break; }
    case WD_TRN_CONVECTION: {                 /* fe_2d_transport_wd_convection_triangle (:39-48) */
        double rc[3] = {0, 0, 0};
        tri_gradphi_dot_f_g_v(g, djac, a * b, h, fwd, vwd, rc);
        for (i = 0; i < 3; i++) rhs[i].c += rc[i];
        break; }
    case WD_BPRESSURE: {                      /* fe_sw2_wd_boundaryPressure_triangle */
        int e;
        for (e = 0; e < 3; e++) {
            int n1 = e, n2 = (e + 1) % 3;
            double delx = x[n1].x - x[n2].x, dely = x[n2].y - x[n1].y, r[2] = {0, 0};
            line_phi_h_h(1., b, h[n1], h[n2], r);
            rhs[n1].x += dely * r[0]; rhs[n2].x += dely * r[1];
            rhs[n1].y += delx * r[0]; rhs[n2].y += delx * r[1];
        }
        break; }
    }
}

static double wd_wrapper(int kind, dof3 *rhs, const wd_args *A, int redistribute) {
    int i, dry, total = 0, pass = 0, only;
    for (i = 0; i < 3; i++) { dry = (A->h[i] <= 0.0) ? 1 : 0; total += dry; pass += dry << i; }
    if (total == 3) return 0;
    if (total == 0) {
        wd_func(kind, A->x, A->h, A->grad, A->v, A->vwd, A->fwd, A->djac, A->a, A->b, rhs);
        return 1.0;
    }
    if (total == 1) wd_func(kind, A->x, A->h, A->grad, A->v, A->vwd, A->fwd, A->djac, A->a, A->b, rhs);
    else pass = 7 - pass;
    only = pass / 2;
    double nh[3] = {0, 0, 0}, nf[3] = {0, 0, 0};
    v2 nx[3], nv[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (i = 0; i < 3; i++) {
        if (i != only) {
            double xsi = A->h[i] / (A->h[i] - A->h[only]);
            nx[i].x = A->x[i].x + xsi * (A->x[only].x - A->x[i].x);
            nx[i].y = A->x[i].y + xsi * (A->x[only].y - A->x[i].y);
            if (A->vwd) {
                nv[i].x = A->vwd[i].x + xsi * (A->vwd[only].x - A->vwd[i].x);
                nv[i].y = A->vwd[i].y + xsi * (A->vwd[only].y - A->vwd[i].y);
            }
            if (A->fwd) nf[i] = A->fwd[i] + xsi * (A->fwd[only] - A->fwd[i]);
        } else {
            nx[i] = A->x[i];
            nh[i] = A->h[i];
            if (A->fwd) nf[i] = A->fwd[i];
            if (A->vwd) nv[i] = A->vwd[i];
        }
    }
    double edjac = A->djac;
    double djac = ((nx[1].x - nx[0].x) * (nx[2].y - nx[0].y) - (nx[1].y - nx[0].y) * (nx[2].x - nx[0].x)) / 2.0;
    if (djac / edjac < ORC_SMALL) return (double) (total % 2);
    v2 ng[3];
    const v2 *gp = NULL;
    if (A->grad) {                            /* GRAD_SHAPE, macro.h:793 */
        ng[0].x = 0.5 * (nx[1].y - nx[2].y) / djac; ng[1].x = 0.5 * (nx[2].y - nx[0].y) / djac;
        ng[2].x = 0.5 * (nx[0].y - nx[1].y) / djac; ng[0].y = 0.5 * (nx[2].x - nx[1].x) / djac;
        ng[1].y = 0.5 * (nx[0].x - nx[2].x) / djac; ng[2].y = 0.5 * (nx[1].x - nx[0].x) / djac;
        gp = ng;
    }
    dof3 nr[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    wd_func(kind, nx, nh, gp, A->v, A->vwd ? nv : NULL, A->fwd ? nf : NULL, djac, A->a, A->b, nr);
    double factor = (total >> 1) - (total % 2);
    if (redistribute) {                       /* RE_DISTRIBUTE, macro.h:803 */
        for (i = 0; i < 3; i++) {
            if (i == only) continue;
            double ax = nx[i].x - A->x[only].x, ay = nx[i].y - A->x[only].y;
            double bx = A->x[i].x - A->x[only].x, by = A->x[i].y - A->x[only].y;
            double xsi = sqrt((ax * ax + ay * ay) / (bx * bx + by * by));
            nr[only].c += (1.0 - xsi) * nr[i].c; nr[only].x += (1.0 - xsi) * nr[i].x; nr[only].y += (1.0 - xsi) * nr[i].y;
            nr[i].c *= xsi; nr[i].x *= xsi; nr[i].y *= xsi;
        }
    }
    for (i = 0; i < 3; i++) { rhs[i].c += factor * nr[i].c; rhs[i].x += factor * nr[i].x; rhs[i].y += factor * nr[i].y; }
    factor *= djac / edjac;
    return factor + ((factor < 0) ? 1.0 : 0.0);
}

static double wd_factor(const v2 *x, const double *h, double djac) {   /* fe_sw2_wet_dry_factor :31-73 */
    dof3 dummy[3];
    wd_args A = {x, h, NULL, NULL, NULL, NULL, djac, 0, 0};
    int i, total = 0;
    for (i = 0; i < 3; i++) total += (h[i] <= 0.0);
    if (total == 3) return 0.0;
    if (total == 0) return 1.0;
    /* same clipping as the wrapper; the integrand result is discarded */
    memset(dummy, 0, sizeof dummy);
    return wd_wrapper(WD_AVG, dummy, &A, 0);
}

static void wd_average(const v2 *x, const double *h, const v2 *vel, double djac, double *havg, v2 *vavg) {
    dof3 av[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};             /* fe_sw2_wd_average :19-39 */
    wd_args A = {x, h, NULL, NULL, vel, h, djac, 1., 1.};
    double f = wd_wrapper(WD_AVG, av, &A, 0);
    *havg = 0.; vavg->x = 0.; vavg->y = 0.;
    if (f > 0.0) {
        double wet = djac * f;
        *havg = av[0].c / wet; vavg->x = av[0].x / wet; vavg->y = av[0].y / wet;
    }
}

/* fe_sw2_get_EEVF (src/fe/sw2/fe_sw2_get_EEVF.c:33-60): estimated eddy viscosity of mode 1..3 */
static void eevf(int mode, double coef, double gr, double dll, double h_fric, double rough, double area, v2 gu,
                 v2 gv, double vmag, int wd, double *ev_st, double *ev_tr) {
    double vmin = 0.1 * sqrt(gr * dll), evmin = 0., st, tr;
    if (mode == 1) {
        st = 0.0; tr = coef * 2.0 * h_fric * sqrt(rough) * vmag;
        evmin = (coef / 0.5) * vmin * sqrt(area) / 40.; tr = MAXD(tr, evmin);
    } else if (mode == 2) {
        st = 1.3 * h_fric * sqrt(rough) * vmag;
        tr = coef * 0.92 * h_fric * sqrt(rough) * vmag;
        evmin = (coef / 0.5) * vmin * sqrt(area) / 40.; tr = MAXD(tr, evmin);
    } else {
        st = 0.;
        tr = coef * coef * area * sqrt(gu.x * gu.x + gv.y * gv.y + 0.5 * (gu.y + gv.x) * (gu.y + gv.x));
        evmin = (coef / 0.2) * vmin * sqrt(area) / 40.; tr = MAXD(tr, evmin);
    }
    if (wd == 1 || wd == 2) { st = 0.0; tr = MAXD(tr, 5. * evmin); }
    *ev_st = st; *ev_tr = tr;
}

/* ------------------------------------------------------------------------------ */
/* fe_sw2_body_resid (triangles) */

typedef struct {                 /* per-call element inputs (perturbation applied) */
    v2 X[3]; double Z[3];
    double h[3]; v2 vel[3];
    double ho[3]; v2 velo[3];
    double hoo[3]; v2 veloo[3];
} elem_in;

static void gather_elem(const orc_ctx *C, int ie, elem_in *E) {
    int i;
    for (i = 0; i < 3; i++) {
        int n = C->tri[3 * ie + i];
        E->X[i].x = C->x[n]; E->X[i].y = C->y[n]; E->Z[i] = C->z[n];
        E->h[i] = C->h[0][n]; E->vel[i].x = C->u[0][n]; E->vel[i].y = C->v[0][n];
        E->ho[i] = C->h[1][n]; E->velo[i].x = C->u[1][n]; E->velo[i].y = C->v[1][n];
        E->hoo[i] = C->h[2][n]; E->veloo[i].x = C->u[2][n]; E->veloo[i].y = C->v[2][n];
    }
}

static void temporal(const v2 *X, double djac, double dll, const double *h, const v2 *vel, double wdf,
                     double dtf, dof3 *er, int wd_flag) {         /* fe_sw2_temporal :1288-1354 */
    double con = dtf * wdf, uh[3], vh[3], rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
    dof3 rhs[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    int i;
    for (i = 0; i < 3; i++) { uh[i] = vel[i].x * MAXD(h[i], dll); vh[i] = vel[i].y * MAXD(h[i], dll); }
    wd_args A = {X, h, NULL, NULL, NULL, NULL, djac, 1.0, dtf};
    wd_wrapper(WD_CONT_TEMPORAL, rhs, &A, 1);
    tri_phi_f_lump(djac, con, uh, rx);
    tri_phi_f_lump(djac, con, vh, ry);
    for (i = 0; i < 3; i++) {
        if (wd_flag != 2) er[i].c += rhs[i].c;
        er[i].x += rx[i]; er[i].y += ry[i];
    }
}

/* total_stress of an element (fe_sw2_body_resid.c:674-694): wind plus wave stress, each 0 when
 * it is off (both start as 0 and are summed in that order) */
static double surface_stress(const orc_ctx *C, int ie, int y) {
    const double w = C->wsx ? (y ? C->wsy[ie] : C->wsx[ie]) : 0.0;
    const double r = C->wvx ? (y ? C->wvy[ie] : C->wvx[ie]) : 0.0;
    return w + r;
}

static void body_resid(const orc_ctx *C, int ie, const elem_in *E, int pvar, dof3 *er) {
    const sw2gpu_params *P = &C->p;
    const v2 *g = (const v2 *) (C->grad + 6 * ie);
    double djac = C->djac[ie], dt = C->dt, gr = P->gravity, dll = P->drying_lower_limit, dul = P->drying_upper_limit;
    double alpha = P->tau_temporal;
    int imat = C->tri_mat[ie], str = imat, wd = C->wd[ie], i;
    int pressure = (pvar == P_U || pvar == P_V) ? 0 : 1;
    const double *h = E->h, *ho = E->ho;
    const v2 *X = E->X, *vel = E->vel;
    double u[3], v[3], uo[3], vo[3], zero3[3] = {0, 0, 0};
    for (i = 0; i < 3; i++) { u[i] = vel[i].x; v[i] = vel[i].y; uo[i] = E->velo[i].x; vo[i] = E->velo[i].y; }

    double h_avg = (h[0] + h[1] + h[2]) / 3.0;
    double u_avg = (u[0] + u[1] + u[2]) / 3.0, v_avg = (v[0] + v[1] + v[2]) / 3.0;
    v2 gz = {0, 0}, gh = {0, 0}, gu = {0, 0}, gv = {0, 0}, gw;
    for (i = 0; i < 3; i++) {
        gz.x += E->Z[i] * g[i].x; gz.y += E->Z[i] * g[i].y;
        gh.x += h[i] * g[i].x;    gh.y += h[i] * g[i].y;
    }
    for (i = 0; i < 3; i++) {
        gu.x += vel[i].x * g[i].x; gu.y += vel[i].x * g[i].y;
        gv.x += vel[i].y * g[i].x; gv.y += vel[i].y * g[i].y;
    }
    gw.x = gz.x + gh.x; gw.y = gz.y + gh.y;
    double vmag = sqrt(u_avg * u_avg + v_avg * v_avg);
    double vst_i = u_avg / MAXD(vmag, 1.E-8), vst_j = v_avg / MAXD(vmag, 1.E-8);

    double h_wd, h_wd_old;
    v2 vwd, vwd_old;
    wd_average(X, h, vel, djac, &h_wd, &vwd);
    wd_average(X, ho, E->velo, djac, &h_wd_old, &vwd_old);
    double factor = wd_factor(X, h, djac), factor_old = wd_factor(X, ho, djac);
    double factor_older = wd_factor(X, E->hoo, djac);
    double vwd_mag = sqrt(vwd.x * vwd.x + vwd.y * vwd.y);
    double h_fric = MAXD(h_wd, ORC_SMALL);
    double rough = roughness(C, str, h_fric);

    double ev_st = 0., ev_tr = 0.;
    if (C->mat_eev_mode[imat] == 0) {                           /* EVSF :263-276 */
        double xx = C->mat_ev[3 * imat] + P->viscosity, yy = C->mat_ev[3 * imat + 1] + P->viscosity;
        ev_st = fabs(xx - yy);
        ev_tr = MIND(xx, yy);
    } else {
        eevf(C->mat_eev_mode[imat], C->mat_eev_coef[imat], gr, dll, h_fric, rough, djac, gu, gv, vmag, wd,
             &ev_st, &ev_tr);
    }

    for (i = 0; i < 3; i++) { er[i].c = 0; er[i].x = 0; er[i].y = 0; }
    dof3 rhs[3];
    /* the continuity parts of shock capturing and SUPG are kept for transport, as the reference's
     * side output elem_rhs_dacont_extra_terms (:353-355, :400, :1214), by every call */
    double *dac = C->dacont + 3 * ie;
    for (i = 0; i < 3; i++) dac[i] = 0.;

    /* shock capturing :357-400 */
    if (wd == 1 || wd == 2) {
        double gwm = sqrt(gw.x * gw.x + gw.y * gw.y + ORC_SMALL);
        double gum = sqrt(gu.x * gu.x + gu.y * gu.y + ORC_SMALL);
        double gvm = sqrt(gv.x * gv.x + gv.y * gv.y + ORC_SMALL);
        double cu = 0.5 * dul * djac * gum, cv = 0.5 * dul * djac * gvm;
        (void) gwm;
        v2 un = {gu.x / gum, gu.y / gum}, vn = {gv.x / gvm, gv.y / gvm};
        for (i = 0; i < 3; i++) {
            double nx = un.x * gu.x + un.y * gu.y, ny = vn.x * gv.x + vn.y * gv.y;
            rhs[i].c = dt * 0.5 * gr * djac * ((dll * gw.x) * g[i].x + (dll * gw.y) * g[i].y);
            rhs[i].x = cu * dt * djac * nx * (un.x * g[i].x + un.y * g[i].y);
            rhs[i].y = cv * dt * djac * ny * (vn.x * g[i].x + vn.y * g[i].y);
        }
        for (i = 0; i < 3; i++) {
            dac[i] += rhs[i].c;
            er[i].c += rhs[i].c; er[i].x += rhs[i].x; er[i].y += rhs[i].y;
        }
    }

    /* advection :434-457 */
    memset(rhs, 0, sizeof rhs);
    {
        wd_args A = {X, h, g, vel, vel, NULL, djac, dt, -1};
        wd_wrapper(WD_CONVECTION, rhs, &A, 1);
    }
    for (i = 0; i < 3; i++) { er[i].c += rhs[i].c; er[i].x += rhs[i].x; er[i].y += rhs[i].y; }

    /* temporal :481-490 */
    temporal(X, djac, dll, h, vel, factor, 1. + alpha / 2., er, -3);
    temporal(X, djac, dll, ho, E->velo, factor_old, (-1.) * (1. + alpha), er, wd);
    temporal(X, djac, dll, E->hoo, E->veloo, factor_older, alpha / 2., er, wd);

    /* diffusion :504-534 */
    {
        double tmp = h_wd < dul ? dul : h_wd, rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
        v2 fx, fy;
        fx.x = 2. * ev_st * vst_i * (vst_i * gu.x + vst_j * gu.y) + 2. * ev_tr * gu.x;
        fx.y = ev_st * vst_j * (vst_j * gu.y + vst_i * gu.x + vst_i * gv.x + vst_j * gv.y) + ev_tr * (gu.y + gv.x);
        fy.x = ev_st * vst_i * (vst_j * gu.y + vst_i * gu.x + vst_i * gv.x + vst_j * gv.y) + ev_tr * (gu.y + gv.x);
        fy.y = 2. * ev_st * vst_j * (vst_j * gv.y + vst_i * gv.x) + 2. * ev_tr * gv.y;
        tri_gradphi_dot_vbar(g, djac, tmp, fx, rx);
        tri_gradphi_dot_vbar(g, djac, tmp, fy, ry);
        double t1 = dt * factor;
        for (i = 0; i < 3; i++) { er[i].x += t1 * rx[i]; er[i].y += t1 * ry[i]; }
    }

    /* friction :557-577 */
    double resistance = rough / (2.0 * gr);
    {
        double fx[3], fy[3], rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
        for (i = 0; i < 3; i++) {
            double m = sqrt(vel[i].x * vel[i].x + vel[i].y * vel[i].y);
            fx[i] = vel[i].x * m; fy[i] = vel[i].y * m;
        }
        double t1 = dt * gr * resistance * factor;
        tri_phi_f(djac, t1, fx, rx);
        tri_phi_f(djac, t1, fy, ry);
        for (i = 0; i < 3; i++) { er[i].x += rx[i]; er[i].y += ry[i]; }
    }
    v2 bed = {resistance * vwd.x * vwd_mag, resistance * vwd.y * vwd_mag};

    /* Coriolis :639-652 */
    double cspeed = sin((ORC_PI / 180.) * C->mat_cor[imat]) * 2. * ORC_EARTH_ROTAT;
    {
        double rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0}, t1 = dt * factor * cspeed;
        tri_phi_f_g(djac, -t1, h, v, rx);
        tri_phi_f_g(djac, +t1, h, u, ry);
        for (i = 0; i < 3; i++) { er[i].x += rx[i]; er[i].y += ry[i]; }
    }

    /* wind surface stress, fully wet elements only :674-719 (no wave stress: 0) */
    if (wd == 0 && (C->wsx || C->wvx)) {
        double rx[3] = {0, 0, 0}, ry[3] = {0, 0, 0};
        tri_phi(djac, surface_stress(C, ie, 0), rx);
        tri_phi(djac, surface_stress(C, ie, 1), ry);
        for (i = 0; i < 3; i++) { er[i].x -= dt * rx[i]; er[i].y -= dt * ry[i]; }
    }

    /* rainfall :728-754 */
    double water_source = 0.;
    if (C->str_bc[str] == SW2GPU_BCT_WATER_SOURCE) {
        double rc[3] = {0, 0, 0};
        water_source = C->series[C->str_isigma[str]];
        tri_phi(djac, water_source, rc);
        for (i = 0; i < 3; i++) er[i].c -= dt * factor * rc[i];
    }

    /* pressure, bed slope, boundary pressure :761-862 */
    if (pressure) {
        memset(rhs, 0, sizeof rhs);
        { wd_args A = {X, h, g, NULL, NULL, NULL, djac, 1, -0.5 * gr * dt}; wd_wrapper(WD_PRESSURE, rhs, &A, 1); }
        for (i = 0; i < 3; i++) { er[i].c += rhs[i].c; er[i].x += rhs[i].x; er[i].y += rhs[i].y; }
        memset(rhs, 0, sizeof rhs);
        { wd_args A = {X, h, NULL, &gz, NULL, NULL, djac, 1, gr * dt}; wd_wrapper(WD_BODYFORCE, rhs, &A, 1); }
        for (i = 0; i < 3; i++) { er[i].c += rhs[i].c; er[i].x += rhs[i].x; er[i].y += rhs[i].y; }
        memset(rhs, 0, sizeof rhs);
        { wd_args A = {X, h, NULL, NULL, NULL, NULL, djac, 1, 0.5 * dt * gr}; wd_wrapper(WD_BPRESSURE, rhs, &A, 1); }
        for (i = 0; i < 3; i++) { er[i].c += rhs[i].c; er[i].x += rhs[i].x; er[i].y += rhs[i].y; }
    }

    /* SUPG :987-1232 */
    if (!(fabs(h_wd) < ORC_SMALL)) {
        double gf = gr;                                  /* (1 + density_avg) * g, density 0 */
        double hden = MAXD(h_wd, ORC_NQS);
        double le = sqrt(djac * factor_old);            /* get_element_length method 2 */
        double c2 = gf * hden;
        if (hden <= 0.0) c2 = 0.;
        double sr = sqrt(pow(vwd.x, 2) + pow(vwd.y, 2) + c2 + ORC_SMALL);
        double tau = P->tau_pg * le / sr;
        dof3 dfdt[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, adv[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        double dhdt, dudt, dvdt;
        { wd_args A = {X, ho, NULL, NULL, E->velo, ho, djac, 1, 1}; wd_wrapper(WD_AVG, dfdt, &A, 0); }
        dudt = -dfdt[0].x; dvdt = -dfdt[0].y; dhdt = -dfdt[0].c;
        memset(dfdt, 0, sizeof dfdt);
        { wd_args A = {X, h, NULL, NULL, vel, h, djac, 1, 1}; factor = wd_wrapper(WD_AVG, dfdt, &A, 0); }
        dudt += dfdt[0].x; dvdt += dfdt[0].y; dhdt += dfdt[0].c;
        { wd_args A = {X, h, g, NULL, vel, h, djac, dt, 1}; factor = wd_wrapper(WD_GLS_CONVECTION, adv, &A, 0); }
        double xp = gf * (gh.x + gz.x) * dt * factor + 0.0 * dt * factor;
        double yp = gf * (gh.y + gz.y) * dt * factor + 0.0 * dt * factor;
        double xf = gr * bed.x * dt * factor, yf = gr * bed.y * dt * factor;
        double xc = -vwd.y * cspeed, yc = vwd.x * cspeed;
        double c_eq = dhdt + adv[0].c + factor * water_source * djac * dt;
        /* the surface stress enters the strong momentum equations too (:1049-1050); it is zero
         * off fully wet elements (:674-675) */
        double tsx = wd == 0 ? surface_stress(C, ie, 0) : 0.0, tsy = wd == 0 ? surface_stress(C, ie, 1) : 0.0;
        double x_eq = dudt + adv[0].x + (xp + xf / hden) * djac + (xc - tsx / hden) * djac * factor * dt;
        double y_eq = dvdt + adv[0].y + (yp + yf / hden) * djac + (yc - tsy / hden) * djac * factor * dt;
        for (i = 0; i < 3; i++) {
            double rc = g[i].x * (tau * vwd.x * c_eq + tau * h_wd * x_eq) + g[i].y * (tau * vwd.y * c_eq + tau * h_wd * y_eq);
            double rx = g[i].x * (tau * gf * h_wd * c_eq + tau * vwd.x * h_wd * x_eq) + g[i].y * (tau * vwd.y * h_wd * x_eq);
            double ry = g[i].y * (tau * gf * h_wd * c_eq + tau * vwd.y * h_wd * y_eq) + g[i].x * (tau * vwd.x * h_wd * y_eq);
            dac[i] += rc;
            er[i].c += rc; er[i].x += rx; er[i].y += ry;
        }
    }
    (void) zero3; (void) uo; (void) vo; (void) h_wd_old; (void) vwd_old; (void) h_avg;

    /* Dirichlet :1239-1256 */
    for (i = 0; i < 3; i++) {
        int s = C->node_string[C->tri[3 * ie + i]];
        if (s > SW2GPU_NORMAL) {
            int f = C->str_bc[s];
            if (f == SW2GPU_BCT_PRS_DIR) er[i].c = 0.0;
            else if (f == SW2GPU_BCT_VEL_DIR) { er[i].x = 0.0; er[i].y = 0.0; }
            else if (f == SW2GPU_BCT_VEL_PRS_DIR) { er[i].c = 0.0; er[i].x = 0.0; er[i].y = 0.0; }
        }
    }
}

/* ------------------------------------------------------------------------------ */
/* fe_sw2_boundary_resid (edges) */

/* fe_sw2_1d_implicit_flow (:637-): flow through the edge with the current velocity (outflow
 * components only in the momentum fluxes) */
static void implicit_flow(double djac, double dt, v2 n, const double *hh, const v2 *vel, dof3 *er) {
    int i;
    double u[2] = {vel[0].x, vel[1].x}, v[2] = {vel[0].y, vel[1].y};
    double ur[2] = {u[0], u[1]}, vr[2] = {v[0], v[1]}, rc[2] = {0, 0}, rx[2] = {0, 0}, ry[2] = {0, 0};
    for (i = 0; i < 2; i++) if (vel[i].x * n.x + vel[i].y * n.y < ORC_SMALL) { ur[i] = 0.; vr[i] = 0.; }
    line_phi_h_v_dot_n(djac, 1., hh, vel, n, rc);
    line_phi_f_g_h(djac, n.x, ur[0], ur[1], u[0], u[1], hh[0], hh[1], rx);
    line_phi_f_g_h(djac, n.y, vr[0], vr[1], v[0], v[1], hh[0], hh[1], ry);
    line_phi_f_g_h(djac, n.y, ur[0], ur[1], v[0], v[1], hh[0], hh[1], rx);
    line_phi_f_g_h(djac, n.x, vr[0], vr[1], u[0], u[1], hh[0], hh[1], ry);
    for (i = 0; i < 2; i++) { er[i].c += dt * rc[i]; er[i].x += dt * rx[i]; er[i].y += dt * ry[i]; }
}
/* fe_sw2_1d_pressure twice (:773-): the outside water column dep minus the inside one hh */
static void boundary_pressure(double djac, double dt, double gr, v2 n, const double *dep, const double *hh, dof3 *er) {
    int i;
    double r[2] = {0, 0}, t1 = dt * 0.5 * gr;
    line_phi_h_h(djac, 1., dep[0], dep[1], r);
    for (i = 0; i < 2; i++) { er[i].x += t1 * n.x * r[i]; er[i].y += t1 * n.y * r[i]; }
    r[0] = r[1] = 0;
    t1 = dt * 0.5 * (-gr);
    line_phi_h_h(djac, 1., hh[0], hh[1], r);
    for (i = 0; i < 2; i++) { er[i].x += t1 * n.x * r[i]; er[i].y += t1 * n.y * r[i]; }
}

static void boundary_resid(const orc_ctx *C, int ie, const double *hh, const v2 *vel, int pvar, dof3 *er) {
    const sw2gpu_params *P = &C->p;
    int s = C->edge_string[ie], flag = C->str_bc[s], i;
    int pressure = (pvar == P_U || pvar == P_V) ? 0 : 1;
    v2 n = {C->enrml[2 * ie], C->enrml[2 * ie + 1]};
    double djac = C->edjac[ie], dt = C->dt, gr = P->gravity;
    double u[2] = {vel[0].x, vel[1].x}, v[2] = {vel[0].y, vel[1].y};
    double h_avg = 0.5 * (hh[0] + hh[1]);
    if (h_avg < ORC_SMALL) h_avg = ORC_SMALL;
    double z0 = C->z[C->edges[2 * ie]];
    for (i = 0; i < 2; i++) { er[i].c = 0; er[i].x = 0; er[i].y = 0; }
    if (flag == SW2GPU_BCT_VEL_NEU) {                         /* explicit flow :562-604 */
        double flux = -1.0 * C->series[C->str_isigma[s]];
        double rc[2] = {0, 0}, rx[2] = {0, 0}, ry[2] = {0, 0};
        line_phi(djac, 1., rc);
        if (flux < 0) {
            double us = 0., vs = 0.;
            if (h_avg > 0) { us = flux * n.x / h_avg; vs = flux * n.y / h_avg; }
            line_phi(djac, us, rx);
            line_phi(djac, vs, ry);
        } else {
            line_phi_f(djac, 1., u, rx);
            line_phi_f(djac, 1., v, ry);
        }
        double t1 = dt * flux;
        for (i = 0; i < 2; i++) { er[i].c += t1 * rc[i]; er[i].x += t1 * rx[i]; er[i].y += t1 * ry[i]; }
    } else if (flag == SW2GPU_BCT_OUTFLOW || flag == SW2GPU_BCT_PRS_NEU) {
        double dep[2] = {0.0, 0.0};
        if (flag == SW2GPU_BCT_PRS_NEU) {
            double tail = C->series[C->str_isigma[s]];
            dep[0] = tail - z0;
            dep[1] = tail - z0;                                /* both from node 0 (:375-376) */
            if (dep[0] < ORC_SMALL || dep[1] < ORC_SMALL || hh[0] < ORC_SMALL || hh[1] < ORC_SMALL) return;
        }
        implicit_flow(djac, dt, n, hh, vel, er);
        if (flag == SW2GPU_BCT_PRS_NEU && pressure) boundary_pressure(djac, dt, gr, n, dep, hh, er);
    } else if (flag == SW2GPU_BCT_OVH_NEU) {                    /* elevation + velocities :398-440 */
        const int na = C->edges[2 * ie], nb = C->edges[2 * ie + 1];
        const double tail = C->series[C->str_isigma[s]];
        double dep[2] = {tail - C->z[na], tail - C->z[nb]};   /* each node's own bed here */
        if (dep[0] < ORC_SMALL || dep[1] < ORC_SMALL)           /* the reference stops the run (tl_error) */
            fprintf(stderr, "oracle: NB OVH tailwater elevation below the bed on edge %d\n", ie);
        v2 uv = {C->series[C->str_ivx[s]], C->series[C->str_ivy[s]]};
        if (uv.x * n.x + uv.y * n.y < -ORC_SMALL) {             /* inflow: fe_sw2_1d_hvel :882-897 */
            double rc[2] = {0, 0};
            line_phi_h_v_dot_n(djac, 1., hh, vel, n, rc);
            for (i = 0; i < 2; i++) {
                er[i].c += dt * rc[i];
                er[i].x += dt * rc[i] * uv.x;
                er[i].y += dt * rc[i] * uv.y;
            }
        } else {
            implicit_flow(djac, dt, n, hh, vel, er);
        }
        if (pressure) boundary_pressure(djac, dt, gr, n, dep, hh, er);
    }
    for (i = 0; i < 2; i++) {                                  /* Dirichlet :483-498 */
        int ns = C->node_string[C->edges[2 * ie + i]];
        if (ns > SW2GPU_NORMAL) {
            int f = C->str_bc[ns];
            if (f == SW2GPU_BCT_PRS_DIR) er[i].c = 0.0;
            else if (f == SW2GPU_BCT_VEL_DIR) { er[i].x = 0.0; er[i].y = 0.0; }
            else if (f == SW2GPU_BCT_VEL_PRS_DIR) { er[i].c = 0.0; er[i].x = 0.0; er[i].y = 0.0; }
        }
    }
}

/* ------------------------------------------------------------------------------ */
/* context */

static void *dup(const void *p, size_t n) { void *q = malloc(n ? n : 1); if (p && n) memcpy(q, p, n); else memset(q, 0, n ? n : 1); return q; }
static int cmp_int(const void *a, const void *b) { return (*(const int *) a > *(const int *) b) - (*(const int *) a < *(const int *) b); }

static int find_blk(const orc_ctx *C, int i, int j) {
    int lo = C->rowptr[i], hi = C->rowptr[i + 1] - 1;
    while (lo <= hi) { int m = (lo + hi) / 2; if (C->col[m] == j) return m; if (C->col[m] < j) lo = m + 1; else hi = m - 1; }
    return -1;
}

static int build_pattern(orc_ctx *C) {
    int V = C->V, i, k;
    int *deg = (int *) calloc(V, sizeof(int));
    for (i = 0; i < C->T; i++) for (k = 0; k < 3; k++) deg[C->tri[3 * i + k]] += 3;
    for (i = 0; i < C->E; i++) for (k = 0; k < 2; k++) deg[C->edges[2 * i + k]] += 2;
    int *start = (int *) malloc(sizeof(int) * (V + 1));
    start[0] = 0;
    for (i = 0; i < V; i++) start[i + 1] = start[i] + deg[i];
    int *tmp = (int *) malloc(sizeof(int) * (start[V] ? start[V] : 1));
    memset(deg, 0, sizeof(int) * V);
    for (i = 0; i < C->T; i++) for (k = 0; k < 3; k++) { int a = C->tri[3 * i + k], j; for (j = 0; j < 3; j++) tmp[start[a] + deg[a]++] = C->tri[3 * i + j]; }
    for (i = 0; i < C->E; i++) for (k = 0; k < 2; k++) { int a = C->edges[2 * i + k], j; for (j = 0; j < 2; j++) tmp[start[a] + deg[a]++] = C->edges[2 * i + j]; }
    C->rowptr = (int *) malloc(sizeof(int) * (V + 1));
    C->rowptr[0] = 0;
    int nnz = 0;
    for (i = 0; i < V; i++) {
        int *r = tmp + start[i], n = deg[i], m = 0, j;
        qsort(r, n, sizeof(int), cmp_int);
        for (j = 0; j < n; j++) if (j == 0 || r[j] != r[j - 1]) r[m++] = r[j];
        deg[i] = m;
        nnz += m;
        C->rowptr[i + 1] = nnz;
    }
    C->col = (int *) malloc(sizeof(int) * nnz);
    for (i = 0; i < V; i++) memcpy(C->col + C->rowptr[i], tmp + start[i], sizeof(int) * deg[i]);
    C->nnzb = nnz;
    free(tmp); free(start); free(deg);
    C->blk_of_pair = (int *) malloc(sizeof(int) * 9 * (C->T ? C->T : 1));
    for (i = 0; i < C->T; i++) { int a, b; for (a = 0; a < 3; a++) for (b = 0; b < 3; b++) C->blk_of_pair[9 * i + 3 * a + b] = find_blk(C, C->tri[3 * i + a], C->tri[3 * i + b]); }
    C->eblk_of_pair = (int *) malloc(sizeof(int) * 4 * (C->E ? C->E : 1));
    for (i = 0; i < C->E; i++) { int a, b; for (a = 0; a < 2; a++) for (b = 0; b < 2; b++) C->eblk_of_pair[4 * i + 2 * a + b] = find_blk(C, C->edges[2 * i + a], C->edges[2 * i + b]); }
    C->val = (double *) calloc((size_t) 9 * nnz, sizeof(double));
    return 0;
}

/* reverse Cuthill-McKee node order for the banded LU of the oracle's preconditioner */
static void rcm_order(orc_ctx *C) {
    int V = C->V, i, head = 0, tail = 0, k;
    int *deg = (int *) malloc(sizeof(int) * V), *seen = (int *) calloc(V, sizeof(int));
    int *order = (int *) malloc(sizeof(int) * V);
    for (i = 0; i < V; i++) deg[i] = C->rowptr[i + 1] - C->rowptr[i];
    while (tail < V) {
        int s = -1;
        for (i = 0; i < V; i++) if (!seen[i] && (s < 0 || deg[i] < deg[s])) s = i;
        seen[s] = 1; order[tail++] = s;
        while (head < tail) {
            int a = order[head++], n0 = tail;
            for (k = C->rowptr[a]; k < C->rowptr[a + 1]; k++) { int b = C->col[k]; if (!seen[b]) { seen[b] = 1; order[tail++] = b; } }
            /* sort the newly added by degree */
            int p, q;
            for (p = n0 + 1; p < tail; p++) { int t = order[p]; q = p - 1; while (q >= n0 && deg[order[q]] > deg[t]) { order[q + 1] = order[q]; q--; } order[q + 1] = t; }
        }
    }
    C->perm = (int *) malloc(sizeof(int) * V);
    C->iperm = (int *) malloc(sizeof(int) * V);
    for (i = 0; i < V; i++) { C->perm[i] = order[V - 1 - i]; }
    for (i = 0; i < V; i++) C->iperm[C->perm[i]] = i;
    int bw = 0;
    for (i = 0; i < V; i++) for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) { int d = abs(C->iperm[i] - C->iperm[C->col[k]]); if (d > bw) bw = d; }
    C->bandwidth_nodes = bw;
    free(deg); free(seen); free(order);
}

orc_ctx *orc_create(const sw2gpu_mesh *m, const sw2gpu_params *p, int nblock) {
    orc_ctx *C = (orc_ctx *) calloc(1, sizeof(orc_ctx));
    int i, k;
    C->V = m->nnodes; C->T = m->nelems2d; C->E = m->nelems1d; C->S = m->nstrings; C->M = m->nmats; C->NS = m->nseries;
    C->p = *p;
    C->nblock = nblock < 1 ? 1 : nblock;
    C->x = (double *) dup(m->x, sizeof(double) * C->V);
    C->y = (double *) dup(m->y, sizeof(double) * C->V);
    C->z = (double *) dup(m->z, sizeof(double) * C->V);
    C->node_string = (int *) dup(m->node_string, sizeof(int) * C->V);
    C->tri = (int *) dup(m->elem2d_nodes, sizeof(int) * 3 * C->T);
    C->tri_mat = (int *) dup(m->elem2d_mat, sizeof(int) * C->T);
    C->edges = (int *) dup(m->elem1d_nodes, sizeof(int) * 2 * C->E);
    C->edge_string = (int *) dup(m->elem1d_string, sizeof(int) * C->E);
    C->edge_parent = (int *) dup(m->elem1d_parent, sizeof(int) * C->E);
    C->str_bc = (int *) dup(m->str_bc_flag, sizeof(int) * C->S);
    C->str_isigma = (int *) dup(m->str_isigma, sizeof(int) * C->S);
    C->str_ivx = (int *) dup(m->str_ivx, sizeof(int) * C->S);
    C->str_ivy = (int *) dup(m->str_ivy, sizeof(int) * C->S);
    C->str_iu0 = (int *) dup(m->str_iu0, sizeof(int) * C->S);
    C->str_rough = (double *) dup(m->str_rough_height, sizeof(double) * C->S);
    C->mat_eev_mode = (int *) dup(m->mat_eev_mode, sizeof(int) * C->M);
    C->mat_ev = (double *) dup(m->mat_ev, sizeof(double) * 3 * C->M);
    C->mat_eev_coef = (double *) dup(m->mat_eev_coef, sizeof(double) * C->M);
    C->mat_cor = (double *) dup(m->mat_coriolis, sizeof(double) * C->M);
    C->series = (double *) calloc(C->NS > 0 ? C->NS : 1, sizeof(double));
    for (k = 0; k < 3; k++) {
        C->h[k] = (double *) calloc(C->V, sizeof(double));
        C->u[k] = (double *) calloc(C->V, sizeof(double));
        C->v[k] = (double *) calloc(C->V, sizeof(double));
    }
    C->wd = (int *) calloc(C->T ? C->T : 1, sizeof(int));
    C->dacont = (double *) calloc(3 * (size_t) (C->T ? C->T : 1), sizeof(double));
    C->resid = (double *) calloc(3 * C->V, sizeof(double));
    C->sol = (double *) calloc(3 * C->V, sizeof(double));
    C->include = (int *) calloc(C->V, sizeof(int));
    for (i = 0; i < C->V; i++) {                       /* node strings: ids in range, no lids */
        int s = C->node_string[i];
        if (s >= C->S) { fprintf(stderr, "oracle: node %d has bad string %d\n", i, s); free(C); return NULL; }
        if (s > SW2GPU_NORMAL && (C->str_bc[s] == SW2GPU_BCT_LID_DFT || C->str_bc[s] == SW2GPU_BCT_LID_ELV ||
                                  C->str_bc[s] == SW2GPU_BCT_LID_DEP)) {
            fprintf(stderr, "oracle: lid boundary condition on node %d not supported\n", i); free(C); return NULL;
        }
    }
    /* geometry (element_djac_nrml_gradPhi.c:193-273, elem1d_outward_nrml.c) */
    C->djac = (double *) malloc(sizeof(double) * (C->T ? C->T : 1));
    C->grad = (double *) malloc(sizeof(double) * 6 * (C->T ? C->T : 1));
    for (i = 0; i < C->T; i++) {
        int a = C->tri[3 * i], b = C->tri[3 * i + 1], c = C->tri[3 * i + 2];
        double s1x = C->x[b] - C->x[a], s1y = C->y[b] - C->y[a], s2x = C->x[c] - C->x[a], s2y = C->y[c] - C->y[a];
        double cr = s1x * s2y - s2x * s1y;
        double *g = C->grad + 6 * i;
        g[0] = (s1y - s2y) / cr; g[1] = (s2x - s1x) / cr;
        g[2] = s2y / cr;         g[3] = -s2x / cr;
        g[4] = -s1y / cr;        g[5] = s1x / cr;
        C->djac[i] = cr * 0.5;
        if (C->djac[i] < 1e-6) { fprintf(stderr, "oracle: element %d not counter-clockwise\n", i); free(C); return NULL; }
    }
    C->edjac = (double *) malloc(sizeof(double) * (C->E ? C->E : 1));
    C->enrml = (double *) malloc(sizeof(double) * 2 * (C->E ? C->E : 1));
    for (i = 0; i < C->E; i++) {
        int a = C->edges[2 * i], b = C->edges[2 * i + 1], pe = C->edge_parent[i];
        double dx = C->x[b] - C->x[a], dy = C->y[b] - C->y[a], L = sqrt(dx * dx + dy * dy);
        double nx = dy / L, ny = -dx / L;
        double cx = ONE_3 * (C->x[C->tri[3 * pe]] + C->x[C->tri[3 * pe + 1]] + C->x[C->tri[3 * pe + 2]]);
        double cy = ONE_3 * (C->y[C->tri[3 * pe]] + C->y[C->tri[3 * pe + 1]] + C->y[C->tri[3 * pe + 2]]);
        if ((cx - C->x[a]) * nx + (cy - C->y[a]) * ny > 0.) { nx = -nx; ny = -ny; }
        C->edjac[i] = sqrt((C->x[a] - C->x[b]) * (C->x[a] - C->x[b]) + (C->y[a] - C->y[b]) * (C->y[a] - C->y[b]));
        C->enrml[2 * i] = nx; C->enrml[2 * i + 1] = ny;
        int f = C->str_bc[C->edge_string[i]];
        if (f != SW2GPU_BCT_VEL_NEU && f != SW2GPU_BCT_PRS_NEU && f != SW2GPU_BCT_OUTFLOW && f != SW2GPU_BCT_OVH_NEU) {
            fprintf(stderr, "oracle: unsupported edge bc flag %d\n", f); free(C); return NULL;
        }
    }
    build_pattern(C);
    rcm_order(C);
    return C;
}

void orc_destroy(orc_ctx *C) {
    int k;
    if (!C) return;
    free(C->x); free(C->y); free(C->z); free(C->node_string); free(C->tri); free(C->tri_mat);
    free(C->edges); free(C->edge_string); free(C->edge_parent); free(C->str_bc); free(C->str_isigma);
    free(C->str_ivx); free(C->str_ivy); free(C->str_iu0); free(C->str_rough); free(C->mat_eev_mode);
    free(C->mat_ev); free(C->mat_eev_coef); free(C->mat_cor); free(C->series); free(C->wsx); free(C->wsy);
    free(C->wvx); free(C->wvy);
    for (k = 0; k < 3; k++) { free(C->h[k]); free(C->u[k]); free(C->v[k]); }
    free(C->wd); free(C->dacont); free(C->resid); free(C->sol); free(C->include); free(C->djac); free(C->grad);
    free(C->edjac); free(C->enrml); free(C->rowptr); free(C->col); free(C->blk_of_pair); free(C->eblk_of_pair);
    free(C->val); free(C->perm); free(C->iperm);
    free(C->trn_refc); free(C->trn_dm); free(C->trn_bc); free(C->trn_ser); free(C->conc); free(C->bcmask);
    free(C->tval); free(C->tres); free(C->tsol);
    free(C);
}

int orc_nnzb(const orc_ctx *C) { return C->nnzb; }
int orc_bandwidth(const orc_ctx *C) { return C->bandwidth_nodes; }
void orc_pattern(const orc_ctx *C, int *rowptr, int *col) {
    memcpy(rowptr, C->rowptr, sizeof(int) * (C->V + 1));
    memcpy(col, C->col, sizeof(int) * C->nnzb);
}

void orc_set_state(orc_ctx *C, int level, const double *h, const double *u, const double *v) {
    memcpy(C->h[level], h, sizeof(double) * C->V);
    memcpy(C->u[level], u, sizeof(double) * C->V);
    memcpy(C->v[level], v, sizeof(double) * C->V);
}
void orc_get_state(const orc_ctx *C, int level, double *h, double *u, double *v) {
    memcpy(h, C->h[level], sizeof(double) * C->V);
    memcpy(u, C->u[level], sizeof(double) * C->V);
    memcpy(v, C->v[level], sizeof(double) * C->V);
}
void orc_set_dt(orc_ctx *C, double dt, const double *series) {
    C->dt = dt;
    if (C->NS > 0 && series) memcpy(C->series, series, sizeof(double) * C->NS);
}
void orc_get_wd(const orc_ctx *C, int *wd) { memcpy(wd, C->wd, sizeof(int) * C->T); }
/* elem_rhs_dacont_extra_terms, vertex-major like the reference's [3][T] array: out[i T + e] */
void orc_get_dacont(const orc_ctx *C, double *out) {
    int e, i;
    for (i = 0; i < 3; i++)
        for (e = 0; e < C->T; e++) out[(size_t) i * C->T + e] = C->dacont[3 * e + i];
}
void orc_set_wd(orc_ctx *C, const int *wd) { memcpy(C->wd, wd, sizeof(int) * C->T); }

/* fe_sw2_wdflag (src/fe/sw2/fe_sw2_wdflag.c:24-75) */
void orc_wdflag(orc_ctx *C) {
    int *tmp = (int *) calloc(C->V, sizeof(int)), e, i;
    for (e = 0; e < C->T; e++) {
        int wet = 0;
        for (i = 0; i < 3; i++) if (C->h[0][C->tri[3 * e + i]] > 0.0) wet++;
        if (wet != 3) for (i = 0; i < 3; i++) tmp[C->tri[3 * e + i]] = 1;
    }
    for (e = 0; e < C->T; e++) {
        const int *n = C->tri + 3 * e;
        C->wd[e] = 0;
        for (i = 0; i < 3; i++) if (tmp[n[i]] != 0) C->wd[e] = 1;
        if (C->h[0][n[0]] < 0 && C->h[0][n[1]] < 0 && C->h[0][n[2]] < 0 &&
            C->h[1][n[0]] < 0 && C->h[1][n[1]] < 0 && C->h[1][n[2]] < 0) C->wd[e] = 2;
    }
    free(tmp);
}

/* single element residual (unit tests): out[9] = node-major (c, x, y) */
/* boundary edge ie's residual (out[3 i + {c, x, y}] for its two nodes) at the current level,
 * with the perturbation psign * eps of variable pvar at its node pnode; also its length and
 * outward normal (geo = djac, nx, ny) */
void orc_edge_resid(orc_ctx *C, int ie, double eps, int pnode, int pvar, int psign, double *out, double *geo) {
    double hh[2];
    v2 vel[2];
    dof3 er[2];
    int i;
    for (i = 0; i < 2; i++) {
        int n = C->edges[2 * ie + i];
        hh[i] = C->h[0][n];
        vel[i].x = C->u[0][n];
        vel[i].y = C->v[0][n];
    }
    if (pvar == P_H) hh[pnode] += psign * eps;
    else if (pvar == P_U) vel[pnode].x += psign * eps;
    else if (pvar == P_V) vel[pnode].y += psign * eps;
    boundary_resid(C, ie, hh, vel, pvar, er);
    for (i = 0; i < 2; i++) { out[3 * i] = er[i].c; out[3 * i + 1] = er[i].x; out[3 * i + 2] = er[i].y; }
    geo[0] = C->edjac[ie];
    geo[1] = C->enrml[2 * ie];
    geo[2] = C->enrml[2 * ie + 1];
}

/* element ie's area and P1 shape gradients: out = djac, gx0, gy0, gx1, gy1, gx2, gy2 */
void orc_geometry(const orc_ctx *C, int ie, double *out) {
    int i;
    out[0] = C->djac[ie];
    for (i = 0; i < 6; i++) out[1 + i] = C->grad[6 * ie + i];
}

void orc_body_resid(orc_ctx *C, int ie, double eps, int pnode, int pvar, int psign, double *out) {
    elem_in E; dof3 er[3]; int i;
    gather_elem(C, ie, &E);
    if (pvar == P_H) E.h[pnode] += psign * eps;
    else if (pvar == P_U) E.vel[pnode].x += psign * eps;
    else if (pvar == P_V) E.vel[pnode].y += psign * eps;
    body_resid(C, ie, &E, pvar, er);
    for (i = 0; i < 3; i++) { out[3 * i] = er[i].c; out[3 * i + 1] = er[i].x; out[3 * i + 2] = er[i].y; }
}

/* fe_sw2_resid (src/fe/sw2/fe_sw2_resid.c:29-216); R ordered [u, v, h] per node */
void orc_resid(orc_ctx *C, double *R) {
    int e, i;
    memset(C->resid, 0, sizeof(double) * 3 * C->V);
    for (e = 0; e < C->T; e++) {
        elem_in E; dof3 er[3];
        gather_elem(C, e, &E);
        body_resid(C, e, &E, P_NONE, er);
        for (i = 0; i < 3; i++) {
            int n = C->tri[3 * e + i];
            if (C->h[1][n] <= 0.) { er[i].x = 0.0; er[i].y = 0.0; C->u[0][n] = 0.; C->v[0][n] = 0.; }
        }
        for (i = 0; i < 3; i++) {
            int n = C->tri[3 * e + i];
            C->resid[3 * n] -= er[i].x; C->resid[3 * n + 1] -= er[i].y; C->resid[3 * n + 2] -= er[i].c;
        }
    }
    for (e = 0; e < C->E; e++) {
        double hh[2]; v2 vel[2]; dof3 er[2];
        for (i = 0; i < 2; i++) { int n = C->edges[2 * e + i]; hh[i] = C->h[0][n]; vel[i].x = C->u[0][n]; vel[i].y = C->v[0][n]; }
        boundary_resid(C, e, hh, vel, P_NONE, er);
        for (i = 0; i < 2; i++) {
            int n = C->edges[2 * e + i];
            if (C->h[1][n] <= 0.) { er[i].x = 0.0; er[i].y = 0.0; C->u[0][n] = 0.; C->v[0][n] = 0.; }
        }
        for (i = 0; i < 2; i++) {
            int n = C->edges[2 * e + i];
            C->resid[3 * n] -= er[i].x; C->resid[3 * n + 1] -= er[i].y; C->resid[3 * n + 2] -= er[i].c;
        }
    }
    if (R) memcpy(R, C->resid, sizeof(double) * 3 * C->V);
}

/* NUM_DIFF_EPSILON (macro.h:669-673) */
static double fd_eps(double var) {
    double p = sqrt(ORC_SMALL), e = fabs(var) * (1. + p);
    e -= fabs(var);
    if (e < p) e = p;
    return e;
}

/* fe_assign_mom_db_dof3 / fe_assign_dacont_db_dof3 (src/fe/fe_assign_elem_mat_db.c:30-55, 196-219)
 * M[var][row*n+col] with var 0 = u, 1 = v, 2 = h and entries dof3 (c, x, y) */
static void mom_db(int i, int n, dof3 M[3][9]) {
    int j;
    for (j = n * i; j < n * i + n; j++) { M[0][j].x = 0.; M[0][j].y = 0.; M[1][j].x = 0.; M[1][j].y = 0.; M[2][j].x = 0.; M[2][j].y = 0.; }
    for (j = i; j < n * n; j += n) { M[0][j].x = 0.; M[0][j].y = 0.; M[0][j].c = 0.; M[1][j].x = 0.; M[1][j].y = 0.; M[1][j].c = 0.; }
    M[0][i * (n + 1)].x = 1.;
    M[1][i * (n + 1)].y = 1.;
}
static void dacont_db(int i, int n, dof3 M[3][9]) {
    int j;
    for (j = n * i; j < n * i + n; j++) { M[0][j].c = 0.; M[1][j].c = 0.; M[2][j].c = 0.; }
    for (j = i; j < n * n; j += n) { M[2][j].x = 0.; M[2][j].y = 0.; M[2][j].c = 0.; }
    M[2][i * (n + 1)].c = 1.;
}

static void add_block(orc_ctx *C, int blk, const dof3 M[3][9], int idx) {
    double *b = C->val + 9 * (size_t) blk;           /* fe_global_matrix_assemble_sw2 :203-211 */
    b[0] += M[0][idx].x; b[1] += M[1][idx].x; b[2] += M[2][idx].x;
    b[3] += M[0][idx].y; b[4] += M[1][idx].y; b[5] += M[2][idx].y;
    b[6] += M[0][idx].c; b[7] += M[1][idx].c; b[8] += M[2][idx].c;
}

/* fe_sw2_load: FD Jacobian in sorted BCSR + tiny-diagonal fix of R (uses C->resid) */
void orc_load(orc_ctx *C) {
    int e, i, j, k;
    memset(C->val, 0, sizeof(double) * 9 * (size_t) C->nnzb);
    for (e = 0; e < C->T; e++) {
        dof3 M[3][9];
        memset(M, 0, sizeof M);
        elem_in E0;
        gather_elem(C, e, &E0);
        for (i = 0; i < 3; i++) {
            int n = C->tri[3 * e + i];
            double eps[3] = {fd_eps(C->u[0][n]), fd_eps(C->v[0][n]), fd_eps(C->h[0][n])};
            int pv[3] = {P_U, P_V, P_H}, var;
            for (var = 0; var < 3; var++) {
                /* reference order: head first (perturb_sw2_head), then u and v */
                int vv = (var + 2) % 3;
                elem_in Ep = E0, Em = E0;
                dof3 rp[3], rm[3];
                if (pv[vv] == P_H) { Ep.h[i] += eps[vv]; Em.h[i] -= eps[vv]; }
                else if (pv[vv] == P_U) { Ep.vel[i].x += eps[vv]; Em.vel[i].x -= eps[vv]; }
                else { Ep.vel[i].y += eps[vv]; Em.vel[i].y -= eps[vv]; }
                body_resid(C, e, &Ep, pv[vv], rp);
                body_resid(C, e, &Em, pv[vv], rm);
                double e2 = 2.0 * eps[vv];
                for (k = 0; k < 3; k++) {          /* elem_matrix_deriv (fe_elem_utilities.c:518-524) */
                    M[vv][i + 3 * k].x = (rp[k].x - rm[k].x) / e2;
                    M[vv][i + 3 * k].y = (rp[k].y - rm[k].y) / e2;
                    M[vv][i + 3 * k].c = (rp[k].c - rm[k].c) / e2;
                }
            }
        }
        for (i = 0; i < 3; i++) {
            int n = C->tri[3 * e + i];
            int ns = C->node_string[i];            /* element-local index used as node id (:103) */
            if (C->h[1][n] <= 0.) mom_db(i, 3, M);
            if (ns > SW2GPU_NORMAL) {
                int f = C->str_bc[ns];
                if (f == SW2GPU_BCT_PRS_DIR) dacont_db(i, 3, M);
                else if (f == SW2GPU_BCT_VEL_DIR) mom_db(i, 3, M);
                else if (f == SW2GPU_BCT_VEL_PRS_DIR) { dacont_db(i, 3, M); mom_db(i, 3, M); }
            }
        }
        for (i = 0; i < 3; i++) for (j = 0; j < 3; j++) add_block(C, C->blk_of_pair[9 * e + 3 * i + j], M, 3 * i + j);
    }
    for (e = 0; e < C->E; e++) {
        dof3 M[3][9];
        memset(M, 0, sizeof M);
        double h0[2]; v2 v0[2];
        for (i = 0; i < 2; i++) { int n = C->edges[2 * e + i]; h0[i] = C->h[0][n]; v0[i].x = C->u[0][n]; v0[i].y = C->v[0][n]; }
        for (i = 0; i < 2; i++) {
            int n = C->edges[2 * e + i];
            double eps[3] = {fd_eps(C->u[0][n]), fd_eps(C->v[0][n]), fd_eps(C->h[0][n])};
            int pv[3] = {P_U, P_V, P_H}, var;
            for (var = 0; var < 3; var++) {
                int vv = (var + 2) % 3;
                double hp[2] = {h0[0], h0[1]}, hm[2] = {h0[0], h0[1]};
                v2 vp[2] = {v0[0], v0[1]}, vm[2] = {v0[0], v0[1]};
                dof3 rp[2], rm[2];
                if (pv[vv] == P_H) { hp[i] += eps[vv]; hm[i] -= eps[vv]; }
                else if (pv[vv] == P_U) { vp[i].x += eps[vv]; vm[i].x -= eps[vv]; }
                else { vp[i].y += eps[vv]; vm[i].y -= eps[vv]; }
                boundary_resid(C, e, hp, vp, pv[vv], rp);
                boundary_resid(C, e, hm, vm, pv[vv], rm);
                double e2 = 2.0 * eps[vv];
                for (k = 0; k < 2; k++) {
                    M[vv][i + 2 * k].x = (rp[k].x - rm[k].x) / e2;
                    M[vv][i + 2 * k].y = (rp[k].y - rm[k].y) / e2;
                    M[vv][i + 2 * k].c = (rp[k].c - rm[k].c) / e2;
                }
            }
        }
        for (i = 0; i < 2; i++) {
            int n = C->edges[2 * e + i];
            int ns = C->node_string[i];
            if (C->h[1][n] <= 0.) mom_db(i, 2, M);
            if (ns > SW2GPU_NORMAL) {
                int f = C->str_bc[ns];
                if (f == SW2GPU_BCT_PRS_DIR) dacont_db(i, 2, M);
                else if (f == SW2GPU_BCT_VEL_DIR) mom_db(i, 2, M);
                else if (f == SW2GPU_BCT_VEL_PRS_DIR) { dacont_db(i, 2, M); mom_db(i, 2, M); }
            }
        }
        for (i = 0; i < 2; i++) for (j = 0; j < 2; j++) add_block(C, C->eblk_of_pair[4 * e + 2 * i + j], M, 2 * i + j);
    }
    /* tiny diagonal fix (fe_sw2_load.c:218-236) */
    for (i = 0; i < C->V; i++) {
        double *d = C->val + 9 * (size_t) find_blk(C, i, i);
        if (fabs(d[0]) < ORC_NQS) { d[0] = ORC_NQS; if (fabs(C->resid[3 * i]) < ORC_NQS) C->resid[3 * i] = -ORC_NQS * C->u[0][i]; }
        if (fabs(d[4]) < ORC_NQS) { d[4] = ORC_NQS; if (fabs(C->resid[3 * i + 1]) < ORC_NQS) C->resid[3 * i + 1] = -ORC_NQS * C->v[0][i]; }
        if (fabs(d[8]) < ORC_NQS) d[8] = ORC_NQS;
    }
}

void orc_get_matrix(const orc_ctx *C, double *val, double *resid) {
    if (val) memcpy(val, C->val, sizeof(double) * 9 * (size_t) C->nnzb);
    if (resid) memcpy(resid, C->resid, sizeof(double) * 3 * C->V);
}
void orc_set_matrix(orc_ctx *C, const double *val, const double *resid) {
    if (val) memcpy(C->val, val, sizeof(double) * 9 * (size_t) C->nnzb);
    if (resid) memcpy(C->resid, resid, sizeof(double) * 3 * C->V);
}

/* ------------------------------------------------------------------------------ */
/* linear solve: spv_jacobi scaling, block-LU preconditioned BiCGSTAB, unscaling   */

static void amult(const orc_ctx *C, const double *x, double *y) {   /* solv_amult.c:92-129 */
    int i, k, a, b;
    for (i = 0; i < C->V; i++) {
        double s[3] = {0, 0, 0};
        for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) {
            const double *m = C->val + 9 * (size_t) k;
            const double *xx = x + 3 * C->col[k];
            for (a = 0; a < 3; a++) for (b = 0; b < 3; b++) s[a] += m[3 * a + b] * xx[b];
        }
        y[3 * i] = s[0]; y[3 * i + 1] = s[1]; y[3 * i + 2] = s[2];
    }
}

typedef struct {            /* banded LU of contiguous blocks of the RCM-ordered dofs */
    int n, nb;               /* dofs, blocks */
    int *bstart, *bw;        /* per block: first dof (permuted), half bandwidth (dofs) */
    double **band;           /* per block: (2*bw+1) x len */
    int *fail;
} bandlu;

static void band_factor(const orc_ctx *C, bandlu *L) {
    int V = C->V, n = 3 * V, b;
    L->n = n;
    L->nb = C->nblock;
    L->bstart = (int *) malloc(sizeof(int) * (L->nb + 1));
    L->bw = (int *) calloc(L->nb, sizeof(int));
    L->band = (double **) calloc(L->nb, sizeof(double *));
    for (b = 0; b <= L->nb; b++) L->bstart[b] = 3 * (int) ((long long) V * b / L->nb);
    /* bandwidth per block */
    int i, k, a, q;
    for (i = 0; i < V; i++) {
        int pi = C->iperm[i], blk = (int) ((long long) pi * L->nb / V);
        while (blk > 0 && 3 * pi < L->bstart[blk]) blk--;
        while (3 * pi >= L->bstart[blk + 1]) blk++;
        for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) {
            int pj = C->iperm[C->col[k]];
            if (3 * pj < L->bstart[blk] || 3 * pj >= L->bstart[blk + 1]) continue;
            int d = 3 * abs(pi - pj) + 2;
            if (d > L->bw[blk]) L->bw[blk] = d;
        }
    }
    for (b = 0; b < L->nb; b++) {
        int len = L->bstart[b + 1] - L->bstart[b], w = L->bw[b], W = 2 * w + 1;
        double *B = (double *) calloc((size_t) len * W, sizeof(double));
        L->band[b] = B;
        /* load: row r (local), col c (local) at B[r*W + (c - r + w)] */
        for (i = 0; i < V; i++) {
            int pi = C->iperm[i];
            if (3 * pi < L->bstart[b] || 3 * pi >= L->bstart[b + 1]) continue;
            for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) {
                int pj = C->iperm[C->col[k]];
                if (3 * pj < L->bstart[b] || 3 * pj >= L->bstart[b + 1]) continue;
                const double *m = C->val + 9 * (size_t) k;
                for (a = 0; a < 3; a++) for (q = 0; q < 3; q++) {
                    int r = 3 * pi + a - L->bstart[b], c = 3 * pj + q - L->bstart[b];
                    B[(size_t) r * W + (c - r + w)] = m[3 * a + q];
                }
            }
        }
        /* Doolittle LU without pivoting within the band */
        int r, c, j;
        for (r = 0; r < len; r++) {
            double piv = B[(size_t) r * W + w];
            if (piv == 0.0) piv = B[(size_t) r * W + w] = ORC_SMALL;
            int rend = r + w < len - 1 ? r + w : len - 1;
            for (j = r + 1; j <= rend; j++) {
                double *Rj = B + (size_t) j * W;
                double l = Rj[r - j + w] / piv;
                if (l == 0.0) continue;
                Rj[r - j + w] = l;
                const double *Rr = B + (size_t) r * W;
                int cend = r + w < len - 1 ? r + w : len - 1;
                for (c = r + 1; c <= cend; c++) Rj[c - j + w] -= l * Rr[c - r + w];
            }
        }
    }
}

static void band_solve(const orc_ctx *C, const bandlu *L, const double *in, double *out) {
    int b, i, a;
    double *t = (double *) malloc(sizeof(double) * L->n);
    for (i = 0; i < C->V; i++) for (a = 0; a < 3; a++) t[3 * C->iperm[i] + a] = in[3 * i + a];
    for (b = 0; b < L->nb; b++) {
        int s = L->bstart[b], len = L->bstart[b + 1] - s, w = L->bw[b], W = 2 * w + 1, r, c;
        const double *B = L->band[b];
        double *x = t + s;
        for (r = 0; r < len; r++) {
            int c0 = r - w > 0 ? r - w : 0;
            double acc = x[r];
            for (c = c0; c < r; c++) acc -= B[(size_t) r * W + (c - r + w)] * x[c];
            x[r] = acc;
        }
        for (r = len - 1; r >= 0; r--) {
            int c1 = r + w < len - 1 ? r + w : len - 1;
            double acc = x[r];
            for (c = r + 1; c <= c1; c++) acc -= B[(size_t) r * W + (c - r + w)] * x[c];
            x[r] = acc / B[(size_t) r * W + w];
        }
    }
    for (i = 0; i < C->V; i++) for (a = 0; a < 3; a++) out[3 * i + a] = t[3 * C->iperm[i] + a];
    free(t);
}

static void band_free(bandlu *L) {
    int b;
    for (b = 0; b < L->nb; b++) free(L->band[b]);
    free(L->band); free(L->bstart); free(L->bw);
}

static double inf_norm(const double *a, int n) { double m = 0; int i; for (i = 0; i < n; i++) if (fabs(a[i]) > m) m = fabs(a[i]); return m; }
static double dotp(const double *a, const double *b, int n) { double s = 0; int i; for (i = 0; i < n; i++) s += a[i] * b[i]; return s; }

/* Solves val * x = rhs; val is overwritten with the scaled matrix.  Returns the
 * number of BiCGSTAB iterations, or -1 when max_lin_it was reached. */
int orc_linear_solve(orc_ctx *C, double *rhs, double *x) {
    int n = 3 * C->V, i, k, a, b;
    double *S = (double *) malloc(sizeof(double) * n);
    /* spv_jacobi (src/solver/spv_jacobi.c:222-317): row max over diagonal and off-diagonal blocks */
    for (i = 0; i < n; i++) S[i] = 0.0;
    for (i = 0; i < C->V; i++)
        for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) {
            const double *m = C->val + 9 * (size_t) k;
            for (a = 0; a < 3; a++) for (b = 0; b < 3; b++) if (fabs(m[3 * a + b]) > S[3 * i + a]) S[3 * i + a] = fabs(m[3 * a + b]);
        }
    double small_factor = 1.0 / sqrt(ORC_SMALL);
    for (i = 0; i < n; i++) S[i] = (S[i] < ORC_SMALL) ? small_factor : 1.0 / sqrt(fabs(S[i]));
    for (i = 0; i < n; i++) rhs[i] *= S[i];
    for (i = 0; i < C->V; i++)
        for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) {
            double *m = C->val + 9 * (size_t) k;
            int j = C->col[k];
            for (a = 0; a < 3; a++) for (b = 0; b < 3; b++) m[3 * a + b] *= S[3 * i + a] * S[3 * j + b];
        }
    bandlu L;
    band_factor(C, &L);
    /* solv_bcgstab (src/solver/solv_bcgstab.c:39-301), initial guess 0 */
    double *r = calloc(n, 8), *p = calloc(n, 8), *Ap = calloc(n, 8), *Mp = calloc(n, 8), *q = calloc(n, 8);
    double *s = calloc(n, 8), *As = calloc(n, 8), *Ms = calloc(n, 8), *u = calloc(n, 8), *bb = calloc(n, 8);
    band_solve(C, &L, rhs, bb);                       /* b <- M^-1 b */
    memcpy(u, bb, sizeof(double) * n);
    amult(C, u, Mp);
    band_solve(C, &L, Mp, Ap);
    for (i = 0; i < n; i++) r[i] = bb[i] - Ap[i];
    memset(Mp, 0, sizeof(double) * (size_t) n); memset(Ap, 0, sizeof(double) * (size_t) n);
    memcpy(q, r, sizeof(double) * n);
    double rnorm = inf_norm(r, n), bnorm = inf_norm(bb, n);
    double rhop = 1.0, alpha = 1.0, omega = 1.0, rho = dotp(r, q, n), beta, gamma;
    double atol = C->p.lin_atol, rtol = C->p.lin_rtol;
    int it = 0;
    while (rnorm > (atol + bnorm * rtol) && it < C->p.max_lin_it) {
        it++;
        beta = (rho * alpha) / (rhop * omega);
        for (i = 0; i < n; i++) { p[i] -= omega * Ap[i]; p[i] *= beta; p[i] += r[i]; }
        amult(C, p, Mp);
        band_solve(C, &L, Mp, Ap);
        gamma = dotp(q, Ap, n);
        alpha = rho / gamma;
        for (i = 0; i < n; i++) s[i] = r[i] - alpha * Ap[i];
        amult(C, s, Ms);
        band_solve(C, &L, Ms, As);
        omega = dotp(As, s, n);
        gamma = dotp(As, As, n);
        omega = omega / gamma;
        rhop = rho;
        rho = -1.0 * omega * dotp(As, q, n);
        for (i = 0; i < n; i++) { u[i] += alpha * p[i]; u[i] += omega * s[i]; }
        for (i = 0; i < n; i++) r[i] = s[i] - omega * As[i];
        rnorm = inf_norm(r, n);
    }
    for (i = 0; i < n; i++) x[i] = u[i] * S[i];       /* solv_return_old.c:5-38 */
    band_free(&L);
    free(r); free(p); free(Ap); free(Mp); free(q); free(s); free(As); free(Ms); free(u); free(bb); free(S);
    return (it == C->p.max_lin_it) ? -1 : it;
}

/* ------------------------------------------------------------------------------ */
/* Newton step */

static void init_state(orc_ctx *C) {                  /* fe_sw2_init (src/fe/sw2/fe_sw2_init.c:24-92) */
    int i;
    memcpy(C->u[0], C->u[1], sizeof(double) * C->V);
    memcpy(C->v[0], C->v[1], sizeof(double) * C->V);
    memcpy(C->h[0], C->h[1], sizeof(double) * C->V);
    for (i = 0; i < C->V; i++) {
        int s = C->node_string[i];
        if (s > SW2GPU_NORMAL) {
            int f = C->str_bc[s];
            if (f == SW2GPU_BCT_VEL_DIR || f == SW2GPU_BCT_VEL_PRS_DIR) { C->u[0][i] = C->series[C->str_ivx[s]]; C->v[0][i] = C->series[C->str_ivy[s]]; }
            if (f == SW2GPU_BCT_PRS_DIR || f == SW2GPU_BCT_VEL_PRS_DIR) C->h[0][i] = C->series[C->str_iu0[s]];
        }
    }
    orc_wdflag(C);
}

static void norms(orc_ctx *C, double *rmax, double *rl2, double *imax) {   /* get_residual_norms :40-151 */
    int i, j;
    double l2 = 0, mx = 0, im = 0;
    for (i = 0; i < C->V; i++) C->include[i] = (MIND(C->h[0][i], C->h[1][i]) > 0) ? 1 : 0;
    for (i = 0; i < C->V; i++) for (j = 0; j < 3; j++) {
        double r = C->resid[3 * i + j], s = C->sol[3 * i + j];
        if (fabs(s) > im && C->include[i]) im = fabs(s);
        if (fabs(r) > mx && C->include[i]) mx = fabs(r);
        l2 += r * r;
    }
    *rmax = mx; *rl2 = sqrt(l2 / (C->V * 3)); *imax = im;
}

static void inc(orc_ctx *C) {                         /* fe_sw2_inc.c:24-57 */
    int i;
    for (i = 0; i < C->V; i++) { C->u[0][i] += C->sol[3 * i]; C->v[0][i] += C->sol[3 * i + 1]; C->h[0][i] += C->sol[3 * i + 2]; }
}

/* one time step: shift (fe_sw2.c:43-50) + Newton (fe_newton).  Returns 0 on success,
 * SW2GPU_E_NEWTON / E_LINEAR / E_NAN on failure (state reset to old level). */
int orc_step(orc_ctx *C, double dt, const double *series, sw2gpu_stats *st) {
    int V = C->V, i;
    memcpy(C->h[2], C->h[1], 8 * V); memcpy(C->u[2], C->u[1], 8 * V); memcpy(C->v[2], C->v[1], 8 * V);
    memcpy(C->h[1], C->h[0], 8 * V); memcpy(C->u[1], C->u[0], 8 * V); memcpy(C->v[1], C->v[0], 8 * V);
    orc_set_dt(C, dt, series);
    const sw2gpu_params *P = &C->p;
    double rmax, rl2, imax, old_l2;
    int it = 0, lin_total = 0, cuts_total = 0, solv_ok = 1, isnan_flag = 0;
    init_state(C);
    orc_resid(C, NULL);
    norms(C, &rmax, &rl2, &imax);
    double *rhs = (double *) malloc(sizeof(double) * 3 * V);
    int keep;
    do {
        orc_load(C);
        memcpy(rhs, C->resid, sizeof(double) * 3 * V);
        int lits = orc_linear_solve(C, rhs, C->sol);
        if (lits < 0) { solv_ok = 0; lits = P->max_lin_it; }
        lin_total += lits;
        inc(C);
        for (i = 0; i < 3 * V; i++) C->sol[i] = -C->sol[i];
        old_l2 = rl2;
        orc_resid(C, NULL);
        norms(C, &rmax, &rl2, &imax);
        if (isnan(rl2) || isinf(rl2)) { solv_ok = 0; isnan_flag = 1; }
        int cuts = 0;
        while (rmax > P->tol_nonlin && rl2 > old_l2 && cuts < P->max_linesearch_cuts) {
            for (i = 0; i < 3 * V; i++) C->sol[i] *= 0.5;
            inc(C);
            orc_resid(C, NULL);
            norms(C, &rmax, &rl2, &imax);
            cuts++;
        }
        cuts_total += cuts;
        it++;
        keep = solv_ok && it < P->max_nonlin_it && rmax < 1.0E+20 && (rmax > P->tol_nonlin && imax > P->inc_nonlin);
    } while (keep);
    free(rhs);
    int rc = SW2GPU_OK;
    if (!solv_ok || (rmax > P->tol_nonlin && imax > P->inc_nonlin) || rmax >= 1.0E+20) {
        rc = isnan_flag ? SW2GPU_E_NAN : (!solv_ok ? SW2GPU_E_LINEAR : SW2GPU_E_NEWTON);
        init_state(C);
    }
    if (st) {
        memset(st, 0, sizeof(*st));
        st->status = rc; st->newton_its = it; st->linear_its = lin_total; st->linesearch_cuts = cuts_total;
        st->resid_max = rmax; st->resid_l2 = rl2; st->inc_max = imax;
        for (i = 0; i < C->T; i++) if (C->wd[i]) st->wd_elems++;
    }
    return rc;
}

/* ------------------------------------------------------------------------------ */
/* grid mass diagnostics (src/tools/tl_grid_mass.c) */

/* fe_3m2d_dry_wet_factornew (tl_grid_mass.c:289-346): the wrapper's corner clip with "dry"
 * meaning h < 0 (not <= 0); also returns the number of dry vertices (0 or 3 when the clipped
 * corner is negligible) */
static double mass_wet_factor(const v2 *x, const double *h, double edjac, int *num_dry) {
    int i, total = 0, pass = 0, only;
    v2 nx[3];
    for (i = 0; i < 3; i++) {
        int dry = h[i] < 0.0;
        total += dry;
        pass += dry << i;
    }
    if (total == 3) { *num_dry = 3; return 0.0; }
    if (total == 0) { *num_dry = 0; return 1.0; }
    if (total != 1) pass = 7 - pass;
    only = pass / 2;
    for (i = 0; i < 3; i++) {
        if (i != only) {
            double xsi = h[i] / (h[i] - h[only]);
            nx[i].x = x[i].x + xsi * (x[only].x - x[i].x);
            nx[i].y = x[i].y + xsi * (x[only].y - x[i].y);
        } else {
            nx[i] = x[i];
        }
    }
    double djac = ((nx[1].x - nx[0].x) * (nx[2].y - nx[0].y) - (nx[1].y - nx[0].y) * (nx[2].x - nx[0].x)) / 2.0;
    if (djac / edjac < ORC_SMALL) {
        int odd = total % 2;
        *num_dry = odd == 1 ? 0 : 3;
        return (double) odd;
    }
    double factor = (double) ((total >> 1) - (total % 2));
    *num_dry = total;
    factor *= djac / edjac;
    return factor + ((factor < 0) ? 1.0 : 0.0);
}

static double tri_f(double djac, double c, const double *f) {   /* integrate_triangle_f, elem2d :60 */
    return c * djac * (f[0] + f[1] + f[2]) / 3.0;
}

/* tl_find_grid_mass_elem2d (tl_grid_mass.c:20-97): water mass of time level `level`; a
 * partially dry triangle adds its wet part and, with one dry vertex, the negative depth of the
 * dry corner counted as positive mass */
double orc_grid_mass(const orc_ctx *C, int level, double density) {
    const double *depth = C->h[level];
    double mass = 0.0;
    int e, i;
    for (e = 0; e < C->T; e++) {
        double eh[3], hneg[3] = {0.0, 0.0, 0.0}, f1, f2;
        v2 x[3];
        int num_dry;
        for (i = 0; i < 3; i++) {
            const int n = C->tri[3 * e + i];
            eh[i] = depth[n];
            x[i].x = C->x[n];
            x[i].y = C->y[n];
        }
        const double factor = mass_wet_factor(x, eh, C->djac[e], &num_dry);
        switch (num_dry) {
            case 1:
                for (i = 0; i < 3; i++)
                    if (eh[i] < 0.0) hneg[i] = eh[i];
                f1 = 1.0;
                f2 = -1.0 * (1.0 - factor);
                break;
            case 2:
                for (i = 0; i < 3; i++)
                    if (eh[i] < 0.0) { hneg[i] = eh[i]; eh[i] = 0.0; }
                f1 = factor;
                f2 = 0.0;
                break;
            default:
                f1 = factor;
                f2 = 0.0;
                break;
        }
        mass += tri_f(C->djac[e], f1, eh) + tri_f(C->djac[e], f2, hneg);
    }
    return mass * density;
}

/* The mass flux of one step for tl_find_grid_mass_error_elem2d (tl_grid_mass.c:102-159), at
 * the current level: water sources over BCT_WATER_SOURCE elements (the series value
 * `series_now[isigma]`, the wet/dry factor of fe_sw2_wet_dry_factor) and the implicit flow through
 * the boundary edges, -integrate_line_h_f(djac, density dt, v.n, h) per edge with the djac of
 * the first edge for every edge (grid->elem1d->djac, :141-142, kept).  The caller accumulates
 * these and forms |mass - accumulated flux - initial mass|. */
double orc_mass_flux(const orc_ctx *C, double density, double dt, const double *series_now) {
    double body = 0.0, edge = 0.0;
    int e, i;
    for (e = 0; e < C->T; e++) {
        const int s = C->tri_mat[e];
        if (C->str_bc[s] != SW2GPU_BCT_WATER_SOURCE) continue;
        double eh[3];
        v2 x[3];
        for (i = 0; i < 3; i++) {
            const int n = C->tri[3 * e + i];
            eh[i] = C->h[0][n];
            x[i].x = C->x[n];
            x[i].y = C->y[n];
        }
        const double factor = wd_factor(x, eh, C->djac[e]);
        body += series_now[C->str_isigma[s]] * C->djac[e] * dt * density * factor;
    }
    for (e = 0; e < C->E; e++) {
        double vn[2], eh[2];
        for (i = 0; i < 2; i++) {
            const int n = C->edges[2 * e + i];
            eh[i] = C->h[0][n];
            vn[i] = C->u[0][n] * C->enrml[2 * e] + C->v[0][n] * C->enrml[2 * e + 1];
        }
        const double t1 = C->edjac[0] * ONE_6 * (density * dt);    /* integrate_line_h_f, elem1d :18 */
        edge -= t1 * ((2 * vn[0] + vn[1]) * eh[0] + (vn[0] + 2 * vn[1]) * eh[1]);
    }
    return body + edge;
}

/* ------------------------------------------------------------------------------ */
/* Adaption error indicator (ssw_2d_calculate_elem_error, src/structs/ssw_2d.c:424-500):
 * per element the steady continuity residual at the vertices, ((h_i - h_old_i) / dt +
 * u_i dh/dx + v_i dh/dy + h_i (du/dx + dv/dy))^2, summed over the three vertices, square root,
 * times the area; elem_error = that / refine_tol[material] (0.5 for an element with wd_flag > 0);
 * node_error = the unscaled element values averaged over each node's elements (:471-496).  The
 * state is level 0 (the step's result) and level 1 (its old level), dt the step's. */
void orc_elem_error(const orc_ctx *C, const double *refine_tol, double *elem_error, double *node_error) {
    int e, i;
    int *cnt = (int *) calloc((size_t) C->V, sizeof(int));
    for (i = 0; i < C->V; i++) node_error[i] = 0.;
    for (e = 0; e < C->T; e++) {
        const int *n = C->tri + 3 * e;
        const double *g = C->grad + 6 * e;
        double hh[3], ho[3], uu[3], vv[3], c[3];
        double dhdx = 0., dhdy = 0., dudx = 0., dvdy = 0.;
        for (i = 0; i < 3; i++) {
            hh[i] = C->h[0][n[i]]; ho[i] = C->h[1][n[i]]; uu[i] = C->u[0][n[i]]; vv[i] = C->v[0][n[i]];
        }
        for (i = 0; i < 3; i++) {
            dhdx += g[2 * i] * hh[i];
            dhdy += g[2 * i + 1] * hh[i];
            dudx += g[2 * i] * uu[i];
            dvdy += g[2 * i + 1] * vv[i];
        }
        for (i = 0; i < 3; i++) {
            c[i] = (hh[i] - ho[i]) / C->dt;
            c[i] += uu[i] * dhdx;
            c[i] += vv[i] * dhdy;
            c[i] += hh[i] * (dudx + dvdy);
            c[i] = c[i] * c[i];
        }
        double err = sqrt(c[0] + c[1] + c[2]) * C->djac[e];
        for (i = 0; i < 3; i++) {
            node_error[n[i]] += err;
            cnt[n[i]] += 1;
        }
        err /= refine_tol[C->tri_mat[e]];
        elem_error[e] = err;
        if (C->wd[e] > 0) elem_error[e] = 0.5;
    }
    for (i = 0; i < C->V; i++) node_error[i] /= (double) cnt[i];
    free(cnt);
}

/* ------------------------------------------------------------------------------ */
/* Wind (meteor_update, swind_elem2d_get_local_stress, src/structs/smeteor.c:241-300;
 * winds_proc_wu, src/meteor/winds_proc_wu.c:5-26): the nodal wind values stress_x/y (what
 * meteor_update puts in winds[node].stress) turned into a shear per the element's material
 * flag (0: the value itself, 1: Wu's drag law; the depth-dependent form 2 is not restated),
 * summed over the three vertices and scaled by windatt^2 / (3 density).  NULL stresses turn the
 * term off. */
static void wind_wu(double gravity, double xs, double ys, double *sx, double *sy) {
    double wmag = sqrt(pow(xs, 2.0) + pow(ys, 2.0) + 1e-10), x = xs, y = ys, cd;
    if (gravity > 10.) { wmag *= 0.3048; x *= 0.3048; y *= 0.3048; }
    cd = (0.8 + 0.065 * wmag) * .001;
    if (gravity > 10.) { *sx = 1.225 * cd * x * wmag * 0.020885; *sy = 1.225 * cd * y * wmag * 0.020885; }
    else { *sx = 1.225 * cd * x * wmag; *sy = 1.225 * cd * y * wmag; }
}
int orc_set_wind(orc_ctx *C, const int *mat_flag, const double *mat_windatt, const double *stress_x,
                 const double *stress_y) {
    int e, i;
    free(C->wsx); free(C->wsy);
    C->wsx = C->wsy = NULL;
    if (!stress_x || !stress_y) return 0;
    C->wsx = (double *) calloc((size_t) (C->T ? C->T : 1), sizeof(double));
    C->wsy = (double *) calloc((size_t) (C->T ? C->T : 1), sizeof(double));
    const double rho = C->p.density;
    for (e = 0; e < C->T; e++) {
        const int m = C->tri_mat[e];
        if (mat_flag[m] < 0 || mat_flag[m] > 1) return 1;
        double wx = 0., wy = 0.;
        for (i = 0; i < 3; i++) {
            const int n = C->tri[3 * e + i];
            double sx = 0., sy = 0.;
            if (rho > 0.0) {
                if (mat_flag[m] == 0) { sx = stress_x[n]; sy = stress_y[n]; }
                else wind_wu(C->p.gravity, stress_x[n], stress_y[n], &sx, &sy);
            }
            wx += sx;
            wy += sy;
        }
        const double f = pow(mat_windatt[m], 2.0) / (3 * rho);
        C->wsx[e] = wx * f;
        C->wsy[e] = wy * f;
    }
    return 0;
}

/* Wave radiation stress from nodal radiation stresses (swave_elem2d_get_local_stress,
 * src/structs/smeteor.c:312-327, the CSTORM_WSID OFF branch): per element
 * -sum_i (dphi_i/dx Sxx_i + dphi_i/dy Sxy_i), -sum_i (dphi_i/dx Sxy_i + dphi_i/dy Syy_i), in vertex
 * order.  NULL arrays: off. */
void orc_set_waves(orc_ctx *C, const double *rxx, const double *rxy, const double *ryy) {
    int e, i;
    free(C->wvx); free(C->wvy);
    C->wvx = C->wvy = NULL;
    if (!rxx || !rxy || !ryy) return;
    C->wvx = (double *) calloc((size_t) (C->T ? C->T : 1), sizeof(double));
    C->wvy = (double *) calloc((size_t) (C->T ? C->T : 1), sizeof(double));
    for (e = 0; e < C->T; e++) {
        double sx = 0., sy = 0.;
        for (i = 0; i < 3; i++) {
            const int n = C->tri[3 * e + i];
            const double gx = C->grad[6 * e + 2 * i], gy = C->grad[6 * e + 2 * i + 1];
            sx -= (gx * rxx[n] + gy * rxy[n]);
            sy -= (gx * rxy[n] + gy * ryy[n]);
        }
        C->wvx[e] = sx;
        C->wvy[e] = sy;
    }
}

/* ------------------------------------------------------------------------------ */
/* 2D constituent transport (src/fe/transport/), after an accepted SW2 step.
 * A general constituent (CN CON) moves with the water velocity: mfcf = 1 and vcf = 0
 * (scon_init, src/structs/scon.c:38-50), so the constituent velocity (vel + vcf) * mfcf of
 * fe_2d_transport_body_resid.c:183-187 is the water velocity.  Source/sink terms belong to
 * sediment only (:469-487); salinity, temperature (baroclinic coupling) and the vorticity
 * constituent are not restated. */

#define ORC_BCT_DIR 1                  /* define.h:375 */
#define ORC_BCT_NEU 3                  /* define.h:377 */
#define ORC_BCT_CEQ 36                 /* define.h:388 */

static double *TC(const orc_ctx *C, int t, int level) { return C->conc + ((size_t) 3 * t + level) * C->V; }

int orc_trn_setup(orc_ctx *C, int ntrn, const double *refc, const double *dm, const int *bc, const int *ser) {
    int k;
    free(C->trn_refc); free(C->trn_dm); free(C->trn_bc); free(C->trn_ser); free(C->conc); free(C->bcmask);
    free(C->tval); free(C->tres); free(C->tsol);
    C->ntrn = ntrn;
    C->trn_refc = (double *) dup(refc, sizeof(double) * ntrn);
    C->trn_dm = (double *) dup(dm, sizeof(double) * ntrn * C->M);
    C->trn_bc = (int *) dup(bc, sizeof(int) * ntrn * C->S);
    C->trn_ser = (int *) dup(ser, sizeof(int) * ntrn * C->S);
    C->conc = (double *) calloc((size_t) 3 * (ntrn ? ntrn : 1) * C->V, sizeof(double));
    C->bcmask = (int *) calloc(C->V, sizeof(int));
    C->tval = (double *) calloc(C->nnzb ? C->nnzb : 1, sizeof(double));
    C->tres = (double *) calloc(C->V, sizeof(double));
    C->tsol = (double *) calloc(C->V, sizeof(double));
    for (k = 0; k < ntrn * C->S; k++) {
        int f = C->trn_bc[k];
        if (f != 0 && f != ORC_BCT_DIR && f != ORC_BCT_NEU) return -1;
        if ((f == ORC_BCT_DIR || f == ORC_BCT_NEU) && (C->trn_ser[k] < 0 || C->trn_ser[k] >= C->NS)) return -1;
    }
    for (k = 0; k < ntrn; k++) if (!(C->trn_refc[k] != 0.0)) return -1;
    for (k = 0; k < ntrn; k++) {
        int e;
        for (e = 0; e < C->E; e++) if (C->trn_bc[k * C->S + C->edge_string[e]] == ORC_BCT_DIR) return -1;
    }
    return 0;
}
void orc_trn_set_conc(orc_ctx *C, int t, int level, const double *c) { memcpy(TC(C, t, level), c, sizeof(double) * C->V); }
void orc_trn_get_conc(const orc_ctx *C, int t, int level, double *c) { memcpy(c, TC(C, t, level), sizeof(double) * C->V); }
void orc_set_dacont(orc_ctx *C, const double *in) {   /* vertex-major [3][T], as orc_get_dacont */
    int i, e;
    for (i = 0; i < 3; i++) for (e = 0; e < C->T; e++) C->dacont[3 * e + i] = in[(size_t) i * C->T + e];
}
void orc_trn_get_bcmask(const orc_ctx *C, int *mask) { memcpy(mask, C->bcmask, sizeof(int) * C->V); }

static int trn_dirichlet(const orc_ctx *C, int t, int node) {
    int s = C->node_string[node];
    if (s <= SW2GPU_NORMAL) return 0;
    return C->trn_bc[t * C->S + s] == ORC_BCT_DIR || C->trn_bc[t * C->S + s] == ORC_BCT_CEQ;
}

/* fe_2d_trns_temporal (fe_2d_transport_body_resid.c:692-726): one level's wrapped temporal term
 * times dt_factor */
static void trn_temporal(const v2 *X, double djac, const double *hh, const double *cc, double dtf, double *er) {
    dof3 r[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    wd_args A = {X, hh, NULL, NULL, NULL, cc, djac, 1., 1.};
    int i;
    wd_wrapper(WD_TRN_TEMPORAL, r, &A, 1);
    for (i = 0; i < 3; i++) er[i] += dtf * r[i].c;
}

/* fe_2d_transport_body_resid (src/fe/transport/fe_2d_transport_body_resid.c:50-676), triangles;
 * pnode >= 0 perturbs the concentration of local node pnode by psign * eps (PERTURB_C) */
static void trn_body_resid(const orc_ctx *C, int t, int ie, double eps, int pnode, int psign, double *er) {
    const sw2gpu_params *P = &C->p;
    const int *nd = C->tri + 3 * ie;
    const double djac = C->djac[ie], dt = C->dt, alpha = P->tau_temporal, dll = P->drying_lower_limit;
    const v2 *g = (const v2 *) (C->grad + 6 * ie);
    const int imat = C->tri_mat[ie], wd = C->wd[ie];
    const double *c0 = TC(C, t, 0), *c1 = TC(C, t, 1), *c2 = TC(C, t, 2);
    double c[3], co[3], coo[3], h[3], ho[3], hoo[3], uc[3], vc[3];
    v2 X[3], vcon[3];
    int i;
    for (i = 0; i < 3; i++) {
        int n = nd[i];
        X[i].x = C->x[n]; X[i].y = C->y[n];
        c[i] = c0[n]; co[i] = c1[n]; coo[i] = c2[n];
        h[i] = C->h[0][n]; ho[i] = C->h[1][n]; hoo[i] = C->h[2][n];
        vcon[i].x = (C->u[0][n] + 0.0) * 1.0;               /* (vel + vcf) * mfcf (:183-187) */
        vcon[i].y = (C->v[0][n] + 0.0) * 1.0;
        uc[i] = vcon[i].x; vc[i] = vcon[i].y;
    }
    if (pnode >= 0) c[pnode] += psign * eps;                /* :171 */

    /* elemental averages and gradients (:207-222) */
    double c_avg = tri_f(1., 1., c), h_avg = tri_f(1., 1., h);
    double u_avg = tri_f(1., 1., uc), v_avg = tri_f(1., 1., vc);
    v2 gc = {0, 0}, gu = {0, 0}, gv = {0, 0};
    for (i = 0; i < 3; i++) { gc.x += c[i] * g[i].x; gc.y += c[i] * g[i].y; }
    for (i = 0; i < 3; i++) {
        gu.x += vcon[i].x * g[i].x; gu.y += vcon[i].x * g[i].y;
        gv.x += vcon[i].y * g[i].x; gv.y += vcon[i].y * g[i].y;
    }
    double vmag = sqrt(u_avg * u_avg + v_avg * v_avg);

    /* wet/dry factors and averages (:242-256).  fe_sw2_wd_average's integrand averages the
     * clipped depth whatever function it is given (fe_sw2_wet_dry_integrations.c:101-102), so
     * the second call, made for the concentration, returns the wet-area depth average too. */
    double factor = 1., h_wd = h_avg, c_wd = c_avg;
    v2 vwd = {u_avg, v_avg};
    if (wd != 0) {
        v2 unused;
        wd_average(X, h, vcon, djac, &h_wd, &vwd);
        wd_average(X, h, NULL, djac, &c_wd, &unused);
        factor = wd_factor(X, h, djac);
    }

    /* friction and diffusion coefficients (:258-290) */
    double h_fric = MAXD(h_avg, ORC_SMALL);
    double rough = roughness(C, imat, h_fric);
    double dxx = 0.0, dyy = 0.0, dxy = C->trn_dm[t * C->M + imat];
    if (C->mat_eev_mode[imat] != 0) {
        double st, tr;
        eevf(C->mat_eev_mode[imat], C->mat_eev_coef[imat], P->gravity, dll, h_fric, rough, djac, gu, gv, vmag, wd,
             &st, &tr);
        dxx = st; dxy = tr; dyy = st;
    }
    v2 vdir = {u_avg / MAXD(vmag, 1.E-8), v_avg / MAXD(vmag, 1.E-8)};   /* :293-295 */

    for (i = 0; i < 3; i++) er[i] = 0.0;
    /* temporal (:376-400) */
    trn_temporal(X, djac, h, c, (1. + alpha / 2.), er);
    trn_temporal(X, djac, ho, co, (-1.) * (1. + alpha), er);
    trn_temporal(X, djac, hoo, coo, (alpha / 2.), er);
    /* advection (:402-427) */
    {
        dof3 r[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        wd_args A = {X, h, g, NULL, vcon, c, djac, dt, -1.};
        wd_wrapper(WD_TRN_CONVECTION, r, &A, 1);
        for (i = 0; i < 3; i++) er[i] += r[i].c;
    }
    /* diffusion (:429-463), VT_2D_TENS2D_VECT2D_PROD_AI (macro.h:726-728) */
    {
        double factor_diff = MAXD(factor, .01);
        double depth = MAXD(h_wd, ORC_SMALL);
        double depth_diff = MAXD(depth, dll * .01);
        v2 flux;
        flux.x = dxx * vdir.x * (vdir.x * gc.x + vdir.y * gc.y) + dxy * gc.x;
        flux.y = dyy * vdir.y * (vdir.x * gc.x + vdir.y * gc.y) + dxy * gc.y;
        double r[3] = {0, 0, 0};
        tri_gradphi_dot_vbar(g, dt * depth_diff * factor_diff, djac, flux, r);
        for (i = 0; i < 3; i++) er[i] += r[i];
    }
    /* SUPG (:567-617): fe_get_supg_tau method 2 (fe_get_supg_tau.c:176-183) with the area
     * element length sqrt(area) (:285-290); the strong residual is the advection term alone */
    {
        double fn = sqrt(u_avg * u_avg + v_avg * v_avg);
        double le = sqrt(djac);
        double tau = (le / (fn + 2. * ORC_NQS)) * P->tau_pg;
        double conv = h_wd * (vwd.x * gc.x + vwd.y * gc.y);
        double strong = 0. + conv + factor * (0. + 0.);
        double r[3] = {0, 0, 0};
        tri_gradphi_dot_vbar(g, tau * dt * strong, djac, vwd, r);
        for (i = 0; i < 3; i++) er[i] += r[i];
    }
    /* the flow's extra continuity terms (:619-634) */
    for (i = 0; i < 3; i++) er[i] += c_wd * C->dacont[3 * ie + i];
    /* Dirichlet nodes (:641-660) */
    for (i = 0; i < 3; i++) if (trn_dirichlet(C, t, nd[i])) er[i] = 0.0;
}

static void line_phi_f_g(double djac, double c, const double *f, const double *g, double *I) {  /* elem1d:101-105 */
    double t1 = ONE_12 * djac * c;
    I[0] += t1 * ((3 * f[0] + f[1]) * g[0] + (f[0] + f[1]) * g[1]);
    I[1] += t1 * ((f[0] + f[1]) * g[0] + (f[0] + 3 * f[1]) * g[1]);
}

/* fe_2d_transport_boundary_resid (src/fe/transport/fe_2d_transport_boundary_resid.c:37-300) */
static void trn_edge_resid(const orc_ctx *C, int t, int ie, double eps, int pnode, int psign, double *er) {
    const int *nd = C->edges + 2 * ie;
    const int str = C->edge_string[ie], hflag = C->str_bc[str];
    const int cflag = C->trn_bc[t * C->S + str], cser = C->trn_ser[t * C->S + str];
    const double c_inv = 1. / C->trn_refc[t], dt = C->dt, djac = C->edjac[ie];
    const v2 n = {C->enrml[2 * ie], C->enrml[2 * ie + 1]};
    double c[2], h[2], vn[2];
    int i;
    for (i = 0; i < 2; i++) {
        int k = nd[i];
        c[i] = TC(C, t, 0)[k];
        h[i] = C->h[0][k];
        vn[i] = C->u[0][k] * n.x + C->v[0][k] * n.y;
    }
    if (pnode >= 0) c[pnode] += psign * eps;
    er[0] = er[1] = 0.0;
    if (hflag == SW2GPU_BCT_VEL_NEU) {                                  /* :186-214 */
        double flux = -1.0 * C->series[C->str_isigma[str]];
        if (flux < -ORC_SMALL) {
            /* con_bc_flag > NORMAL: only NB TRN (BCT_NEU) reaches here, setup refuses DB TRN on
             * edge strings, whose isigma the reference would read unset */
            if (cflag == ORC_BCT_NEU) line_phi(djac, C->series[cser] * c_inv * flux * dt, er);
        } else {
            line_phi_f(djac, flux * dt, c, er);
        }
    } else if (hflag == SW2GPU_BCT_OUTFLOW) {                           /* :216-231 */
        line_phi_f_g_h(djac, dt, vn[0], vn[1], h[0], h[1], c[0], c[1], er);
    } else if (hflag == SW2GPU_BCT_PRS_NEU) {                           /* :233-257 */
        double hf = 0.5 * (vn[0] * h[0] + vn[1] * h[1]);
        if (hf >= 0.) line_phi_f_g_h(djac, dt, vn[0], vn[1], h[0], h[1], c[0], c[1], er);
        else if (cflag == ORC_BCT_NEU) line_phi_f_g(djac, C->series[cser] * c_inv * dt, h, vn, er);
    }
    for (i = 0; i < 2; i++) {                                           /* :281-296 */
        if (h[i] < 0.0) er[i] = 0.0;
        if (trn_dirichlet(C, t, nd[i])) er[i] = 0.0;
    }
}

/* fe_transport_resid (src/fe/transport/fe_transport_resid.c:33-221): wet and partially wet
 * triangles (wd_flag 0 or 1), then the boundary edges; Dirichlet rows stay 0; entries below
 * SMALL are zeroed */
void orc_trn_resid(orc_ctx *C, int t, double *R) {
    int e, i;
    memset(C->tres, 0, sizeof(double) * C->V);
    for (e = 0; e < C->T; e++) {
        if (C->wd[e] != 0 && C->wd[e] != 1) continue;
        double er[3];
        trn_body_resid(C, t, e, 0., -1, 1, er);
        for (i = 0; i < 3; i++) { int n = C->tri[3 * e + i]; if (!C->bcmask[n]) C->tres[n] -= er[i]; }
    }
    for (e = 0; e < C->E; e++) {
        double er[2];
        trn_edge_resid(C, t, e, 0., -1, 1, er);
        for (i = 0; i < 2; i++) { int n = C->edges[2 * e + i]; if (!C->bcmask[n]) C->tres[n] -= er[i]; }
    }
    for (i = 0; i < C->V; i++) if (fabs(C->tres[i]) < ORC_SMALL) C->tres[i] = 0.0;
    if (R) memcpy(R, C->tres, sizeof(double) * C->V);
}

/* perturb_c's step (fe_transport_load.c:258-275): the node's concentration clamped to
 * [1, property[0]], NUM_DIFF_EPSILON_GENERAL with the fraction 0.1 (macro.h:676-680) */
static double trn_eps(double cn, double refc) {
    double ce = cn, e;
    if (ce < 1.0) ce = 1.0;
    if (ce > refc) ce = refc;
    e = fabs(ce) * (1. + 0.1);
    e -= fabs(ce);
    if (e < 0.1) e = 0.1;
    return e;
}

/* fe_transport_load (src/fe/transport/fe_transport_load.c:41-225) with perturb_c (:227-340):
 * central differences of every triangle (whatever its wd_flag) and edge, assembled by
 * fe_global_matrix_assemble_scalar (fe_assemble_matrix.c:51-138: entries of magnitude SMALL
 * or less are dropped), then diagonals below NOT_QUITE_SMALL raised to it
 * (check_matrix_diagonal_for_nonexistant_entries, tl_matrix.c:59-67) */
void orc_trn_load(orc_ctx *C, int t) {
    int e, i, j, k;
    const double *c = TC(C, t, 0), refc = C->trn_refc[t];
    memset(C->tval, 0, sizeof(double) * (size_t) C->nnzb);
    for (e = 0; e < C->T; e++) {
        double M[9];
        for (i = 0; i < 3; i++) {
            double eps = trn_eps(c[C->tri[3 * e + i]], refc), rp[3], rm[3];
            trn_body_resid(C, t, e, eps, i, +1, rp);
            trn_body_resid(C, t, e, eps, i, -1, rm);
            for (k = 0; k < 3; k++) M[i + 3 * k] = (rp[k] - rm[k]) / (2.0 * eps);   /* elem_matrix_deriv_1dof */
        }
        for (i = 0; i < 3; i++) for (j = 0; j < 3; j++) {
            double v = M[3 * i + j];
            if (fabs(v) > ORC_SMALL) C->tval[C->blk_of_pair[9 * e + 3 * i + j]] += v;
        }
    }
    for (e = 0; e < C->E; e++) {
        double M[4];
        for (i = 0; i < 2; i++) {
            double eps = trn_eps(c[C->edges[2 * e + i]], refc), rp[2], rm[2];
            trn_edge_resid(C, t, e, eps, i, +1, rp);
            trn_edge_resid(C, t, e, eps, i, -1, rm);
            for (k = 0; k < 2; k++) M[i + 2 * k] = (rp[k] - rm[k]) / (2.0 * eps);
        }
        for (i = 0; i < 2; i++) for (j = 0; j < 2; j++) {
            double v = M[2 * i + j];
            if (fabs(v) > ORC_SMALL) C->tval[C->eblk_of_pair[4 * e + 2 * i + j]] += v;
        }
    }
    for (i = 0; i < C->V; i++) {
        double *d = C->tval + find_blk(C, i, i);
        if (fabs(*d) < ORC_NQS) *d = ORC_NQS;
    }
}
void orc_trn_get_matrix(const orc_ctx *C, double *val, double *resid) {
    if (val) memcpy(val, C->tval, sizeof(double) * (size_t) C->nnzb);
    if (resid) memcpy(resid, C->tres, sizeof(double) * C->V);
}

/* fe_transport_init (src/fe/transport/fe_transport_init.c:24-116) */
void orc_trn_init(orc_ctx *C, int t) {
    double *c = TC(C, t, 0);
    const double *co = TC(C, t, 1), c_inv = 1. / C->trn_refc[t];
    int i;
    for (i = 0; i < C->V; i++) {
        if (isnan(c[i]) || isinf(c[i])) c[i] = 0.0;
        C->bcmask[i] = 0;
        c[i] = co[i];
        if (C->h[0][i] <= ORC_NQS) c[i] = 0.0;
    }
    for (i = 0; i < C->V; i++) {
        int s = C->node_string[i];
        if (s > SW2GPU_NORMAL && C->trn_bc[t * C->S + s] == ORC_BCT_DIR) {
            C->bcmask[i] = 1;
            c[i] = C->series[C->trn_ser[t * C->S + s]] * c_inv;
        }
    }
}

/* scalar banded LU of the spv_jacobi-scaled system in reverse Cuthill-McKee order: the exact
 * solve the reference's profile LU preconditioner gives its BiCGSTAB (one iteration) */
static int trn_linear_solve(orc_ctx *C, const double *rhs, double *x) {
    int V = C->V, i, k, r, c, j;
    double *S = (double *) malloc(sizeof(double) * V);
    for (i = 0; i < V; i++) {                            /* spv_jacobi: row max */
        double m = 0.0;
        for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) if (fabs(C->tval[k]) > m) m = fabs(C->tval[k]);
        S[i] = (m < ORC_SMALL) ? 1.0 / sqrt(ORC_SMALL) : 1.0 / sqrt(m);
    }
    int w = 0;
    for (i = 0; i < V; i++)
        for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) {
            int d = abs(C->iperm[i] - C->iperm[C->col[k]]);
            if (d > w) w = d;
        }
    int W = 2 * w + 1;
    double *B = (double *) calloc((size_t) V * W, sizeof(double)), *y = (double *) malloc(sizeof(double) * V);
    for (i = 0; i < V; i++) {
        int pi = C->iperm[i];
        for (k = C->rowptr[i]; k < C->rowptr[i + 1]; k++) {
            int pj = C->iperm[C->col[k]];
            B[(size_t) pi * W + (pj - pi + w)] = C->tval[k] * S[i] * S[C->col[k]];
        }
        y[pi] = rhs[i] * S[i];
    }
    for (r = 0; r < V; r++) {                            /* Doolittle, no pivoting */
        double piv = B[(size_t) r * W + w];
        if (piv == 0.0) piv = B[(size_t) r * W + w] = ORC_SMALL;
        int rend = r + w < V - 1 ? r + w : V - 1;
        for (j = r + 1; j <= rend; j++) {
            double *Rj = B + (size_t) j * W, l = Rj[r - j + w] / piv;
            if (l == 0.0) continue;
            Rj[r - j + w] = l;
            for (c = r + 1; c <= rend; c++) Rj[c - j + w] -= l * B[(size_t) r * W + (c - r + w)];
        }
    }
    for (r = 0; r < V; r++) {
        int c0 = r - w > 0 ? r - w : 0;
        double acc = y[r];
        for (c = c0; c < r; c++) acc -= B[(size_t) r * W + (c - r + w)] * y[c];
        y[r] = acc;
    }
    for (r = V - 1; r >= 0; r--) {
        int c1 = r + w < V - 1 ? r + w : V - 1;
        double acc = y[r];
        for (c = r + 1; c <= c1; c++) acc -= B[(size_t) r * W + (c - r + w)] * y[c];
        y[r] = acc / B[(size_t) r * W + w];
    }
    for (i = 0; i < V; i++) x[i] = y[C->iperm[i]] * S[i];
    free(S); free(B); free(y);
    return 1;
}

static void trn_norms(orc_ctx *C, double *rmax, double *rl2, double *imax) {   /* get_residual_norms, nsys 1 */
    int i;
    double l2 = 0, mx = 0, im = 0;
    for (i = 0; i < C->V; i++) {
        int inc = MIND(C->h[0][i], C->h[1][i]) > 0;        /* include_node_in_residual (fe_newton.c:177-188) */
        double r = C->tres[i], s = C->tsol[i];
        if (fabs(s) > im && inc) im = fabs(s);
        if (fabs(r) > mx && inc) mx = fabs(r);
        l2 += r * r;
    }
    *rmax = mx; *rl2 = sqrt(l2 / C->V); *imax = im;
}

static void trn_inc(orc_ctx *C, int t) {                    /* fe_transport_inc.c:24-61 */
    double *c = TC(C, t, 0);
    int i;
    for (i = 0; i < C->V; i++) c[i] += C->tsol[i];
}

/* fe_transport (fe_transport.c:58-74) for constituent t: level shift, then fe_newton with the
 * transport functions, whose linear-problem test keeps iterating while the residual max norm
 * exceeds tol_nonlin (fe_newton.c:817-823, :855-856).  Uses the flow's current levels, wd_flag,
 * dt, series values and side output as the last SW2 step left them. */
int orc_trn_step(orc_ctx *C, int t, sw2gpu_stats *st) {
    const sw2gpu_params *P = &C->p;
    int V = C->V, i, it = 0, lin_total = 0, cuts_total = 0, solv_ok = 1, isnan_flag = 0, keep;
    double rmax, rl2, imax, old_l2;
    memcpy(TC(C, t, 2), TC(C, t, 1), sizeof(double) * V);
    memcpy(TC(C, t, 1), TC(C, t, 0), sizeof(double) * V);
    memset(C->tsol, 0, sizeof(double) * V);
    orc_trn_init(C, t);
    orc_trn_resid(C, t, NULL);
    trn_norms(C, &rmax, &rl2, &imax);
    const int lin_test = P->tol_nonlin > ORC_SMALL;
    do {
        orc_trn_load(C, t);
        lin_total += trn_linear_solve(C, C->tres, C->tsol);
        trn_inc(C, t);
        for (i = 0; i < V; i++) C->tsol[i] = -C->tsol[i];
        old_l2 = rl2;
        orc_trn_resid(C, t, NULL);
        trn_norms(C, &rmax, &rl2, &imax);
        if (isnan(rl2) || isinf(rl2)) { solv_ok = 0; isnan_flag = 1; }
        int cuts = 0;
        while (rmax > P->tol_nonlin && rl2 > old_l2 && cuts < P->max_linesearch_cuts) {
            for (i = 0; i < V; i++) C->tsol[i] *= 0.5;
            trn_inc(C, t);
            orc_trn_resid(C, t, NULL);
            trn_norms(C, &rmax, &rl2, &imax);
            cuts++;
        }
        cuts_total += cuts;
        it++;
        keep = solv_ok && it < P->max_nonlin_it && rmax < 1.0E+20 && (lin_test && rmax > P->tol_nonlin);
    } while (keep);
    int rc = SW2GPU_OK;
    if (!solv_ok || (lin_test && rmax > P->tol_nonlin) || rmax >= 1.0E+20) {
        rc = isnan_flag ? SW2GPU_E_NAN : (!solv_ok ? SW2GPU_E_LINEAR : SW2GPU_E_NEWTON);
        orc_trn_init(C, t);
    }
    if (st) {
        memset(st, 0, sizeof(*st));
        st->status = rc; st->newton_its = it; st->linear_its = lin_total; st->linesearch_cuts = cuts_total;
        st->resid_max = rmax; st->resid_l2 = rl2; st->inc_max = imax;
    }
    return rc;
}

/* one element's transport residual, for checking the device physics element by element */
void orc_trn_body_resid(orc_ctx *C, int t, int ie, double eps, int pnode, int psign, double *out) {
    trn_body_resid(C, t, ie, eps, pnode, psign, out);
}
void orc_trn_edge_resid(orc_ctx *C, int t, int ie, double eps, int pnode, int psign, double *out) {
    trn_edge_resid(C, t, ie, eps, pnode, psign, out);
}

/* scon_calculate_elem2d_error (src/structs/scon.c:282-361): the constituents' adaption error
 * indicator at the current and old levels and the last dt.  Per element and constituent the
 * steady transport residual h (c - c_old) / dt + u h dc/dx + h c du/dx + h v dc/dy + h c dv/dy at
 * each vertex, less its element mean, as a root sum of squares times the area; elem_error[e]
 * (in/out, e.g. the flow's indicator first, as fe_main calls them, src/fe/fe_main.c:625-628) keeps
 * the largest of its value and every constituent's error over refine_tol[k * M + material];
 * node_error[k * V + n] (may be NULL) the constituent's element errors averaged over n's elements */
void orc_trn_elem_error(const orc_ctx *C, const double *refine_tol, double *elem_error, double *node_error) {
    int V = C->V, e, i, k;
    int *cnt = (int *) calloc(V, sizeof(int));
    double *nerr = (double *) calloc((size_t) (C->ntrn ? C->ntrn : 1) * V, sizeof(double));
    for (e = 0; e < C->T; e++) {
        const int *nd = C->tri + 3 * e;
        const v2 *g = (const v2 *) (C->grad + 6 * e);
        double hh[3], uu[3], vv[3], dudx = 0., dvdy = 0.;
        for (i = 0; i < 3; i++) { hh[i] = C->h[0][nd[i]]; uu[i] = C->u[0][nd[i]]; vv[i] = C->v[0][nd[i]]; }
        for (i = 0; i < 3; i++) {
            cnt[nd[i]] += 1;
            dudx += g[i].x * uu[i];
            dvdy += g[i].y * vv[i];
        }
        for (k = 0; k < C->ntrn; k++) {
            const double *c = TC(C, k, 0), *co = TC(C, k, 1);
            double cc[3], cp[3], dcdx = 0., dcdy = 0., coef[3], err;
            for (i = 0; i < 3; i++) { cc[i] = c[nd[i]]; cp[i] = co[nd[i]]; }
            for (i = 0; i < 3; i++) { dcdx += g[i].x * cc[i]; dcdy += g[i].y * cc[i]; }
            for (i = 0; i < 3; i++)
                coef[i] = hh[i] * (cc[i] - cp[i]) / C->dt + uu[i] * hh[i] * dcdx + hh[i] * cc[i] * dudx +
                          hh[i] * vv[i] * dcdy + hh[i] * cc[i] * dvdy;
            err = (1. / 3.) * (coef[0] + coef[1] + coef[2]);
            for (i = 0; i < 3; i++) { coef[i] -= err; coef[i] = coef[i] * coef[i]; }
            err = sqrt(coef[0] + coef[1] + coef[2]) * C->djac[e];
            for (i = 0; i < 3; i++) nerr[(size_t) k * V + nd[i]] += err;
            err /= refine_tol[k * C->M + C->tri_mat[e]];
            if (err > elem_error[e]) elem_error[e] = err;
        }
    }
    if (node_error)
        for (k = 0; k < C->ntrn; k++)
            for (i = 0; i < V; i++) node_error[(size_t) k * V + i] = nerr[(size_t) k * V + i] / cnt[i];
    free(cnt); free(nerr);
}
