// trn_physics.cuh -- device-side 2D constituent transport element physics for sm_100a.
//
// trn_elem_resid() evaluates AdH's fe_2d_transport_body_resid
// (src/fe/transport/fe_2d_transport_body_resid.c:50-676) for one linear triangle and
// trn_edge_resid() its fe_2d_transport_boundary_resid (fe_2d_transport_boundary_resid.c:37-300)
// for one boundary edge, for a general constituent carried by the water velocity (mfcf = 1,
// vcf = 0: scon_init, src/structs/scon.c:38-50; source and sink terms belong to sediment only).
// The wet/dry clipping is the SW2 one (wd_apply, make_clip of sw2_physics.cuh).
//
// GPU structure (not the reference's): everything an FD Jacobian column leaves unchanged -- the
// old and older temporal terms, the wet/dry averages of depth and velocity, the diffusion
// tensor, the flow direction and the SUPG tau -- is formed once per element (TrnPre) and the
// column's evaluations read it back; the terms are added in the reference's order, so a
// residual has the same bits however its parts were obtained.
#pragma once
#include "sw2_physics.cuh"

namespace sw2 {

constexpr int kTrnBctDir = 1;   // define.h:375 (DB TRN)
constexpr int kTrnBctNeu = 3;   // define.h:377 (NB TRN)
// the flow's edge kinds (DevMesh::bkind)
constexpr int kEdgeVel = 1;     // NB VEL, BCT_VEL_NEU
constexpr int kEdgeTailwater = 2;   // NB OTW, BCT_PRS_NEU
constexpr int kEdgeOutflow = 3; // NB OF, BCT_OUTFLOW
constexpr int kEdgeOvh = 4;     // NB OVH, BCT_OVH_NEU: no transport term

// model constants of a transport solve
struct TrnParams {
    double g, dll, alpha, tau_pg, dt;
};

// one triangle: geometry, the flow's three levels, the constituent's old levels, the flow's
// side output elem_rhs_dacont_extra_terms, wd_flag and the held (Dirichlet) vertices
struct TrnElem {
    double x[3], y[3], djac, gx[3], gy[3];
    double h[3], ho[3], hoo[3], u[3], v[3];
    double co[3], coo[3], dac[3];
    double ks, eev_coef, dm;    // material: roughness height, EEV coefficient, MP DF d_m
    int eev_mode, wd;
    unsigned dir;               // bit i: vertex i held
};

// the parts of the element residual that do not depend on the current concentration
struct TrnPre {
    double to[3], too[3];       // t(n) and t(n-1) temporal contributions
    double h_wd, vwx, vwy;      // wet-area averages of the depth and the velocity (full averages when wet)
    double factor;              // wet/dry factor of the current depth
    double dxx, dxy, dyy;       // diffusion tensor (MP DF or estimated eddy viscosity)
    double vdx, vdy;            // flow direction of the element-average velocity
    double tau;                 // SUPG tau (fe_get_supg_tau method 2, area element length)
};

// integrate_triangle_phi_f_g (fe_elem2d_integrations.c:281-287)
__device__ __forceinline__ void trn_phi_f_g(double djac, double c, const double* f, const double* g, double* I) {
    const double gs = 2 * (g[0] + g[1] + g[2]), t1 = c * djac * kOne60;
    I[0] += t1 * (f[0] * (gs + 4 * g[0]) + f[1] * (gs - g[2]) + f[2] * (gs - g[1]));
    I[1] += t1 * (f[1] * (gs + 4 * g[1]) + f[2] * (gs - g[0]) + f[0] * (gs - g[2]));
    I[2] += t1 * (f[2] * (gs + 4 * g[2]) + f[1] * (gs - g[0]) + f[0] * (gs - g[1]));
}
// integrate_triangle_gradPhi_dot_vbar (fe_elem2d_integrations.c:422)
__device__ __forceinline__ void trn_gradphi_dot_vbar(const double* gx, const double* gy, double djac, double c,
                                                     double vx, double vy, double* I) {
    const double t1 = c * djac;
#pragma unroll
    for (int i = 0; i < 3; i++) I[i] += t1 * (vx * gx[i] + vy * gy[i]);
}

// one level's temporal term (fe_2d_trns_temporal, :692-726, with the wrapped integrand
// fe_2d_transport_wd_temporal_triangle, fe_2d_transport_wet_dry_integrations.c:86-99), times dtf
__device__ __forceinline__ void trn_temporal(const double* x, const double* y, const double* h, const double* c,
                                             double djac, double dtf, double* out) {
    double r[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto integ = [&](const double* X, const double* Y, const double* H, const double*, const double*, double dj,
                     bool clipped, const Clip& cc, double (&q)[3][3]) {
        double cv[3], I[3] = {0, 0, 0};
#pragma unroll
        for (int i = 0; i < 3; i++) cv[i] = cval(cc, clipped, c, i);
        trn_phi_f_g(dj, 1. * 1., H, cv, I);
#pragma unroll
        for (int i = 0; i < 3; i++) q[i][0] += I[i];
    };
    wd_apply<false>(x, y, h, nullptr, nullptr, djac, 1, r, integ);
#pragma unroll
    for (int i = 0; i < 3; i++) out[i] = dtf * r[i][0];
}

__device__ __forceinline__ void trn_prepare(const TrnElem& E, const TrnParams& P, TrnPre& pre) {
    double uc[3], vc[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        uc[i] = (E.u[i] + 0.0) * 1.0;   // (vel + vcf) * mfcf (:183-187)
        vc[i] = (E.v[i] + 0.0) * 1.0;
    }
    trn_temporal(E.x, E.y, E.ho, E.co, E.djac, (-1.) * (1. + P.alpha), pre.to);
    trn_temporal(E.x, E.y, E.hoo, E.coo, E.djac, (P.alpha / 2.), pre.too);
    const double h_avg = avg3(E.h), u_avg = avg3(uc), v_avg = avg3(vc);
    double gux = 0, guy = 0, gvx = 0, gvy = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        gux += uc[i] * E.gx[i];
        guy += uc[i] * E.gy[i];
        gvx += vc[i] * E.gx[i];
        gvy += vc[i] * E.gy[i];
    }
    const double vmag = sqrt(u_avg * u_avg + v_avg * v_avg);
    pre.h_wd = h_avg;
    pre.vwx = u_avg;
    pre.vwy = v_avg;
    pre.factor = 1.0;
    if (E.wd != 0) pre.factor = wd_average<false>(E.x, E.y, E.h, uc, vc, E.djac, pre.h_wd, pre.vwx, pre.vwy);
    // diffusion (:258-290): MP DF on the transverse entry, or the estimated eddy viscosity
    const double h_fric = fmax(h_avg, kSmall);
    const double rough = (E.ks > kSmall) ? drag_coef(h_fric, E.ks) : 0.0;
    pre.dxx = 0.0;
    pre.dyy = 0.0;
    pre.dxy = E.dm;
    if (E.eev_mode != 0) {
        double st, tr;
        eev_coefficients(E.eev_mode, E.eev_coef, P.g, P.dll, h_fric, rough, E.djac, gux, guy, gvx, gvy, vmag, E.wd,
                         st, tr);
        pre.dxx = st;
        pre.dxy = tr;
        pre.dyy = st;
    }
    pre.vdx = u_avg / fmax(vmag, 1.E-8);   // :293-295
    pre.vdy = v_avg / fmax(vmag, 1.E-8);
    // fe_get_supg_tau method 2 (fe_get_supg_tau.c:176-183), le = sqrt(area) (:285-290)
    const double fn = sqrt(u_avg * u_avg + v_avg * v_avg);
    pre.tau = (sqrt(E.djac) / (fn + 2. * kNotQuiteSmall)) * P.tau_pg;
}

// The element residual at concentration c (perturbation applied), added term by term in the
// reference's order: temporal t(n+1), t(n), t(n-1); advection; diffusion; SUPG; the flow's extra
// continuity terms; held vertices zeroed.
__device__ __forceinline__ void trn_elem_resid(const TrnElem& E, const TrnPre& pre, const double* c,
                                               const TrnParams& P, double* er) {
    double uc[3], vc[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        uc[i] = (E.u[i] + 0.0) * 1.0;
        vc[i] = (E.v[i] + 0.0) * 1.0;
        er[i] = 0.0;
    }
    double tn[3];
    trn_temporal(E.x, E.y, E.h, c, E.djac, (1. + P.alpha / 2.), tn);
#pragma unroll
    for (int i = 0; i < 3; i++) er[i] += tn[i];
#pragma unroll
    for (int i = 0; i < 3; i++) er[i] += pre.to[i];
#pragma unroll
    for (int i = 0; i < 3; i++) er[i] += pre.too[i];
    // advection (:402-427): fe_2d_transport_wd_convection_triangle
    // (fe_2d_transport_wet_dry_integrations.c:39-48) with vars (dt, -1) under the wrapper
    {
        double r[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double cdt = P.dt * -1.;
        auto integ = [&](const double* X, const double* Y, const double* H, const double* GX, const double* GY,
                         double dj, bool clipped, const Clip& cc, double (&q)[3][3]) {
            double cv[3], uu[3], vv[3], b[3] = {0, 0, 0};
#pragma unroll
            for (int i = 0; i < 3; i++) {
                cv[i] = cval(cc, clipped, c, i);
                uu[i] = cval(cc, clipped, uc, i);
                vv[i] = cval(cc, clipped, vc, i);
            }
            // integrate_triangle_gradPhi_dot_f_g_v (fe_elem2d_integrations.c:571-587)
            trn_phi_f_g(dj, cdt, H, cv, b);
            const double ix = uu[0] * b[0] + uu[1] * b[1] + uu[2] * b[2];
            const double iy = vv[0] * b[0] + vv[1] * b[1] + vv[2] * b[2];
#pragma unroll
            for (int i = 0; i < 3; i++) q[i][0] += ix * GX[i] + iy * GY[i];
        };
        wd_apply<false>(E.x, E.y, E.h, E.gx, E.gy, E.djac, 1, r, integ);
#pragma unroll
        for (int i = 0; i < 3; i++) er[i] += r[i][0];
    }
    double gcx = 0, gcy = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        gcx += c[i] * E.gx[i];
        gcy += c[i] * E.gy[i];
    }
    // diffusion (:429-463) with VT_2D_TENS2D_VECT2D_PROD_AI (macro.h:726-728)
    {
        const double factor_diff = fmax(pre.factor, .01);
        const double depth = fmax(pre.h_wd, kSmall);
        const double depth_diff = fmax(depth, P.dll * .01);
        const double vd = pre.vdx * gcx + pre.vdy * gcy;
        const double fx = pre.dxx * pre.vdx * vd + pre.dxy * gcx;
        const double fy = pre.dyy * pre.vdy * vd + pre.dxy * gcy;
        double r[3] = {0, 0, 0};
        trn_gradphi_dot_vbar(E.gx, E.gy, P.dt * depth_diff * factor_diff, E.djac, fx, fy, r);
#pragma unroll
        for (int i = 0; i < 3; i++) er[i] += r[i];
    }
    // SUPG (:567-617): the strong residual is the advection term alone
    {
        const double conv = pre.h_wd * (pre.vwx * gcx + pre.vwy * gcy);
        const double strong = 0. + conv + pre.factor * (0. + 0.);
        double r[3] = {0, 0, 0};
        trn_gradphi_dot_vbar(E.gx, E.gy, pre.tau * P.dt * strong, E.djac, pre.vwx, pre.vwy, r);
#pragma unroll
        for (int i = 0; i < 3; i++) er[i] += r[i];
    }
    // the flow's extra continuity terms (:619-634); fe_sw2_wd_average's integrand averages the
    // clipped depth whatever it is given (fe_sw2_wet_dry_integrations.c:101-102), so in a partially
    // wet element the coefficient is the wet-area depth average, not the concentration's
    const double c_wd = (E.wd != 0) ? pre.h_wd : avg3(c);
#pragma unroll
    for (int i = 0; i < 3; i++) er[i] += c_wd * E.dac[i];
#pragma unroll
    for (int i = 0; i < 3; i++)
        if (E.dir & (1u << i)) er[i] = 0.0;   // :641-660
}

// one boundary edge (fe_2d_transport_boundary_resid.c:37-300)
struct TrnEdge {
    double djac, nx, ny;        // length and outward normal
    double h[2], u[2], v[2];    // the flow's current level
    int kind;                   // the edge's flow condition (kEdge*)
    int cflag;                  // its NB TRN flag for this constituent (0 or kTrnBctNeu)
    double flux_in;             // NB VEL: the step value of the string's unit-discharge series
    double c_user;              // NB TRN: the step value of its concentration series over property[0]
    unsigned dir;               // bit i: vertex i held
};

__device__ __forceinline__ void trn_edge_resid(const TrnEdge& B, const double* c, double dt, double* er) {
    double vn[2];
#pragma unroll
    for (int i = 0; i < 2; i++) vn[i] = B.u[i] * B.nx + B.v[i] * B.ny;
    er[0] = er[1] = 0.0;
    if (B.kind == kEdgeVel) {                   // BCT_VEL_NEU (:186-214)
        const double flux = -1.0 * B.flux_in;
        if (flux < -kSmall) {
            if (B.cflag == kTrnBctNeu) {        // integrate_line_phi
                const double t1 = 0.5 * B.djac * (B.c_user * flux * dt);
                er[0] += t1;
                er[1] += t1;
            }
        } else {                                // integrate_line_phi_f
            const double t1 = kOne6 * B.djac * (flux * dt);
            er[0] += t1 * (2 * c[0] + c[1]);
            er[1] += t1 * (c[0] + 2 * c[1]);
        }
    } else if (B.kind == kEdgeOutflow || B.kind == kEdgeTailwater) {   // :216-231, :233-257
        const double hf = 0.5 * (vn[0] * B.h[0] + vn[1] * B.h[1]);
        if (B.kind == kEdgeOutflow || hf >= 0.) {   // integrate_line_phi_f_g_h (elem1d:115-119)
            const double f1 = vn[0], f2 = vn[1], g1 = B.h[0], g2 = B.h[1], h1 = c[0], h2 = c[1];
            const double t1 = kOne60 * B.djac * dt;
            er[0] += t1 * ((3 * (4 * f1 + f2) * g1 + (3 * f1 + 2 * f2) * g2) * h1 +
                           ((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h2);
            er[1] += t1 * (((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h1 +
                           ((2 * f1 + 3 * f2) * g1 + 3 * (f1 + 4 * f2) * g2) * h2);
        } else if (B.cflag == kTrnBctNeu) {     // integrate_line_phi_f_g (elem1d:101-105)
            const double t1 = kOne12 * B.djac * (B.c_user * dt);
            er[0] += t1 * ((3 * B.h[0] + B.h[1]) * vn[0] + (B.h[0] + B.h[1]) * vn[1]);
            er[1] += t1 * ((B.h[0] + B.h[1]) * vn[0] + (B.h[0] + 3 * B.h[1]) * vn[1]);
        }
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {               // :281-296
        if (B.h[i] < 0.0) er[i] = 0.0;
        if (B.dir & (1u << i)) er[i] = 0.0;
    }
}

// perturb_c's step (fe_transport_load.c:258-275): the node's concentration clamped to
// [1, property[0]], NUM_DIFF_EPSILON_GENERAL with the fraction 0.1 (macro.h:676-680)
__device__ __forceinline__ double trn_eps(double cn, double refc) {
    double ce = cn;
    if (ce < 1.0) ce = 1.0;
    if (ce > refc) ce = refc;
    double e = fabs(ce) * (1. + 0.1);
    e -= fabs(ce);
    if (e < 0.1) e = 0.1;
    return e;
}

}  // namespace sw2
