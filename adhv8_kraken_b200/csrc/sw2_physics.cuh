// sw2_physics.cuh -- device-side SW2 element physics for sm_100a.
//
// One call of sw2_elem_resid() evaluates the 2D shallow-water element residual of
// AdH's fe_sw2_body_resid (src/fe/sw2/fe_sw2_body_resid.c:45-1267) for a linear
// triangle, in primitive variables (h, u, v), including the wet/dry clipping of
// fe_sw2_wet_dry_wrapper (src/fe/fe_sw2_wet_dry_wrapper.c:106-306).  The result is
// er[node][eq] with eq 0 = continuity (c_eq), 1 = x-momentum, 2 = y-momentum.
//
// GPU structure (not the reference's): the clipping geometry of the current depth
// is computed once per call and reused by every wet/dry-wrapped integrand (the
// reference re-clips for each of the ~8 wrapper calls); all loops over the three
// vertices are unrolled so the element lives in registers.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace sw2 {

constexpr double kSmall = 2.220446049250313e-16;        // DBL_EPSILON (define.h:27)
constexpr double kNotQuiteSmall = 1.1920928955078125e-07;  // FLT_EPSILON (define.h:28)
constexpr double kOne3 = 0.333333333333333333333333;
constexpr double kOne6 = 0.166666666666666666666667;
constexpr double kOne12 = 0.083333333333333333333333;
constexpr double kOne30 = 0.033333333333333333333333;
constexpr double kOne60 = 0.016666666666666666666667;

enum PerturbVar { kPertNone = -1, kPertU = 1, kPertV = 2, kPertH = 5 };

// Model constants of one instance (kernel parameter).
struct PhysParams {
    double g, dll, dul, alpha, tau_pg, dt;
};

// Per-material constants, precomputed on the host (sin() of the Coriolis latitude,
// EVS sums, the Manning roughness height) plus the step's water-source value.
struct MatParams {
    double ks;          // fterms.eqrheight (<= kSmall: no drag)
    double ev_st, ev_tr;// EVS: |xx - yy|, min(xx, yy) incl. molecular viscosity
    double eev_coef;
    double cor_speed;   // sin(lat) * 2 * EARTH_ROTAT
    double water_src;   // step-averaged source value when the string is BCT_WATER_SOURCE
    int eev_mode;       // 0 = EVS
    int has_source;
};

struct ElemIn {
    double x[3], y[3], z[3];
    double h[3], u[3], v[3];        // current iterate (perturbation applied)
    double ho[3], uo[3], vo[3];     // old time level
    double hoo[3], uoo[3], voo[3];  // older time level
    double djac, gx[3], gy[3];
    double wsx, wsy;                // wind surface stress of the element (0: none)
};

// a[k] for a runtime k in 0..2 as selects, so register arrays stay in registers
__device__ __forceinline__ double sel3(const double* a, int k) { return (k == 0) ? a[0] : ((k == 1) ? a[1] : a[2]); }

// ---------------------------------------------------------------------------------
// wet/dry clipping of one depth array (the geometric part of fe_sw2_wet_dry_wrapper)
struct Clip {
    int total, only, degenerate;
    double factor;      // (total >> 1) - (total % 2)
    double ret;         // value the wrapper returns
    double ndjac;
    double nx[3], ny[3], nh[3], xsi[3];
};

__device__ __forceinline__ void make_clip(const double* x, const double* y, const double* h, double djac, Clip& c) {
    int total = 0, pass = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        int dry = (h[i] <= 0.0) ? 1 : 0;
        total += dry;
        pass += dry << i;
    }
    c.total = total;
    c.degenerate = 0;
    c.only = 0;
    c.factor = 0.0;
    c.ndjac = djac;
    if (total == 3) { c.ret = 0.0; return; }
    if (total == 0) { c.ret = 1.0; return; }
    if (total != 1) pass = 7 - pass;
    int only = pass / 2;
    c.only = only;
    const double ho = sel3(h, only), xo = sel3(x, only), yo = sel3(y, only);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (i != only) {
            double xsi = h[i] / (h[i] - ho);
            c.xsi[i] = xsi;
            c.nx[i] = x[i] + xsi * (xo - x[i]);
            c.ny[i] = y[i] + xsi * (yo - y[i]);
            c.nh[i] = 0.0;
        } else {
            c.xsi[i] = 0.0;
            c.nx[i] = x[i];
            c.ny[i] = y[i];
            c.nh[i] = h[i];
        }
    }
    double nd = ((c.nx[1] - c.nx[0]) * (c.ny[2] - c.ny[0]) - (c.ny[1] - c.ny[0]) * (c.nx[2] - c.nx[0])) / 2.0;
    c.ndjac = nd;
    if (nd / djac < kSmall) {
        c.degenerate = 1;
        c.ret = (double)(total % 2);
        return;
    }
    double f = (double)((total >> 1) - (total % 2));
    c.factor = f;
    double fr = f * (nd / djac);
    c.ret = fr + ((fr < 0) ? 1.0 : 0.0);
}

// return value of the wrapper / fe_sw2_wet_dry_factor for a depth array
__device__ __forceinline__ double clip_factor(const double* x, const double* y, const double* h, double djac) {
    Clip c;
    make_clip(x, y, h, djac, c);
    return c.ret;
}

// Wraps an integrand the way fe_sw2_wet_dry_wrapper does: full element, and/or the
// clipped corner scaled by the signed factor, optionally redistributed (RE_DISTRIBUTE).
// The integrand functor is called as f(x, y, h, gx, gy, djac, vinterp, rhs[3][3]) where
// vinterp(i, w, v) returns the clipped value of a vertex quantity.
template <bool WET, class F>
__device__ __forceinline__ void wd_apply(const double* x, const double* y, const double* h,
                                         const double* gx, const double* gy, double djac, int redistribute,
                                         double (&rhs)[3][3], F&& f) {
    Clip c;
    if (WET) {             // caller guarantees h > 0 at every vertex: the wrapper's full-element case
        c.total = 0;
        c.only = 0;
        f(x, y, h, gx, gy, djac, false, c, rhs);
        return;
    }
    make_clip(x, y, h, djac, c);
    if (c.total == 3) return;
    if (c.total == 0 || c.total == 1) {
        f(x, y, h, gx, gy, djac, false, c, rhs);
        if (c.total == 0) return;
    }
    if (c.degenerate) return;
    double ngx[3], ngy[3];
    double nd = c.ndjac;
    ngx[0] = 0.5 * (c.ny[1] - c.ny[2]) / nd;
    ngx[1] = 0.5 * (c.ny[2] - c.ny[0]) / nd;
    ngx[2] = 0.5 * (c.ny[0] - c.ny[1]) / nd;
    ngy[0] = 0.5 * (c.nx[2] - c.nx[1]) / nd;
    ngy[1] = 0.5 * (c.nx[0] - c.nx[2]) / nd;
    ngy[2] = 0.5 * (c.nx[1] - c.nx[0]) / nd;
    double nr[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    f(c.nx, c.ny, c.nh, ngx, ngy, nd, true, c, nr);
    if (redistribute) {
        const int o = c.only;
        const double xo = sel3(x, o), yo = sel3(y, o);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            if (i == o) continue;
            double ax = c.nx[i] - xo, ay = c.ny[i] - yo;
            double bx = x[i] - xo, by = y[i] - yo;
            double xs = sqrt((ax * ax + ay * ay) / (bx * bx + by * by));
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const double add = (1.0 - xs) * nr[i][q];
#pragma unroll
                for (int t = 0; t < 3; t++)
                    if (t == o) nr[t][q] += add;
                nr[i][q] *= xs;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int q = 0; q < 3; q++) rhs[i][q] += c.factor * nr[i][q];
}

// clipped value of a vertex quantity (FIXED_POS with the clip weights)
__device__ __forceinline__ double cval(const Clip& c, bool clipped, const double* f, int i) {
    if (!clipped || i == c.only) return f[i];
    return f[i] + c.xsi[i] * (sel3(f, c.only) - f[i]);
}

// wetted-area averages (fe_sw2_wd_average, src/fe/sw2/fe_sw2_wet_dry_integrations.c:19-39):
// returns the wrapper factor and writes the averaged depth and velocity.
template <bool WET>
__device__ __forceinline__ double wd_average(const double* x, const double* y, const double* h,
                                             const double* u, const double* v, double djac, double& havg,
                                             double& uavg, double& vavg) {
    double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto integ = [&](const double* X, const double* Y, const double* H, const double*, const double*, double dj,
                     bool clipped, const Clip& cc, double (&r)[3][3]) {
        double t1 = (H[0] + H[1] + H[2]) / 3.0;
        double t2 = (cval(cc, clipped, u, 0) + cval(cc, clipped, u, 1) + cval(cc, clipped, u, 2)) / 3.0;
        double t3 = (cval(cc, clipped, v, 0) + cval(cc, clipped, v, 1) + cval(cc, clipped, v, 2)) / 3.0;
        r[0][0] += dj * t1;
        r[0][1] += dj * t2;
        r[0][2] += dj * t3;
    };
    wd_apply<WET>(x, y, h, nullptr, nullptr, djac, 0, acc, integ);
    const double f = WET ? 1.0 : clip_factor(x, y, h, djac);
    havg = 0.0;
    uavg = 0.0;
    vavg = 0.0;
    if (f > 0.0) {
        double wet = djac * f;
        havg = acc[0][0] / wet;
        uavg = acc[0][1] / wet;
        vavg = acc[0][2] / wet;
    }
    return f;
}

__device__ __forceinline__ double drag_coef(double depth, double ks) {  // fr_bedshstr_drag_coef.c:18-40
    depth = fmax(depth, 1.E-8);
    ks = fmax(ks, 1.E-8);
    double rh = (ks > 29.7 * depth) ? 1. / 29.7 : depth / ks;
    double bta = 29.7 * rh;
    double t = (.4 * bta) / ((bta + 1) * (log(bta + 1) - 1) + 1);
    return 2. * (t * t);
}

// estimated eddy viscosity of mode 1..3 (fe_sw2_get_EEVF, src/fe/sw2/fe_sw2_get_EEVF.c:33-60):
// streamwise and transverse coefficients from the friction depth, the drag coefficient, the
// element area, the velocity gradients and the average speed
__device__ __forceinline__ void eev_coefficients(int mode, double coef, double g, double dll, double h_fric,
                                                 double rough, double area, double gux, double guy, double gvx,
                                                 double gvy, double vmag, int wd_flag, double& ev_st, double& ev_tr) {
    const double vmin = 0.1 * sqrt(g * dll);
    double evmin;
    if (mode == 1) {
        ev_st = 0.0;
        ev_tr = coef * 2.0 * h_fric * sqrt(rough) * vmag;
        evmin = (coef / 0.5) * vmin * sqrt(area) / 40.;
    } else if (mode == 2) {
        ev_st = 1.3 * h_fric * sqrt(rough) * vmag;
        ev_tr = coef * 0.92 * h_fric * sqrt(rough) * vmag;
        evmin = (coef / 0.5) * vmin * sqrt(area) / 40.;
    } else {
        ev_st = 0.;
        ev_tr = coef * coef * area * sqrt(gux * gux + gvy * gvy + 0.5 * (guy + gvx) * (guy + gvx));
        evmin = (coef / 0.2) * vmin * sqrt(area) / 40.;
    }
    ev_tr = fmax(ev_tr, evmin);
    if (wd_flag == 1 || wd_flag == 2) {
        ev_st = 0.0;
        ev_tr = fmax(ev_tr, 5. * evmin);
    }
}

// ---------------------------------------------------------------------------------
// Parts of the fully wet residual that depend on one part of the iterate only.  An FD
// Jacobian column perturbs one variable at one vertex, so what depends only on the old
// levels, only on the depth or only on the velocity is shared by many of an element's 18
// perturbed evaluations: the Jacobian kernel forms those parts once per element (wet_levels,
// wet_depth, wet_pre_velocity) and the evaluations read them back.  Each part is formed by
// the same function either way, so the residual has the same bits however a part was obtained.
__device__ __forceinline__ double dot3(const double* f, const double* g) {
    double s = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) s += f[i] * g[i];
    return s;
}
__device__ __forceinline__ double avg3(const double* f) { return (f[0] + f[1] + f[2]) / 3.0; }
// integral of a vertex quantity over the (fully wet) element, as the wrapped integrands form it
__device__ __forceinline__ double wet_integral(const double* f, double djac) { return 0.0 + djac * avg3(f); }
// temporal term of one level (fe_sw2_temporal :1288-1354) with the wet/dry factor 1
__device__ __forceinline__ void wet_temporal(const double* H, const double* U, const double* V, double djac, double dtf,
                                             double dll, bool cont, double (&c)[3][3]) {
    const double fs = H[0] + H[1] + H[2], t1 = djac * dtf * kOne12;
    const double con = dtf * 1.0;
    const double t2 = djac * con * kOne3;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (cont) c[i][0] = 0.0 + t1 * (fs + H[i]);
        c[i][1] = t2 * (U[i] * fmax(H[i], dll));
        c[i][2] = t2 * (V[i] * fmax(H[i], dll));
    }
}

struct WetLevels {              // old and older levels
    double gzx, gzy, le, d0[3]; // d0: minus the old-level integrals of h, u, v (SUPG)
    double to[3][3], too[3][3]; // t(n) and t(n-1) temporal contributions [vertex][eq]
};
struct WetDepth {               // current depth
    double ghx, ghy, hint, h_wd, rough, resistance, tnc[3];
};
struct WetVel {                 // one current velocity component
    double avg, gx, gy, vint, wd;
};
struct WetPre {
    WetLevels L;
    WetDepth D;
    WetVel U, V;
    double vmag, vst_i, vst_j, vwd_mag;     // both velocity components
    double fx[3], fy[3];                    // per-vertex friction fluxes
};
// which parts an evaluation leaves unchanged: kFixH / kFixU / kFixV, and vertex i's velocity
// unchanged at bit kFixNode + i
enum WetFix : unsigned { kFixH = 1u, kFixU = 2u, kFixV = 4u, kFixNode = 3 };

__device__ __forceinline__ void wet_levels(const ElemIn& in, const PhysParams& P, WetLevels& L) {
    L.gzx = dot3(in.z, in.gx);
    L.gzy = dot3(in.z, in.gy);
    L.le = sqrt(in.djac * 1.0);
    L.d0[0] = -wet_integral(in.ho, in.djac);
    L.d0[1] = -wet_integral(in.uo, in.djac);
    L.d0[2] = -wet_integral(in.vo, in.djac);
    wet_temporal(in.ho, in.uo, in.vo, in.djac, (-1.) * (1. + P.alpha), P.dll, true, L.to);
    if (P.alpha != 0.0) wet_temporal(in.hoo, in.uoo, in.voo, in.djac, P.alpha / 2., P.dll, true, L.too);
}
__device__ __forceinline__ void wet_depth(const ElemIn& in, const double* hc, const PhysParams& P, const MatParams& M,
                                          WetDepth& D) {
    D.ghx = dot3(hc, in.gx);
    D.ghy = dot3(hc, in.gy);
    D.hint = wet_integral(hc, in.djac);
    D.h_wd = D.hint / in.djac;
    const double h_fric = fmax(D.h_wd, kSmall);
    D.rough = (M.ks > kSmall) ? drag_coef(h_fric, M.ks) : 0.0;
    D.resistance = D.rough / (2.0 * P.g);
    double c[3][3];
    wet_temporal(hc, hc, hc, in.djac, 1. + P.alpha / 2., P.dll, true, c);
#pragma unroll
    for (int i = 0; i < 3; i++) D.tnc[i] = c[i][0];
}
__device__ __forceinline__ void wet_vel(const ElemIn& in, const double* f, WetVel& W) {
    W.avg = avg3(f);
    W.gx = dot3(f, in.gx);
    W.gy = dot3(f, in.gy);
    W.vint = wet_integral(f, in.djac);
    W.wd = W.vint / in.djac;
}
__device__ __forceinline__ void flow_dir(double ua, double va, double& vmag, double& vi, double& vj) {
    vmag = sqrt(ua * ua + va * va);
    vi = ua / fmax(vmag, 1.E-8);
    vj = va / fmax(vmag, 1.E-8);
}
__device__ __forceinline__ void friction_flux(double u, double v, double& fx, double& fy) {
    const double m = sqrt(u * u + v * v);
    fx = u * m;
    fy = v * m;
}
__device__ __forceinline__ void wet_pre_velocity(const ElemIn& in, WetPre& p) {
    wet_vel(in, in.u, p.U);
    wet_vel(in, in.v, p.V);
    flow_dir(p.U.avg, p.V.avg, p.vmag, p.vst_i, p.vst_j);
    p.vwd_mag = sqrt(p.U.wd * p.U.wd + p.V.wd * p.V.wd);
#pragma unroll
    for (int i = 0; i < 3; i++) friction_flux(in.u[i], in.v[i], p.fx[i], p.fy[i]);
}

// ---------------------------------------------------------------------------------
// the element residual
//   in:       the element's static data and old / older levels (may live in shared memory)
//   hc,uc,vc: the current iterate at the three vertices, perturbation applied (registers)
//   wd_flag:  element wet/dry flag of the Newton solve (fe_sw2_wdflag)
//   pvar:     kPertNone / kPertU / kPertV / kPertH (u, v perturbations drop the pressure terms)
//   dflag[3]: Dirichlet flags of the element's nodes (bit0 PRS_DIR, bit1 VEL_DIR, bit2 VEL_PRS_DIR)
//   PRE:      (fully wet only) the parts named by `fix` are read from `pre` (see WetPre)
//   dac[3]:   when given, receives the continuity parts of shock capturing and SUPG per vertex, the
//             side output elem_rhs_dacont_extra_terms that transport reads (:353-355, :400, :1214)
template <bool WET, bool PRE = false>
__device__ __forceinline__ void elem_resid_impl(const ElemIn& in, const double* hc, const double* uc, const double* vc,
                                                int wd_flag, int pvar, const PhysParams& P, const MatParams& M,
                                                const int* dflag, double (&er)[3][3], const WetPre* pre = nullptr,
                                                unsigned fix = 0u, double* dac = nullptr) {
    static_assert(WET || !PRE, "precomputed parts exist for fully wet elements only");
    const double djac = in.djac, dt = P.dt, g = P.g, dll = P.dll, dul = P.dul;
    const double* gx = in.gx;
    const double* gy = in.gy;
    const bool pressure = !(pvar == kPertU || pvar == kPertV);
    const bool fh = PRE && (fix & kFixH), fu = PRE && (fix & kFixU), fv = PRE && (fix & kFixV);

    // averages and gradients (:193-221)
    WetDepth D;
    WetVel Uw, Vw;
    if (fu) Uw = pre->U;
    else wet_vel(in, uc, Uw);
    if (fv) Vw = pre->V;
    else wet_vel(in, vc, Vw);
    const double u_avg = Uw.avg, v_avg = Vw.avg;
    const double gux = Uw.gx, guy = Uw.gy, gvx = Vw.gx, gvy = Vw.gy;
    double gzx, gzy, ghx, ghy;
    if (PRE) {
        gzx = pre->L.gzx;
        gzy = pre->L.gzy;
    } else {
        gzx = dot3(in.z, gx);
        gzy = dot3(in.z, gy);
    }
    if (WET) {
        if (fh) D = pre->D;
        else wet_depth(in, hc, P, M, D);
        ghx = D.ghx;
        ghy = D.ghy;
    } else {
        ghx = dot3(hc, gx);
        ghy = dot3(hc, gy);
    }
    const double gwx = gzx + ghx, gwy = gzy + ghy;
    double vmag, vst_i, vst_j;
    if (fu && fv) {
        vmag = pre->vmag;
        vst_i = pre->vst_i;
        vst_j = pre->vst_j;
    } else {
        flow_dir(u_avg, v_avg, vmag, vst_i, vst_j);
    }

    double h_wd, u_wd, v_wd, factor, factor_old, factor_older, vwd_mag, rough;
    if (WET) {      // the wrapper's full-element case: factors 1, wetted-area averages
        h_wd = D.h_wd;
        u_wd = Uw.wd;
        v_wd = Vw.wd;
        factor = factor_old = factor_older = 1.0;
        vwd_mag = (fu && fv) ? pre->vwd_mag : sqrt(u_wd * u_wd + v_wd * v_wd);
        rough = D.rough;
    } else {
        factor = wd_average<WET>(in.x, in.y, hc, uc, vc, djac, h_wd, u_wd, v_wd);
        factor_old = clip_factor(in.x, in.y, in.ho, djac);
        factor_older = clip_factor(in.x, in.y, in.hoo, djac);
        vwd_mag = sqrt(u_wd * u_wd + v_wd * v_wd);
        rough = (M.ks > kSmall) ? drag_coef(fmax(h_wd, kSmall), M.ks) : 0.0;
    }
    const double h_fric = fmax(h_wd, kSmall);

    // eddy viscosity (:263-291, fe_sw2_get_EEVF.c:33-60)
    double ev_st, ev_tr;
    if (M.eev_mode == 0) {
        ev_st = M.ev_st;
        ev_tr = M.ev_tr;
    } else {
        eev_coefficients(M.eev_mode, M.eev_coef, g, dll, h_fric, rough, djac, gux, guy, gvx, gvy, vmag, wd_flag,
                         ev_st, ev_tr);
    }

#pragma unroll
    for (int i = 0; i < 3; i++) er[i][0] = er[i][1] = er[i][2] = 0.0;
    if (dac) dac[0] = dac[1] = dac[2] = 0.0;

    // shock capturing, partially/fully dry elements (:357-400)
    if (!WET && (wd_flag == 1 || wd_flag == 2)) {
        const double gum = sqrt(gux * gux + guy * guy + kSmall);
        const double gvm = sqrt(gvx * gvx + gvy * gvy + kSmall);
        const double cu = 0.5 * dul * djac * gum, cv = 0.5 * dul * djac * gvm;
        const double unx = gux / gum, uny = guy / gum, vnx = gvx / gvm, vny = gvy / gvm;
        const double nx = unx * gux + uny * guy, ny = vnx * gvx + vny * gvy;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const double rc = dt * 0.5 * g * djac * ((dll * gwx) * gx[i] + (dll * gwy) * gy[i]);
            er[i][0] += rc;
            if (dac) dac[i] += rc;
            er[i][1] += cu * dt * djac * nx * (unx * gx[i] + uny * gy[i]);
            er[i][2] += cv * dt * djac * ny * (vnx * gx[i] + vny * gy[i]);
        }
    }

    // advection, wet/dry wrapped with redistribution (:434-457, fe_sw2_wd_convection_triangle)
    {
        double rhs[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double cc = -dt;
        auto integ = [&](const double*, const double*, const double* H, const double* GX, const double* GY,
                         double dj, bool clipped, const Clip& c, double (&r)[3][3]) {
            double uu[3], vv[3];
#pragma unroll
            for (int i = 0; i < 3; i++) {
                uu[i] = cval(c, clipped, uc, i);
                vv[i] = cval(c, clipped, vc, i);
            }
            // integrate_triangle_gradPhi_dot_f_v
            double p1 = 2 * H[0] + H[1] + H[2], p2 = H[0] + 2 * H[1] + H[2], p3 = H[0] + H[1] + 2 * H[2];
            double tx = p1 * uu[0] + p2 * uu[1] + p3 * uu[2];
            double ty = p1 * vv[0] + p2 * vv[1] + p3 * vv[2];
            double con = dj * kOne12 * cc;
            // integrate_triangle_dphi_f_g_h(f = u, g = v, h): x-derivative -> y-momentum
            double ff1 = 3 * uu[0] + uu[1] + uu[2], ff2 = 2 * uu[0] + 2 * uu[1] + uu[2], ff3 = 2 * uu[0] + uu[1] + 2 * uu[2];
            double ff4 = uu[0] + 3 * uu[1] + uu[2], ff5 = uu[0] + 2 * uu[1] + 2 * uu[2], ff6 = uu[0] + uu[1] + 3 * uu[2];
            double gg1 = 2 * ff1 * vv[0] + ff2 * vv[1] + ff3 * vv[2];
            double gg2 = ff2 * vv[0] + 2 * ff4 * vv[1] + ff5 * vv[2];
            double gg3 = ff3 * vv[0] + ff5 * vv[1] + 2 * ff6 * vv[2];
            double cuv = dj * kOne60 * cc * (gg1 * H[0] + gg2 * H[1] + gg3 * H[2]);
            // integrate_triangle_dphi_f_f_h for u (x) and v (y)
            double a0 = uu[0] * uu[0], a1 = uu[1] * uu[1], a2 = uu[2] * uu[2];
            double q1 = 3 * a0 + 2 * uu[0] * uu[1] + a1 + (2 * uu[0] + uu[1]) * uu[2] + a2;
            double q2 = a0 + 2 * uu[0] * uu[1] + 3 * a1 + (uu[0] + 2 * uu[1]) * uu[2] + a2;
            double q3 = a0 + uu[0] * uu[1] + a1 + 2 * (uu[0] + uu[1]) * uu[2] + 3 * a2;
            double cuu = dj * kOne30 * cc * (q1 * H[0] + q2 * H[1] + q3 * H[2]);
            double b0 = vv[0] * vv[0], b1 = vv[1] * vv[1], b2 = vv[2] * vv[2];
            double s1 = 3 * b0 + 2 * vv[0] * vv[1] + b1 + (2 * vv[0] + vv[1]) * vv[2] + b2;
            double s2 = b0 + 2 * vv[0] * vv[1] + 3 * b1 + (vv[0] + 2 * vv[1]) * vv[2] + b2;
            double s3 = b0 + vv[0] * vv[1] + b1 + 2 * (vv[0] + vv[1]) * vv[2] + 3 * b2;
            double cvv = dj * kOne30 * cc * (s1 * H[0] + s2 * H[1] + s3 * H[2]);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                r[i][0] += con * (GX[i] * tx + GY[i] * ty);
                double rx = cuv * GY[i];
                double ry = cuv * GX[i];
                rx += cuu * GX[i];
                ry += cvv * GY[i];
                r[i][1] += rx;
                r[i][2] += ry;
            }
        };
        wd_apply<WET>(in.x, in.y, hc, gx, gy, djac, 1, rhs, integ);
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int q = 0; q < 3; q++) er[i][q] += rhs[i][q];
    }

    // temporal terms t(n+1), t(n), t(n-1) (:481-490, fe_sw2_temporal :1288-1354)
    if (WET) {
        auto add = [&](const double (&c)[3][3], bool cont) {
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int q = 0; q < 3; q++)
                    if (q > 0 || cont) er[i][q] += c[i][q];
        };
        double c[3][3];
        wet_temporal(hc, uc, vc, djac, 1. + P.alpha / 2., dll, false, c);
#pragma unroll
        for (int i = 0; i < 3; i++) c[i][0] = D.tnc[i];
        add(c, true);
        // the old levels' continuity part is dropped for wet/dry flag 2, as in the wrapped form
        if (PRE) {
            add(pre->L.to, wd_flag != 2);
            if (P.alpha != 0.0) add(pre->L.too, wd_flag != 2);
        } else {
            WetLevels L;
            wet_levels(in, P, L);
            add(L.to, wd_flag != 2);
            if (P.alpha != 0.0) add(L.too, wd_flag != 2);
        }
    } else {
        auto temporal = [&](const double* H, const double* U, const double* V, double wdf, double dtf, int flag) {
            double rhs[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            auto integ = [&](const double*, const double*, const double* Hc, const double*, const double*, double dj,
                             bool, const Clip&, double (&r)[3][3]) {
                double fs = Hc[0] + Hc[1] + Hc[2], t1 = dj * dtf * kOne12;
#pragma unroll
                for (int i = 0; i < 3; i++) r[i][0] += t1 * (fs + Hc[i]);
            };
            wd_apply<WET>(in.x, in.y, H, nullptr, nullptr, djac, 1, rhs, integ);
            const double con = dtf * wdf;
            const double t1 = djac * con * kOne3;
#pragma unroll
            for (int i = 0; i < 3; i++) {
                if (flag != 2) er[i][0] += rhs[i][0];
                er[i][1] += t1 * (U[i] * fmax(H[i], dll));
                er[i][2] += t1 * (V[i] * fmax(H[i], dll));
            }
        };
        temporal(hc, uc, vc, factor, 1. + P.alpha / 2., -3);
        temporal(in.ho, in.uo, in.vo, factor_old, (-1.) * (1. + P.alpha), wd_flag);
        if (P.alpha != 0.0)  // the t(n-1) term has weight alpha / 2
            temporal(in.hoo, in.uoo, in.voo, factor_older, P.alpha / 2., wd_flag);
    }

    // diffusion (:504-534)
    {
        const double tmp = (h_wd < dul) ? dul : h_wd;
        const double fxx = 2. * ev_st * vst_i * (vst_i * gux + vst_j * guy) + 2. * ev_tr * gux;
        const double fxy = ev_st * vst_j * (vst_j * guy + vst_i * gux + vst_i * gvx + vst_j * gvy) + ev_tr * (guy + gvx);
        const double fyx = ev_st * vst_i * (vst_j * guy + vst_i * gux + vst_i * gvx + vst_j * gvy) + ev_tr * (guy + gvx);
        const double fyy = 2. * ev_st * vst_j * (vst_j * gvy + vst_i * gvx) + 2. * ev_tr * gvy;
        const double t1 = tmp * djac, t2 = dt * factor;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            er[i][1] += t2 * (t1 * (fxx * gx[i] + fxy * gy[i]));
            er[i][2] += t2 * (t1 * (fyx * gx[i] + fyy * gy[i]));
        }
    }

    // bottom friction (:557-577)
    const double resistance = WET ? D.resistance : rough / (2.0 * g);
    {
        double fx[3], fy[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            if (PRE && ((fix >> (kFixNode + i)) & 1u)) {
                fx[i] = pre->fx[i];
                fy[i] = pre->fy[i];
            } else {
                friction_flux(uc[i], vc[i], fx[i], fy[i]);
            }
        }
        const double t1 = djac * (dt * g * resistance * factor) * kOne12;
        const double sx = fx[0] + fx[1] + fx[2], sy = fy[0] + fy[1] + fy[2];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            er[i][1] += t1 * (sx + fx[i]);
            er[i][2] += t1 * (sy + fy[i]);
        }
    }
    const double bedx = resistance * u_wd * vwd_mag, bedy = resistance * v_wd * vwd_mag;

    // Coriolis (:639-652)
    const double cs = M.cor_speed;
    if (cs != 0.0) {
        const double t1 = dt * factor * cs;
        auto phifg = [&](double c, const double* f, const double* gg, int q) {
            double gs = 2 * (gg[0] + gg[1] + gg[2]), tt = c * djac * kOne60;
            er[0][q] += tt * (f[0] * (gs + 4 * gg[0]) + f[1] * (gs - gg[2]) + f[2] * (gs - gg[1]));
            er[1][q] += tt * (f[1] * (gs + 4 * gg[1]) + f[2] * (gs - gg[0]) + f[0] * (gs - gg[2]));
            er[2][q] += tt * (f[2] * (gs + 4 * gg[2]) + f[1] * (gs - gg[0]) + f[0] * (gs - gg[1]));
        };
        phifg(-t1, hc, vc, 1);
        phifg(+t1, hc, uc, 2);
    }

    // wind surface stress, fully wet elements only (:674-719; no wave stress).  A zero stress
    // would subtract +0.0 from every entry, which changes no bits, so it is skipped.
    if (wd_flag == 0 && (in.wsx != 0.0 || in.wsy != 0.0)) {
        const double tx = in.wsx * djac * kOne3, ty = in.wsy * djac * kOne3;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            er[i][1] -= dt * tx;
            er[i][2] -= dt * ty;
        }
    }

    // rainfall / water source (:728-754)
    const double water_source = M.has_source ? M.water_src : 0.0;
    if (M.has_source) {
        const double rc = water_source * djac * kOne3;
#pragma unroll
        for (int i = 0; i < 3; i++) er[i][0] -= dt * factor * rc;
    }

    // pressure, bed slope and boundary pressure (:761-862), skipped for u/v perturbations
    if (pressure) {
        auto accum = [&](double (&rhs)[3][3]) {
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int q = 0; q < 3; q++) er[i][q] += rhs[i][q];
        };
        double rhs[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double cp = -0.5 * g * dt;
        auto ipress = [&](const double*, const double*, const double* H, const double* GX, const double* GY, double dj,
                          bool, const Clip&, double (&r)[3][3]) {
            double ff = cp * kOne6 * dj * (H[0] * H[0] + H[0] * H[1] + H[1] * H[1] + H[0] * H[2] + H[1] * H[2] + H[2] * H[2]);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                r[i][1] += GX[i] * ff;
                r[i][2] += GY[i] * ff;
            }
        };
        wd_apply<WET>(in.x, in.y, hc, gx, gy, djac, 1, rhs, ipress);
        accum(rhs);
        double rhs2[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double cb = g * dt;
        auto ibody = [&](const double*, const double*, const double* H, const double*, const double*, double dj, bool,
                         const Clip&, double (&r)[3][3]) {
            double sh = H[0] + H[1] + H[2];
            double cx = dj * kOne12 * cb * gzx, cy = dj * kOne12 * cb * gzy;
#pragma unroll
            for (int i = 0; i < 3; i++) {
                r[i][1] += cx * (sh + H[i]);
                r[i][2] += cy * (sh + H[i]);
            }
        };
        wd_apply<WET>(in.x, in.y, hc, nullptr, nullptr, djac, 1, rhs2, ibody);
        accum(rhs2);
        double rhs3[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double cq = 0.5 * dt * g;
        auto ibound = [&](const double* X, const double* Y, const double* H, const double*, const double*, double, bool,
                          const Clip&, double (&r)[3][3]) {
#pragma unroll
            for (int e = 0; e < 3; e++) {
                const int n1 = e, n2 = (e + 1) % 3;
                double delx = X[n1] - X[n2], dely = Y[n2] - Y[n1];
                double t1 = kOne12 * cq;
                double r0 = t1 * (3 * H[n1] * H[n1] + 2 * H[n1] * H[n2] + H[n2] * H[n2]);
                double r1 = t1 * (H[n1] * H[n1] + 2 * H[n1] * H[n2] + 3 * H[n2] * H[n2]);
                r[n1][1] += dely * r0;
                r[n2][1] += dely * r1;
                r[n1][2] += delx * r0;
                r[n2][2] += delx * r1;
            }
        };
        wd_apply<WET>(in.x, in.y, hc, nullptr, nullptr, djac, 1, rhs3, ibound);
        accum(rhs3);
    }

    // SUPG (:987-1232)
    if (!(fabs(h_wd) < kSmall)) {
        const double gf = g;
        const double hden = fmax(h_wd, kNotQuiteSmall);
        const double le = PRE ? pre->L.le : sqrt(djac * factor_old);
        double c2 = gf * hden;
        if (hden <= 0.0) c2 = 0.;
        const double sr = sqrt(u_wd * u_wd + v_wd * v_wd + c2 + kSmall);
        const double tau = P.tau_pg * le / sr;
        // elementally averaged wet/dry time derivatives (wrapped fe_sw2_wd_integrate_triangle_f)
        double dhdt, dudt, dvdt;
        if (WET) {
            double d0[3];
            if (PRE) {
                d0[0] = pre->L.d0[0];
                d0[1] = pre->L.d0[1];
                d0[2] = pre->L.d0[2];
            } else {
                d0[0] = -wet_integral(in.ho, djac);
                d0[1] = -wet_integral(in.uo, djac);
                d0[2] = -wet_integral(in.vo, djac);
            }
            dhdt = d0[0] + D.hint;
            dudt = d0[1] + Uw.vint;
            dvdt = d0[2] + Vw.vint;
        } else {
            {
                double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                auto integ = [&](const double*, const double*, const double* H, const double*, const double*, double dj,
                                 bool clipped, const Clip& c, double (&r)[3][3]) {
                    r[0][0] += dj * ((H[0] + H[1] + H[2]) / 3.0);
                    r[0][1] += dj * ((cval(c, clipped, in.uo, 0) + cval(c, clipped, in.uo, 1) + cval(c, clipped, in.uo, 2)) / 3.0);
                    r[0][2] += dj * ((cval(c, clipped, in.vo, 0) + cval(c, clipped, in.vo, 1) + cval(c, clipped, in.vo, 2)) / 3.0);
                };
                wd_apply<WET>(in.x, in.y, in.ho, nullptr, nullptr, djac, 0, acc, integ);
                dhdt = -acc[0][0];
                dudt = -acc[0][1];
                dvdt = -acc[0][2];
            }
            {
                double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                auto integ = [&](const double*, const double*, const double* H, const double*, const double*, double dj,
                                 bool clipped, const Clip& c, double (&r)[3][3]) {
                    r[0][0] += dj * ((H[0] + H[1] + H[2]) / 3.0);
                    r[0][1] += dj * ((cval(c, clipped, uc, 0) + cval(c, clipped, uc, 1) + cval(c, clipped, uc, 2)) / 3.0);
                    r[0][2] += dj * ((cval(c, clipped, vc, 0) + cval(c, clipped, vc, 1) + cval(c, clipped, vc, 2)) / 3.0);
                };
                wd_apply<WET>(in.x, in.y, hc, nullptr, nullptr, djac, 0, acc, integ);
                dhdt += acc[0][0];
                dudt += acc[0][1];
                dvdt += acc[0][2];
            }
        }
        factor = WET ? 1.0 : clip_factor(in.x, in.y, hc, djac);
        double adv[3] = {0, 0, 0};
        {
            double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            auto integ = [&](const double*, const double*, const double*, const double* GX, const double* GY, double dj,
                             bool clipped, const Clip& c, double (&r)[3][3]) {
                double f0 = cval(c, clipped, hc, 0), f1 = cval(c, clipped, hc, 1), f2 = cval(c, clipped, hc, 2);
                double u0 = cval(c, clipped, uc, 0), u1 = cval(c, clipped, uc, 1), u2 = cval(c, clipped, uc, 2);
                double v0 = cval(c, clipped, vc, 0), v1 = cval(c, clipped, vc, 1), v2 = cval(c, clipped, vc, 2);
                double ha = kOne3 * (f0 + f1 + f2), ua = kOne3 * (u0 + u1 + u2), va = kOne3 * (v0 + v1 + v2);
                double dhdx = GX[0] * f0 + GX[1] * f1 + GX[2] * f2;
                double dhdy = GY[0] * f0 + GY[1] * f1 + GY[2] * f2;
                double dudx = GX[0] * u0 + GX[1] * u1 + GX[2] * u2;
                double dudy = GY[0] * u0 + GY[1] * u1 + GY[2] * u2;
                double dvdx = GX[0] * v0 + GX[1] * v1 + GX[2] * v2;
                double dvdy = GY[0] * v0 + GY[1] * v1 + GY[2] * v2;
                r[0][0] += dj * dt * 1.0 * (ua * dhdx + ha * dudx + va * dhdy + ha * dvdy);
                r[0][1] += dj * dt * 1.0 * (ua * dudx + va * dudy);
                r[0][2] += dj * dt * 1.0 * (ua * dvdx + va * dvdy);
            };
            wd_apply<WET>(in.x, in.y, hc, gx, gy, djac, 0, acc, integ);
            adv[0] = acc[0][0];
            adv[1] = acc[0][1];
            adv[2] = acc[0][2];
        }
        const double xp = gf * (ghx + gzx) * dt * factor;
        const double yp = gf * (ghy + gzy) * dt * factor;
        const double xf = g * bedx * dt * factor, yf = g * bedy * dt * factor;
        const double xc = -v_wd * cs, yc = u_wd * cs;
        const double c_eq = dhdt + adv[0] + factor * water_source * djac * dt;
        // the surface stress of a fully wet element enters the strong momentum equations
        // (:1049-1050).  Without one the reference subtracts 0 / hden, which changes no bits, so
        // the division is skipped (it would cost an FP64 divide in every FD column evaluation).
        const double tsx = wd_flag == 0 ? in.wsx : 0.0, tsy = wd_flag == 0 ? in.wsy : 0.0;
        const double xs = tsx != 0.0 ? xc - tsx / hden : xc, ys = tsy != 0.0 ? yc - tsy / hden : yc;
        const double x_eq = dudt + adv[1] + (xp + xf / hden) * djac + xs * djac * factor * dt;
        const double y_eq = dvdt + adv[2] + (yp + yf / hden) * djac + ys * djac * factor * dt;
        const double tu = tau * u_wd, tv = tau * v_wd, th = tau * h_wd;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const double rc = gx[i] * (tu * c_eq + th * x_eq) + gy[i] * (tv * c_eq + th * y_eq);
            er[i][0] += rc;
            if (dac) dac[i] += rc;
            er[i][1] += gx[i] * (tau * gf * h_wd * c_eq + tu * h_wd * x_eq) + gy[i] * (tv * h_wd * x_eq);
            er[i][2] += gy[i] * (tau * gf * h_wd * c_eq + tv * h_wd * y_eq) + gx[i] * (tu * h_wd * y_eq);
        }
    }

    // Dirichlet nodes (:1239-1256)
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int f = dflag[i];
        if (f & 1) er[i][0] = 0.0;
        if (f & 2) { er[i][1] = 0.0; er[i][2] = 0.0; }
        if (f & 4) { er[i][0] = 0.0; er[i][1] = 0.0; er[i][2] = 0.0; }
    }
}

// general path (some vertex dry at some level, or a wet/dry-flagged element): out of line,
// so the fully wet path below is not charged the clipping code's registers
__device__ __noinline__ void elem_resid_general(const ElemIn& in, const double* hc, const double* uc, const double* vc,
                                                int wd_flag, int pvar, const PhysParams& P, const MatParams& M,
                                                const int* dflag, double (&er)[3][3]) {
    elem_resid_impl<false>(in, hc, uc, vc, wd_flag, pvar, P, M, dflag, er);
}

// the same with the transport side output; a function of its own, so the kernels that never
// ask for that output keep their code
__device__ __noinline__ void elem_resid_general_dac(const ElemIn& in, const double* hc, const double* uc,
                                                    const double* vc, int wd_flag, int pvar, const PhysParams& P,
                                                    const MatParams& M, const int* dflag, double (&er)[3][3],
                                                    double* dac) {
    elem_resid_impl<false>(in, hc, uc, vc, wd_flag, pvar, P, M, dflag, er, nullptr, 0u, dac);
}

__device__ __forceinline__ void sw2_elem_resid(const ElemIn& in, const double* hc, const double* uc, const double* vc,
                                               int wd_flag, int pvar, const PhysParams& P, const MatParams& M,
                                               const int* dflag, double (&er)[3][3], double* dac = nullptr) {
    const bool wet = wd_flag == 0 && hc[0] > 0.0 && hc[1] > 0.0 && hc[2] > 0.0 && in.ho[0] > 0.0 &&
                     in.ho[1] > 0.0 && in.ho[2] > 0.0 && in.hoo[0] > 0.0 && in.hoo[1] > 0.0 && in.hoo[2] > 0.0;
    if (wet)
        elem_resid_impl<true>(in, hc, uc, vc, wd_flag, pvar, P, M, dflag, er, nullptr, 0u, dac);
    else if (dac)
        elem_resid_general_dac(in, hc, uc, vc, wd_flag, pvar, P, M, dflag, er, dac);
    else
        elem_resid_general(in, hc, uc, vc, wd_flag, pvar, P, M, dflag, er);
}

// ---------------------------------------------------------------------------------
// boundary edge residual (fe_sw2_boundary_resid, src/fe/sw2/fe_sw2_boundary_resid.c:72-510)
// kind: 1 = BCT_VEL_NEU, 2 = BCT_PRS_NEU, 3 = BCT_OUTFLOW, 4 = BCT_OVH_NEU.
// Returns er[node][eq] (eq 0 = c, 1 = x, 2 = y).
struct EdgeIn {
    double h[2], u[2], v[2];
    double nx, ny, djac;
    double z0, z1;              // bed elevations of the edge's two nodes
    double bvx, bvy;            // NB OVH: the string's velocity series values (unused by other kinds)
};

__device__ __forceinline__ void line_phi_f_g_h(double djac, double c, double f1, double f2, double g1, double g2,
                                               double h1, double h2, double& i0, double& i1) {
    const double t1 = kOne60 * djac * c;
    i0 += t1 * ((3 * (4 * f1 + f2) * g1 + (3 * f1 + 2 * f2) * g2) * h1 + ((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h2);
    i1 += t1 * (((3 * f1 + 2 * f2) * g1 + (2 * f1 + 3 * f2) * g2) * h1 + ((2 * f1 + 3 * f2) * g1 + 3 * (f1 + 4 * f2) * g2) * h2);
}

// One boundary edge's residual.  kind 1: NB VEL explicit flow, `value` the unit discharge; 2: NB OTW tailwater, `value` the
// water elevation; 3: NB OF free outflow; 4: NB OVH, `value` the water elevation and
// (in.bvx, in.bvy) the prescribed velocity.
__device__ __forceinline__ void sw2_edge_resid(const EdgeIn& in, int kind, double value, int pvar, const PhysParams& P,
                                               const int* dflag, double (&er)[2][3]) {
    const bool pressure = !(pvar == kPertU || pvar == kPertV);
    const double djac = in.djac, dt = P.dt, g = P.g, nx = in.nx, ny = in.ny;
    double h_avg = 0.5 * (in.h[0] + in.h[1]);
    if (h_avg < kSmall) h_avg = kSmall;
#pragma unroll
    for (int i = 0; i < 2; i++) er[i][0] = er[i][1] = er[i][2] = 0.0;
    const double h0 = in.h[0], h1 = in.h[1];
    // depth-weighted normal flux h v.n tested with the edge's linear functions (fe_sw2_1d_*)
    auto normal_flux = [&](double& rc0, double& rc1) {
        const double t1 = djac * kOne12;
        rc0 = t1 * (nx * ((3 * h0 + h1) * in.u[0] + (h0 + h1) * in.u[1]) + ny * ((3 * h0 + h1) * in.v[0] + (h0 + h1) * in.v[1]));
        rc1 = t1 * (nx * ((h0 + h1) * in.u[0] + (h0 + 3 * h1) * in.u[1]) + ny * ((h0 + h1) * in.v[0] + (h0 + 3 * h1) * in.v[1]));
    };
    // fe_sw2_1d_implicit_flow (:637-): flow with the current velocity, outflow components only
    // in the momentum fluxes
    auto implicit_flow = [&]() {
        double ur0 = in.u[0], ur1 = in.u[1], vr0 = in.v[0], vr1 = in.v[1];
        if (in.u[0] * nx + in.v[0] * ny < kSmall) { ur0 = 0.; vr0 = 0.; }
        if (in.u[1] * nx + in.v[1] * ny < kSmall) { ur1 = 0.; vr1 = 0.; }
        double rc0, rc1;
        normal_flux(rc0, rc1);
        double rx0 = 0, rx1 = 0, ry0 = 0, ry1 = 0;
        line_phi_f_g_h(djac, nx, ur0, ur1, in.u[0], in.u[1], h0, h1, rx0, rx1);
        line_phi_f_g_h(djac, ny, vr0, vr1, in.v[0], in.v[1], h0, h1, ry0, ry1);
        line_phi_f_g_h(djac, ny, ur0, ur1, in.v[0], in.v[1], h0, h1, rx0, rx1);
        line_phi_f_g_h(djac, nx, vr0, vr1, in.u[0], in.u[1], h0, h1, ry0, ry1);
        er[0][0] += dt * rc0; er[1][0] += dt * rc1;
        er[0][1] += dt * rx0; er[1][1] += dt * rx1;
        er[0][2] += dt * ry0; er[1][2] += dt * ry1;
    };
    // fe_sw2_1d_pressure twice (:773-): the outside water column (d0, d1) minus the inside one
    auto boundary_pressure = [&](double d0, double d1) {
        double tt = djac * kOne12;
        double p0 = tt * (3 * d0 * d0 + 2 * d0 * d1 + d1 * d1), p1 = tt * (d0 * d0 + 2 * d0 * d1 + 3 * d1 * d1);
        double c1 = dt * 0.5 * g;
        er[0][1] += c1 * nx * p0; er[1][1] += c1 * nx * p1;
        er[0][2] += c1 * ny * p0; er[1][2] += c1 * ny * p1;
        p0 = tt * (3 * h0 * h0 + 2 * h0 * h1 + h1 * h1);
        p1 = tt * (h0 * h0 + 2 * h0 * h1 + 3 * h1 * h1);
        c1 = dt * 0.5 * (-g);
        er[0][1] += c1 * nx * p0; er[1][1] += c1 * nx * p1;
        er[0][2] += c1 * ny * p0; er[1][2] += c1 * ny * p1;
    };
    if (kind == 1) {                       // explicit flow (:562-604)
        const double flux = -1.0 * value;
        const double rc = 0.5 * djac;
        double rx0, rx1, ry0, ry1;
        if (flux < 0) {
            double us = 0., vs = 0.;
            if (h_avg > 0) { us = flux * nx / h_avg; vs = flux * ny / h_avg; }
            rx0 = rx1 = 0.5 * djac * us;
            ry0 = ry1 = 0.5 * djac * vs;
        } else {
            const double t1 = kOne6 * djac;
            rx0 = t1 * (2 * in.u[0] + in.u[1]); rx1 = t1 * (in.u[0] + 2 * in.u[1]);
            ry0 = t1 * (2 * in.v[0] + in.v[1]); ry1 = t1 * (in.v[0] + 2 * in.v[1]);
        }
        const double t1 = dt * flux;
        er[0][0] += t1 * rc; er[1][0] += t1 * rc;
        er[0][1] += t1 * rx0; er[1][1] += t1 * rx1;
        er[0][2] += t1 * ry0; er[1][2] += t1 * ry1;
    } else if (kind == 2 || kind == 3) {   // tailwater (:360-397) and free outflow (:227-240)
        double d0 = 0.0, d1 = 0.0;
        if (kind == 2) {
            d0 = value - in.z0;
            d1 = value - in.z0;             // both depths from node 0 (:375-376)
            if (d0 < kSmall || d1 < kSmall || h0 < kSmall || h1 < kSmall) return;
        }
        implicit_flow();
        if (kind == 2 && pressure) boundary_pressure(d0, d1);
    } else if (kind == 4) {                // elevation and velocity (:398-440)
        // each node's own bed here; an elevation below the bed stops the reference's run
        // (tl_error), the residual is evaluated as written
        const double d0 = value - in.z0, d1 = value - in.z1;
        if (in.bvx * nx + in.bvy * ny < -kSmall) {   // inflow: fe_sw2_1d_hvel (:882-897)
            double rc0, rc1;
            normal_flux(rc0, rc1);
            er[0][0] += dt * rc0; er[1][0] += dt * rc1;
            er[0][1] += dt * rc0 * in.bvx; er[1][1] += dt * rc1 * in.bvx;
            er[0][2] += dt * rc0 * in.bvy; er[1][2] += dt * rc1 * in.bvy;
        } else {
            implicit_flow();
        }
        if (pressure) boundary_pressure(d0, d1);
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int f = dflag[i];
        if (f & 1) er[i][0] = 0.0;
        if (f & 2) { er[i][1] = 0.0; er[i][2] = 0.0; }
        if (f & 4) { er[i][0] = 0.0; er[i][1] = 0.0; er[i][2] = 0.0; }
    }
}

// NUM_DIFF_EPSILON (src/include/macro.h:669-673)
__device__ __forceinline__ double fd_eps(double var) {
    const double p = 1.4901161193847656e-08;  // sqrt(DBL_EPSILON)
    double e = fabs(var) * (1. + p);
    e -= fabs(var);
    if (e < p) e = p;
    return e;
}

}  // namespace sw2
