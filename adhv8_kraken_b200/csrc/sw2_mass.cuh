// Mass-balance diagnostics of the SW2 grid (src/tools/tl_grid_mass.c): the water mass of a time
// level and the mass that crossed the boundary or entered through water sources in one step.
// The per-element and per-edge terms are plain functions of their vertices: the reduction
// kernels (k_mass_partial, k_mass_final) inline them, and compiled as host C++ they are checked
// against the oracle term by term.
#pragma once

#include "sw2_physics.cuh"

namespace sw2 {

// fe_3m2d_dry_wet_factornew (tl_grid_mass.c:289-346): the triangle clipped at its zero-depth
// line with "dry" meaning h < 0 (the solver's own clip uses h <= 0).  Returns the signed wet
// fraction and the number of dry vertices; a clipped corner below kSmall of the element counts
// as no clip (0 dry vertices, fraction 1, for one dry vertex; 3 and 0 for two).
__device__ __forceinline__ double mass_clip(const double* x, const double* y, const double* h, double djac,
                                            int& num_dry) {
    int total = 0, pass = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int dry = (h[i] < 0.0) ? 1 : 0;
        total += dry;
        pass += dry << i;
    }
    if (total == 3) { num_dry = 3; return 0.0; }
    if (total == 0) { num_dry = 0; return 1.0; }
    if (total != 1) pass = 7 - pass;
    const int only = pass / 2;    // the vertex alone on its side of the zero line
    const double ho = sel3(h, only), xo = sel3(x, only), yo = sel3(y, only);
    double cx[3], cy[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (i != only) {
            const double xsi = h[i] / (h[i] - ho);
            cx[i] = x[i] + xsi * (xo - x[i]);
            cy[i] = y[i] + xsi * (yo - y[i]);
        } else {
            cx[i] = x[i];
            cy[i] = y[i];
        }
    }
    const double cd = ((cx[1] - cx[0]) * (cy[2] - cy[0]) - (cy[1] - cy[0]) * (cx[2] - cx[0])) / 2.0;
    if (cd / djac < kSmall) {
        const int odd = total % 2;
        num_dry = odd == 1 ? 0 : 3;
        return (double)odd;
    }
    num_dry = total;
    double f = (double)((total >> 1) - (total % 2));
    f *= cd / djac;
    return f + ((f < 0) ? 1.0 : 0.0);
}

// integrate_triangle_f (src/fe/fe_elem2d_integrations.c:60): c times the integral of a linear field
__device__ __forceinline__ double tri_integral(double djac, double c, double f0, double f1, double f2) {
    return c * djac * (f0 + f1 + f2) / 3.0;
}

// Water mass of one triangle, density 1 (tl_find_grid_mass_elem2d, tl_grid_mass.c:44-82): the
// wet part, and with one dry vertex the dry corner's negative depth counted as positive mass.
__device__ __forceinline__ double elem_mass(const double* x, const double* y, const double* h, double djac) {
    int num_dry;
    const double factor = mass_clip(x, y, h, djac, num_dry);
    double eh[3] = {h[0], h[1], h[2]}, hneg[3] = {0.0, 0.0, 0.0};
    double f1 = factor, f2 = 0.0;
    if (num_dry == 1) {
#pragma unroll
        for (int i = 0; i < 3; i++)
            if (eh[i] < 0.0) hneg[i] = eh[i];
        f1 = 1.0;
        f2 = -1.0 * (1.0 - factor);
    } else if (num_dry == 2) {
#pragma unroll
        for (int i = 0; i < 3; i++)
            if (eh[i] < 0.0) { hneg[i] = eh[i]; eh[i] = 0.0; }
    }
    return tri_integral(djac, f1, eh[0], eh[1], eh[2]) + tri_integral(djac, f2, hneg[0], hneg[1], hneg[2]);
}

// Water a source element adds in one step (tl_find_grid_mass_error_elem2d, tl_grid_mass.c:114-130):
// the source rate over the element's wet part (fe_sw2_wet_dry_factor) times dt and density.
__device__ __forceinline__ double elem_source_mass(const double* x, const double* y, const double* h, double djac,
                                                   double rate, double dt, double density) {
    return rate * djac * dt * density * clip_factor(x, y, h, djac);
}

// Water leaving through one boundary edge in one step (tl_grid_mass.c:133-144): the integral of
// h v.n, integrate_line_h_f (src/fe/fe_elem1d_integrations.c:18), which the caller subtracts.
// djac0 is the length of the grid's first boundary edge, which the reference uses for every
// edge (:142-143).
__device__ __forceinline__ double edge_outflow_term(double djac0, double density, double dt, double h0, double h1,
                                                    double vn0, double vn1) {
    const double t1 = djac0 * kOne6 * (density * dt);
    return t1 * ((2 * vn0 + vn1) * h0 + (vn0 + 2 * vn1) * h1);
}

}  // namespace sw2
