/* Observation harness for the reference AdH executable (test infrastructure only).
 *
 * The reference's own objects are linked unmodified; the linker option
 * ``--wrap=fe_main --wrap=fe_sw2_load --wrap=fe_transport_load`` routes the calls made by the
 * time loop (src/main/adh_func.c:549) and by the Newton driver (src/fe/fe_newton.c:454)
 * through the functions below, which call the originals and then append
 * full-precision records to the binary file named by the environment variable
 * ADH_DUMP:
 *
 *   "step"   after every accepted time step: t_prev, dt, the wall time of the
 *            step's fe_main calls, Newton iterations of the step (including failed
 *            attempts), the number of attempts, and the nodal head / vel.x / vel.y /
 *            wd_flag arrays;
 *   "load"   for the first ADH_DUMP_LOADS calls of fe_sw2_load: the state the
 *            Jacobian was built at (three time levels), the residual vector,
 *            the 3x3 diagonal blocks and every off-diagonal SPARSE_VECT row;
 *   "mass"   when ADH_DUMP_MASS is set, after every accepted step (right after its
 *            "step" records): the reference's mass diagnostics of src/tools/tl_grid_mass.c
 *            -- the initial grid mass (tl_find_grid_mass_elem2d before the first step),
 *            the current grid mass, tl_find_grid_mass_error_elem2d and its accumulated
 *            boundary / source mass flux;
 *   "dacont" when ADH_DUMP_DACONT is set, after every accepted step (after "mass"): the
 *            side output sw->d2->elem_rhs_dacont_extra_terms[3][nelems2d], vertex-major;
 *   "elemerr", "nodeerr" when ADH_DUMP_ERROR is set, after every accepted step (after
 *            "dacont"): the adaption error indicator fe_main computed for the step
 *            (ssw_2d_calculate_elem_error, src/structs/ssw_2d.c:424-500), grid->elem_error
 *            per element and its nodal average sw->error.
 *   "conerr" with "elemerr", for every constituent: its nodal error indicator con[k].error
 *            (scon_calculate_elem2d_error, src/structs/scon.c:282-361), whose element values
 *            fe_main folds into grid->elem_error after the flow's (src/fe/fe_main.c:625-628);
 *   "con"    after every accepted step of a model with constituents (after the records
 *            above): each constituent's concentration array, constituent by constituent;
 *   "tload"  for the first ADH_DUMP_TLOADS calls of fe_transport_load (the transport Newton's
 *            Jacobian, src/fe/transport/fe_transport_load.c:41): the constituent, t_prev and
 *            dt, the three concentration levels, the flow's three levels, wd_flag, the side
 *            output elem_rhs_dacont_extra_terms, bc_mask, then the residual vector, the scalar
 *            diagonal and every off-diagonal SPARSE_VECT row (one value per entry).
 *
 * Record layout: char tag[8]; int32 kind (0 = f64, 1 = i32); int64 count; data.
 */
#include "global_header.h"
#include <time.h>

int __real_fe_main(SSUPER_MODEL *sm);
void __real_fe_sw2_load(SSUPER_MODEL *sm, int imod);
void __real_fe_transport_load(SSUPER_MODEL *sm, int imod);
/* the reference's mass diagnostics (src/tools/tl_grid_mass.c:20, :102); their prototypes are
 * commented out in its headers (src/include/fnctn.h:176-178) */
double tl_find_grid_mass_elem2d(double density, STR_VALUE *str, SSERIES *series_head, double *depth, SGRID *grid,
                                SFLAGS flags);
double tl_find_grid_mass_error_elem2d(double density, double *depth, SVECT2D *vel, SGRID *grid, SFLAGS flags,
                                      double initial_grid_mass, SSERIES *series_head, STR_VALUE *str, double dt,
                                      double *total_time_mass_flux_T);

static FILE *dump_fp = NULL;
static int dump_loads_left = -1;
static int dump_tloads_left = -1;
static int attempts = 0;
static int it_mark = 0;
static double solve_seconds = 0.0;   /* fe_main wall time since the last accepted step */
static int dump_mass = 0;            /* ADH_DUMP_MASS set */
static int dump_dacont = 0;          /* ADH_DUMP_DACONT set */
static int dump_error = 0;           /* ADH_DUMP_ERROR set */
static int mass_ready = 0;
static double mass0 = 0.0, mass_flux_total = 0.0;

static double now_seconds(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}

static void dump_open(void) {
    if (dump_fp != NULL) return;
    const char *path = getenv("ADH_DUMP");
    if (path == NULL) return;
    dump_fp = fopen(path, "wb");
    const char *nl = getenv("ADH_DUMP_LOADS");
    dump_loads_left = nl ? atoi(nl) : 0;
    const char *nt = getenv("ADH_DUMP_TLOADS");
    dump_tloads_left = nt ? atoi(nt) : 0;
    dump_mass = getenv("ADH_DUMP_MASS") != NULL;
    dump_dacont = getenv("ADH_DUMP_DACONT") != NULL;
    dump_error = getenv("ADH_DUMP_ERROR") != NULL;
}

static void put_f64(const char *tag, const double *v, long n) {
    char t[8] = {0};
    int kind = 0;
    long long cnt = n;
    strncpy(t, tag, 8);
    fwrite(t, 1, 8, dump_fp);
    fwrite(&kind, sizeof(int), 1, dump_fp);
    fwrite(&cnt, sizeof(long long), 1, dump_fp);
    fwrite(v, sizeof(double), (size_t) n, dump_fp);
}

static void put_i32(const char *tag, const int *v, long n) {
    char t[8] = {0};
    int kind = 1;
    long long cnt = n;
    strncpy(t, tag, 8);
    fwrite(t, 1, 8, dump_fp);
    fwrite(&kind, sizeof(int), 1, dump_fp);
    fwrite(&cnt, sizeof(long long), 1, dump_fp);
    fwrite(v, sizeof(int), (size_t) n, dump_fp);
}

static void put_state(const char *th, const char *tu, const char *tv, double *h, SVECT2D *vel, int n) {
    double *u = (double *) malloc(sizeof(double) * n);
    double *v = (double *) malloc(sizeof(double) * n);
    int i;
    for (i = 0; i < n; i++) { u[i] = vel[i].x; v[i] = vel[i].y; }
    put_f64(th, h, n);
    put_f64(tu, u, n);
    put_f64(tv, v, n);
    free(u);
    free(v);
}

int __wrap_fe_main(SSUPER_MODEL *sm) {
    int r;
    dump_open();
    if (dump_mass && !mass_ready && dump_fp != NULL) {   /* the initial state, before any shift */
        SMODEL *mod = &(sm->submodel[0]);
        mass0 = tl_find_grid_mass_elem2d(mod->density, mod->str_values, mod->series_head, mod->sw->d2->head,
                                         mod->grid, mod->flag);
        mass_ready = 1;
    }
    double t0 = now_seconds();
    r = __real_fe_main(sm);
    solve_seconds += now_seconds() - t0;
    attempts++;
    if (r == YES && dump_fp != NULL) {
        SMODEL *mod = &(sm->submodel[0]);
        int n = mod->grid->nnodes;
        double hdr[3];
        int ihdr[3];
        hdr[0] = mod->t_prev;
        hdr[1] = sm->dt;
        hdr[2] = solve_seconds;
        ihdr[0] = sm->solver_info.it_count_nonlin - it_mark;
        ihdr[1] = attempts;
        ihdr[2] = n;
        put_f64("step", hdr, 3);
        put_i32("stepi", ihdr, 3);
        put_state("h", "u", "v", mod->sw->d2->head, mod->sw->d2->vel, n);
        put_i32("wd", mod->grid->wd_flag, mod->grid->nelems2d);
        if (dump_mass) {
            double m[4];
            m[0] = mass0;
            m[1] = tl_find_grid_mass_elem2d(mod->density, mod->str_values, mod->series_head, mod->sw->d2->head,
                                            mod->grid, mod->flag);
            m[2] = tl_find_grid_mass_error_elem2d(mod->density, mod->sw->d2->head, mod->sw->d2->vel, mod->grid,
                                                  mod->flag, mass0, mod->series_head, mod->str_values, mod->dt,
                                                  &mass_flux_total);
            m[3] = mass_flux_total;
            put_f64("mass", m, 4);
        }
        if (dump_dacont) {
            int T = mod->grid->nelems2d, i, e;
            double *d = (double *) malloc(sizeof(double) * 3 * (size_t) (T ? T : 1));
            for (i = 0; i < 3; i++)
                for (e = 0; e < T; e++) d[(size_t) i * T + e] = mod->sw->d2->elem_rhs_dacont_extra_terms[i][e];
            put_f64("dacont", d, 3L * T);
            free(d);
        }
        if (dump_error) {
            int k;
            put_f64("elemerr", mod->grid->elem_error, mod->grid->nelems2d);
            put_f64("nodeerr", mod->sw->d2->error, n);
            for (k = 0; k < mod->ntransport; k++) put_f64("conerr", mod->con[k].error, n);
        }
        {
            int k;
            for (k = 0; k < mod->ntransport; k++) put_f64("con", mod->con[k].concentration, n);
        }
        fflush(dump_fp);
        attempts = 0;
        solve_seconds = 0.0;
        it_mark = sm->solver_info.it_count_nonlin;
    }
    return r;
}

void __wrap_fe_sw2_load(SSUPER_MODEL *sm, int imod) {
    dump_open();
    if (dump_fp != NULL && dump_loads_left > 0) {
        SMODEL *mod = &(sm->submodel[imod]);
        int n = mod->grid->nnodes;
        double hdr[2];
        hdr[0] = mod->t_prev;
        hdr[1] = mod->dt;
        put_f64("load", hdr, 2);
        put_state("h", "u", "v", mod->sw->d2->head, mod->sw->d2->vel, n);
        put_state("h1", "u1", "v1", mod->sw->d2->old_head, mod->sw->d2->old_vel, n);
        put_state("h2", "u2", "v2", mod->sw->d2->older_head, mod->sw->d2->older_vel, n);
        put_i32("wd", mod->grid->wd_flag, mod->grid->nelems2d);
    }
    __real_fe_sw2_load(sm, imod);
    if (dump_fp != NULL && dump_loads_left > 0) {
        SMODEL *mod = &(sm->submodel[imod]);
        int n = mod->grid->nnodes, i, nnz = 0, k = 0;
        put_f64("resid", sm->residual, 3 * n);
        put_f64("diag", sm->diagonal, 9 * n);
        int *rowsz = (int *) malloc(sizeof(int) * n);
        for (i = 0; i < n; i++) { rowsz[i] = sm->matrix[i].size; nnz += rowsz[i]; }
        int *cols = (int *) malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
        double *vals = (double *) malloc(sizeof(double) * 9 * (nnz > 0 ? nnz : 1));
        for (i = 0; i < n; i++) {
            memcpy(cols + k, sm->matrix[i].index, sizeof(int) * rowsz[i]);
            memcpy(vals + 9 * k, sm->matrix[i].value, sizeof(double) * 9 * rowsz[i]);
            k += rowsz[i];
        }
        put_i32("rowsz", rowsz, n);
        put_i32("cols", cols, nnz);
        put_f64("vals", vals, 9L * nnz);
        free(rowsz);
        free(cols);
        free(vals);
        fflush(dump_fp);
        dump_loads_left--;
    }
}

void __wrap_fe_transport_load(SSUPER_MODEL *sm, int imod) {
    dump_open();
    if (dump_fp != NULL && dump_tloads_left > 0) {
        SMODEL *mod = &(sm->submodel[imod]);
        SCON *con = &(mod->con[mod->itrns]);
        int n = mod->grid->nnodes, T = mod->grid->nelems2d, i, e;
        double hdr[3];
        hdr[0] = (double) mod->itrns;
        hdr[1] = mod->t_prev;
        hdr[2] = mod->dt;
        put_f64("tload", hdr, 3);
        put_f64("c", con->concentration, n);
        put_f64("c1", con->old_concentration, n);
        put_f64("c2", con->older_concentration, n);
        put_state("h", "u", "v", mod->sw->d2->head, mod->sw->d2->vel, n);
        put_state("h1", "u1", "v1", mod->sw->d2->old_head, mod->sw->d2->old_vel, n);
        put_state("h2", "u2", "v2", mod->sw->d2->older_head, mod->sw->d2->older_vel, n);
        put_i32("wd", mod->grid->wd_flag, T);
        double *d = (double *) malloc(sizeof(double) * 3 * (size_t) (T ? T : 1));
        for (i = 0; i < 3; i++)
            for (e = 0; e < T; e++) d[(size_t) i * T + e] = mod->sw->d2->elem_rhs_dacont_extra_terms[i][e];
        put_f64("dacont", d, 3L * T);
        free(d);
        put_i32("bcmask", mod->bc_mask, n);
    }
    __real_fe_transport_load(sm, imod);
    if (dump_fp != NULL && dump_tloads_left > 0) {
        SMODEL *mod = &(sm->submodel[imod]);
        int n = mod->grid->nnodes, i, nnz = 0, k = 0;
        put_f64("resid", sm->residual, n);
        put_f64("diag", sm->diagonal, n);
        int *rowsz = (int *) malloc(sizeof(int) * n);
        for (i = 0; i < n; i++) { rowsz[i] = sm->matrix[i].size; nnz += rowsz[i]; }
        int *cols = (int *) malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
        double *vals = (double *) malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
        for (i = 0; i < n; i++) {
            memcpy(cols + k, sm->matrix[i].index, sizeof(int) * rowsz[i]);
            memcpy(vals + k, sm->matrix[i].value, sizeof(double) * rowsz[i]);
            k += rowsz[i];
        }
        put_i32("rowsz", rowsz, n);
        put_i32("cols", cols, nnz);
        put_f64("vals", vals, nnz);
        free(rowsz);
        free(cols);
        free(vals);
        fflush(dump_fp);
        dump_tloads_left--;
    }
}
