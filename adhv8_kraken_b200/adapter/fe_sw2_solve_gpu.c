/* fe_sw2_solve_gpu.c -- the reference-side binding of the B200 SW2 step.
 *
 * Compiled with the reference AdH sources (it includes their global_header.h) and linked
 * against libsw2gpu.so.  It replaces fe_sw2_solve(SSUPER_MODEL *, int)
 * (src/fe/sw2/fe_sw2_solve.c:30-57), the only SW2 entry point of the reference's time loop:
 * fe_main (src/fe/fe_main.c:485-489), called from the retry loop of adh_run_func_
 * (src/main/adh_func.c:535-549), after fe_main itself shifted the time levels
 * (fe_sw2, src/fe/sw2/fe_sw2.c:43-50) and the loop averaged every series over the step
 * (sseries_setall_ts_valuesAVG).  Two ways to bind it:
 *
 *   - rename the call in fe_main to fe_sw2_solve_gpu, or
 *   - link the reference with -Wl,--wrap=fe_sw2_solve: its call then lands in
 *     __wrap_fe_sw2_solve below (how this repository's build of the reference does it).
 *
 * Contract, as fe_sw2_solve / fe_newton (src/fe/fe_newton.c:214-912):
 *   YES: head and vel hold t + dt, grid->wd_flag the step's wet/dry flags, the Newton
 *        counters advanced, flag.SOLVE_ATF = YES;
 *   NO:  dt scaled by tc_scale (DT_REDUCE_FACTOR), TIME_ADAPT_FAIL set, the current level
 *        reset to the old one by fe_sw2_init (fe_newton.c:854-892); the time loop retries.
 * Errors that are not a failed step (unsupported input, CUDA errors) end the run through
 * tl_error, as the reference does for its own fatal errors.
 *
 * The host stays authoritative for the state: every call hands the device the two levels the
 * time loop holds (old, older) and reads the new level back, so output, test modules and mass
 * diagnostics of the reference read what they always read.  The device mesh is rebuilt
 * (sw2gpu_create) on the first call and whenever the grid was adapted or its sizes changed.
 *
 * The adaption error indicator that fe_main computes after every accepted step
 * (ssw_2d_calculate_elem_error, src/structs/ssw_2d.c:424-500, called at src/fe/fe_main.c:625
 * and read by error_main / adpt_main) comes from the device too when the reference is linked
 * with -Wl,--wrap=ssw_2d_calculate_elem_error: __wrap_ssw_2d_calculate_elem_error below takes
 * it from the state the device step just produced, and hands over to the host routine
 * whenever the device does not hold that state (before the first GPU step, after a failed one).
 *
 * The transport of general constituents (fe_transport, src/fe/transport/fe_transport.c:31-113,
 * called by fe_main right after the flow, src/fe/fe_main.c:528-531) runs on the device too when
 * the reference is linked with -Wl,--wrap=fe_transport: fe_transport_gpu below solves every
 * constituent on the flow step the device just produced, with the host's concentration levels
 * handed over and read back like the flow's.  Models the library does not transport (sediment,
 * the vorticity constituent, transport-load edges, 3D grids, a flow state not on the device) go to
 * the reference's own fe_transport, which reads the side output this binding copies back.
 */
#include "global_header.h"
#include "sw2gpu.h"

typedef struct {
    sw2gpu_ctx *ctx;
    int nnodes, nelems2d, nelems1d, nstring;
    int nseries;            /* series ids 0 .. nseries - 1 */
    double *h, *u, *v;      /* staging of one time level */
    double *series;         /* step-averaged value of every series, by id */
    int *mat_of;            /* [nstring] material of the elements on each material string, or -1 */
    int32_t *wind_flag;     /* [nstring] MP WND STR of that material (wind runs only) */
    double *wind_att;       /* [nstring] MP WND ATT of that material */
    double *wsx, *wsy;      /* [nnodes] nodal wind values of the coming step */
    double *rxx, *rxy, *ryy;  /* [nnodes] nodal wave radiation stresses (wave runs only) */
    int state_on_device;    /* the host's current and old levels are the device's (last step accepted) */
    int trn_ready;          /* the constituents are set up on the device (sw2gpu_set_transport) */
    double *c;              /* staging of one concentration level */
    sw2gpu_stats *tstats;   /* [ntransport] */
} GPU_SW2;

static GPU_SW2 gpu;

enum { kMinLinIt = 2000 };   /* smallest Krylov iteration cap of the device solve */

static void gpu_fail(const char *what) {
    char msg[600];
    snprintf(msg, sizeof msg, "B200 SW2 step: %s: %s\n", what, sw2gpu_last_error());
    tl_error(msg);
}

/* Boundary edges whose string contributes a residual in fe_sw2_boundary_resid
 * (src/fe/sw2/fe_sw2_boundary_resid.c:212-470).  The library computes VEL, OTW, OF and OVH
 * and rejects the others at create time; an edge of any other string (a wall, a transport
 * string) adds nothing to the reference's residual or Jacobian and is left out. */
static int edge_contributes(int bc_flag) {
    switch (bc_flag) {
        case BCT_VEL_NEU: case BCT_PRS_NEU: case BCT_OUTFLOW: case BCT_OVH_NEU:
        case BCT_DIS_NEU: case BCT_WEIRU: case BCT_WEIRD: case BCT_FLAPU: case BCT_FLAPD:
        case BCT_SLUICEU: case BCT_SLUICED: case BCT_DB_VEL: case BCT_HYBRID_INTERNAL:
            return 1;
        default:
            return 0;
    }
}

static int series_count(SSERIES *head) {
    int n = 0;
    SSERIES *s;
    for (s = head; s != NULL; s = s->next)
        if (s->id + 1 > n) n = s->id + 1;
    return n;
}

static void gpu_release(void) {
    if (gpu.ctx) sw2gpu_destroy(gpu.ctx);
    free(gpu.h); free(gpu.u); free(gpu.v); free(gpu.series); free(gpu.mat_of);
    free(gpu.wind_flag); free(gpu.wind_att); free(gpu.wsx); free(gpu.wsy);
    free(gpu.rxx); free(gpu.rxy); free(gpu.ryy); free(gpu.c); free(gpu.tstats);
    memset(&gpu, 0, sizeof gpu);
}

/* Builds the device mesh (sw2gpu_create): the library indexes the element material tables by
 * the element's string (roughness and water sources live on strings, fe_sw2_body_resid.c), so
 * each material string gets the parameters of the material its elements carry. */
static void gpu_prepare(SSUPER_MODEL *sm, SMODEL *mod) {
    SGRID *g = mod->grid;
    const int V = g->nnodes, T = g->nelems2d, S = mod->nstring;
    int i, k, E = 0;
    gpu_release();
    /* body terms the library does not compute (the wind library's forms and the CSTORM-coupled
     * wave stress of fe_sw2_body_resid.c:679-690, :869-970 baroclinic terms): refuse the model
     * rather than solve without them */
    if (mod->flag.WIND_LIBRARY == ON)
        tl_error("B200 SW2 step: the wind library is not supported\n");
    if (mod->flag.WAVE == ON && mod->flag.CSTORM_WSID != OFF && mod->flag.CSTORM_WSID != 7)
        tl_error("B200 SW2 step: CSTORM-coupled wave stresses are not supported\n");
    if (mod->flag.BAROCLINIC != OFF)
        tl_error("B200 SW2 step: baroclinic terms are not supported\n");
    for (i = 0; i < g->nelems1d; i++) {
        const int s = g->elem1d[i].string;
        if (s >= 0 && s < S && mod->str_values[s].phys_flag == SW2_FLAG &&
            edge_contributes(mod->str_values[s].ol_flow.bc_flag)) E++;
    }
    double *x = malloc(V * sizeof(double)), *y = malloc(V * sizeof(double)), *z = malloc(V * sizeof(double));
    int32_t *nstr = malloc(V * sizeof(int32_t));
    int32_t *tri = malloc((3 * (size_t) T + 1) * sizeof(int32_t)), *emat = malloc((T + 1) * sizeof(int32_t));
    int32_t *edg = malloc((2 * (size_t) E + 1) * sizeof(int32_t)), *estr = malloc((E + 1) * sizeof(int32_t));
    int32_t *epar = malloc((E + 1) * sizeof(int32_t));
    int32_t *bc = malloc((S + 1) * sizeof(int32_t)), *isg = malloc((S + 1) * sizeof(int32_t));
    int32_t *ivx = malloc((S + 1) * sizeof(int32_t)), *ivy = malloc((S + 1) * sizeof(int32_t));
    int32_t *iu0 = malloc((S + 1) * sizeof(int32_t)), *mode = malloc((S + 1) * sizeof(int32_t));
    int32_t *mat_of = malloc((S + 1) * sizeof(int32_t));
    double *ks = malloc((S + 1) * sizeof(double)), *ev = malloc((3 * (size_t) S + 1) * sizeof(double));
    double *coef = malloc((S + 1) * sizeof(double)), *cor = malloc((S + 1) * sizeof(double));
    for (i = 0; i < V; i++) {
        x[i] = g->node[i].x; y[i] = g->node[i].y; z[i] = g->node[i].z;
        nstr[i] = g->node[i].string < 0 ? SW2GPU_NORMAL : g->node[i].string;
    }
    for (k = 0; k < S; k++) mat_of[k] = -1;
    for (i = 0; i < T; i++) {
        if (g->elem2d[i].nnodes != 3) tl_error("B200 SW2 step: triangles only\n");
        for (k = 0; k < 3; k++) tri[3 * i + k] = g->elem2d[i].nodes[k];
        emat[i] = g->elem2d[i].string;
        if (emat[i] >= 0 && emat[i] < S) mat_of[emat[i]] = g->elem2d[i].mat;
    }
    for (i = 0, k = 0; i < g->nelems1d; i++) {
        const int s = g->elem1d[i].string;
        if (!(s >= 0 && s < S && mod->str_values[s].phys_flag == SW2_FLAG &&
              edge_contributes(mod->str_values[s].ol_flow.bc_flag))) continue;
        edg[2 * k] = g->elem1d[i].nodes[0];
        edg[2 * k + 1] = g->elem1d[i].nodes[1];
        estr[k] = s;
        epar[k] = g->elem1d[i].elem2d;
        k++;
    }
    for (k = 0; k < S; k++) {
        const STR_VALUE *st = &mod->str_values[k];
        bc[k] = st->ol_flow.bc_flag;
        isg[k] = st->ol_flow.isigma;
        ivx[k] = st->ol_flow.ivx;
        ivy[k] = st->ol_flow.ivy;
        iu0[k] = st->ol_flow.iu_0;
        ks[k] = st->fterms.eqrheight;
        mode[k] = 0; ev[3 * k] = ev[3 * k + 1] = ev[3 * k + 2] = 0.0; coef[k] = 0.0; cor[k] = 0.0;
        if (mat_of[k] >= 0) {
            const SMAT_SW *m = mod->mat[mat_of[k]].sw;
            mode[k] = (m->EEVF == YES) ? m->eev_mode : 0;
            ev[3 * k] = m->ev.xx; ev[3 * k + 1] = m->ev.yy; ev[3 * k + 2] = m->ev.xy;
            coef[k] = m->eev_coef;
            cor[k] = m->coriolis;
        }
    }
    gpu.nseries = series_count(mod->series_head);
    sw2gpu_mesh me;
    me.nnodes = V; me.nelems2d = T; me.nelems1d = E; me.nstrings = S; me.nmats = S; me.nseries = gpu.nseries;
    me.x = x; me.y = y; me.z = z; me.node_string = nstr;
    me.elem2d_nodes = tri; me.elem2d_mat = emat;
    me.elem1d_nodes = edg; me.elem1d_string = estr; me.elem1d_parent = epar;
    me.str_bc_flag = bc; me.str_isigma = isg; me.str_ivx = ivx; me.str_ivy = ivy; me.str_iu0 = iu0;
    me.str_rough_height = ks;
    me.mat_eev_mode = mode; me.mat_ev = ev; me.mat_eev_coef = coef; me.mat_coriolis = cor;
    sw2gpu_params p;
    memset(&p, 0, sizeof p);
    p.gravity = mod->gravity; p.density = mod->density; p.viscosity = mod->viscosity;
    p.drying_lower_limit = mod->drying_lower_limit; p.drying_upper_limit = mod->drying_upper_limit;
    p.tau_temporal = mod->tau_temporal; p.tau_pg = mod->tau_pg;
    p.tol_nonlin = sm->tol_nonlin; p.inc_nonlin = sm->inc_nonlin;
    p.max_nonlin_it = sm->max_nonlin_it;
    /* IP MIT bounds the reference's BiCGSTAB, whose preconditioner is an exact LU of the node
     * blocks (one or two iterations); the device preconditions with 3x3 block Jacobi, which needs
     * more iterations for the same system, so its cap is at least kMinLinIt */
    p.max_lin_it = sm->solver_info.max_lin_it > kMinLinIt ? sm->solver_info.max_lin_it : kMinLinIt;
    p.max_linesearch_cuts = sm->solver_info.max_nonlin_linesearch_cuts;
    p.precision = SW2GPU_FP64;
    /* the device Krylov solve's own floor (the library's default): each Newton iteration is
     * solved to a relative 1e-8 at least, tightened against tol_nonlin as the residual falls */
    p.lin_rtol = 1e-8; p.lin_atol = 1e-30;
    /* OP BLK 1 with OP PRE 1 (the reference's default) preconditions with an exact LU of the
     * whole system, so its BiCGSTAB converges at any time-step length: the device takes the same
     * exact solve (a banded LU) whenever the band fits, else block-Jacobi BiCGSTAB */
    int rc = SW2GPU_E_ARG;
    if (mod->nblock == 1 && mod->solver_info.prec_value == 1) {
        p.precond = SW2GPU_PREC_BAND;
        rc = sw2gpu_create(&me, &p, NULL, &gpu.ctx);
    }
    if (rc != SW2GPU_OK) {
        p.precond = SW2GPU_PREC_BJACOBI;
        rc = sw2gpu_create(&me, &p, NULL, &gpu.ctx);
    }
    free(x); free(y); free(z); free(nstr); free(tri); free(emat); free(edg); free(estr); free(epar);
    free(bc); free(isg); free(ivx); free(ivy); free(iu0); free(mode); free(ks); free(ev);
    free(coef); free(cor);
    gpu.mat_of = mat_of;
    gpu.nstring = S;
    if (rc != SW2GPU_OK) gpu_fail("sw2gpu_create");
    if (sm->solver_info.force_nonlin_it == YES)   /* the device resets a failed step; it cannot keep it */
        tl_error("B200 SW2 step: force_nonlin_it (accept a failed Newton solve) is not supported\n");
    if (mod->ntransport > 0 && sw2gpu_set_dacont(gpu.ctx, 1) != SW2GPU_OK) gpu_fail("sw2gpu_set_dacont");
    gpu.nnodes = V; gpu.nelems2d = T; gpu.nelems1d = g->nelems1d;
    gpu.h = malloc(V * sizeof(double)); gpu.u = malloc(V * sizeof(double)); gpu.v = malloc(V * sizeof(double));
    if (mod->flag.WIND == ON) {   /* the material wind forms, indexed like the library's material table */
        gpu.wind_flag = malloc((S + 1) * sizeof(int32_t));
        gpu.wind_att = malloc((S + 1) * sizeof(double));
        gpu.wsx = malloc(V * sizeof(double));
        gpu.wsy = malloc(V * sizeof(double));
        for (k = 0; k < S; k++) {
            gpu.wind_flag[k] = gpu.mat_of[k] >= 0 ? mod->mat[gpu.mat_of[k]].sw->wind_flag : 0;
            gpu.wind_att[k] = gpu.mat_of[k] >= 0 ? mod->mat[gpu.mat_of[k]].sw->windatt : 1.0;
        }
    }
    if (mod->flag.WAVE == ON) {
        gpu.rxx = malloc(V * sizeof(double));
        gpu.rxy = malloc(V * sizeof(double));
        gpu.ryy = malloc(V * sizeof(double));
    }
    gpu.series = malloc((gpu.nseries + 1) * sizeof(double));
}

/* one level of the host state to device level `level` */
static void put_level(int level, const double *head, const SVECT2D *vel) {
    int i;
    for (i = 0; i < gpu.nnodes; i++) { gpu.h[i] = head[i]; gpu.u[i] = vel[i].x; gpu.v[i] = vel[i].y; }
    if (sw2gpu_set_state(gpu.ctx, level, gpu.h, gpu.u, gpu.v) != SW2GPU_OK) gpu_fail("sw2gpu_set_state");
}

int fe_sw2_solve_gpu(SSUPER_MODEL *sm, int isubModel) {
    SMODEL *mod = &(sm->submodel[isubModel]);
    SSW_2D *sw = mod->sw->d2;
    SGRID *g = mod->grid;
    SSERIES *s;
    int i;
    assert(sw && g);
    if (!gpu.ctx || mod->flag.ADAPTED_THE_GRID == YES || g->nnodes != gpu.nnodes || g->nelems2d != gpu.nelems2d ||
        g->nelems1d != gpu.nelems1d)
        gpu_prepare(sm, mod);
    sm->solver_info.refresh = YES;
    sm->solver_info.PRN_NEWTON = HYD;
    sm->solver_info.LINEAR_PROBLEM = NO;
    /* sw2gpu_step shifts the device levels itself (older <- old <- current); fe_main already
     * shifted the host's, so the host's old level goes in as the device's current one and its
     * older level as the device's old one */
    put_level(0, sw->old_head, sw->old_vel);
    put_level(1, sw->older_head, sw->older_vel);
    for (i = 0; i < gpu.nseries; i++) gpu.series[i] = 0.0;
    for (s = mod->series_head; s != NULL; s = s->next)
        if (s->id >= 0 && s->id < gpu.nseries && s->ivalue != NULL) gpu.series[s->id] = s->ivalue[0];
    if (gpu.wsx) {   /* the nodal winds meteor_update set for this step (fe_sw2_body_resid.c:679-686) */
        for (i = 0; i < gpu.nnodes; i++) { gpu.wsx[i] = sw->winds[i].stress.x; gpu.wsy[i] = sw->winds[i].stress.y; }
        if (sw2gpu_set_wind(gpu.ctx, gpu.wind_flag, gpu.wind_att, gpu.wsx, gpu.wsy) != SW2GPU_OK)
            gpu_fail("sw2gpu_set_wind");
    }
    if (gpu.rxx) {   /* the nodal radiation stresses (hot file or wave series, fe_sw2_body_resid.c:689-690) */
        for (i = 0; i < gpu.nnodes; i++) {
            gpu.rxx[i] = sw->waves[i].rads.xx; gpu.rxy[i] = sw->waves[i].rads.xy; gpu.ryy[i] = sw->waves[i].rads.yy;
        }
        if (sw2gpu_set_waves(gpu.ctx, gpu.rxx, gpu.rxy, gpu.ryy) != SW2GPU_OK) gpu_fail("sw2gpu_set_waves");
    }
    sw2gpu_stats st;
    gpu.state_on_device = 0;
    const int rc = sw2gpu_step(gpu.ctx, sm->dt, gpu.series, &st);
    sm->nonlinear_it_total += st.newton_its;
    sm->solver_info.it_count_nonlin += st.newton_its;
    for (i = 0; i < sm->nsubmodels; i++)
        if (sm->submodel[i].proc_flag == 1) sm->submodel[i].flag.SOLVE_ATF = NO;
    if (rc == SW2GPU_OK) {
        if (sw2gpu_get_state(gpu.ctx, 0, gpu.h, gpu.u, gpu.v) != SW2GPU_OK) gpu_fail("sw2gpu_get_state");
        for (i = 0; i < gpu.nnodes; i++) { sw->head[i] = gpu.h[i]; sw->vel[i].x = gpu.u[i]; sw->vel[i].y = gpu.v[i]; }
        if (sw2gpu_get_wd_flag(gpu.ctx, g->wd_flag) != SW2GPU_OK) gpu_fail("sw2gpu_get_wd_flag");
        if (gpu.rxx) {   /* the nodal wave stresses the host residual leaves behind for output: every
                          * fully wet SW2 element, in element order, stores its stress at its nodes
                          * (fe_sw2_resid.c:74-80, fe_sw2_body_resid.c:689-690, smeteor.c:333-337) */
            int e;
            for (e = 0; e < gpu.nelems2d; e++)
                if (g->wd_flag[e] == 0 && mod->str_values[g->elem2d[e].string].phys_flag == SW2_FLAG)
                    swave_elem2d_get_local_stress(2, mod->flag.CSTORM_WSID, sw->waves, g->elem2d[e], g->elem2d[e].nodes);
        }
        if (mod->ntransport > 0) {   /* [3][nelems2d], read by the transport solve */
            double *dac = malloc(3 * (size_t) gpu.nelems2d * sizeof(double));
            int k;
            if (sw2gpu_get_dacont(gpu.ctx, dac) != SW2GPU_OK) gpu_fail("sw2gpu_get_dacont");
            for (k = 0; k < 3; k++)
                memcpy(sw->elem_rhs_dacont_extra_terms[k], dac + (size_t) k * gpu.nelems2d,
                       gpu.nelems2d * sizeof(double));
            free(dac);
        }
        for (i = 0; i < sm->nsubmodels; i++)
            if (sm->submodel[i].proc_flag == 1) sm->submodel[i].flag.SOLVE_ATF = YES;
        sm->solver_info.PRN_NEWTON = OFF;
        gpu.state_on_device = 1;
        return YES;
    }
    if (rc != SW2GPU_E_NEWTON && rc != SW2GPU_E_LINEAR && rc != SW2GPU_E_NAN) gpu_fail("sw2gpu_step");
    /* a failed step (fe_newton.c:854-892): dt * DT_REDUCE_FACTOR, every submodel told, the
     * current level back at the old one */
    for (i = 0; i < sm->nsubmodels; i++)
        if (sm->submodel[i].proc_flag == 1) sm->submodel[i].flag.UMFPACK_FAIL = NO;
    if (sm->solver_info.force_nonlin_it == YES) return YES;
    tc_scale(&sm->dt);
    for (i = 0; i < sm->nsubmodels; i++) {
        sm->submodel[i].dt = sm->dt;
        if (sm->submodel[i].proc_flag == 1) sm->submodel[i].flag.TIME_ADAPT_FAIL = YES;
    }
    fe_sw2_init(sm, isubModel);
    sm->solver_info.it_count_nonlin_failed += st.newton_its;
    return NO;
}

/* The adaption error indicator from the device (the linker's --wrap=ssw_2d_calculate_elem_error
 * binding): valid when the device holds the accepted step's current and old levels for this grid;
 * otherwise the reference's own routine runs. */
void __real_ssw_2d_calculate_elem_error(SSW_2D *sw, SGRID *grid, SMAT *mat, double dt);
void __wrap_ssw_2d_calculate_elem_error(SSW_2D *sw, SGRID *grid, SMAT *mat, double dt) {
    int k;
    if (!gpu.ctx || !gpu.state_on_device || grid->nnodes != gpu.nnodes || grid->nelems2d != gpu.nelems2d) {
        __real_ssw_2d_calculate_elem_error(sw, grid, mat, dt);
        return;
    }
    /* the library's material table is indexed by material string (gpu_prepare) */
    double *tol = malloc((gpu.nstring + 1) * sizeof(double));
    for (k = 0; k < gpu.nstring; k++) tol[k] = gpu.mat_of[k] >= 0 ? mat[gpu.mat_of[k]].sw->refine_tolerance : 1.0;
    if (sw2gpu_elem_error(gpu.ctx, tol, grid->elem_error, sw->error) != SW2GPU_OK) gpu_fail("sw2gpu_elem_error");
    free(tol);
}

/* ---- constituent transport ---- */

int __real_fe_transport(SSUPER_MODEL *sm, int isubModel);

static int transport_on_device(SMODEL *mod) {
    int k, i;
    if (!gpu.ctx || !gpu.state_on_device || mod->grid->ndim != 2 || mod->grid->nnodes != gpu.nnodes ||
        mod->grid->nelems2d != gpu.nelems2d || mod->flag.VORTICITY == ON || mod->is_sediment_running ||
        mod->nstring != gpu.nstring)
        return 0;
    for (k = 0; k < mod->ntransport; k++)
        if (mod->con[k].type != CON) return 0;
    for (i = 0; i < mod->grid->nelems1d; i++) {   /* a transport load edge (BCT_NEU_LOAD, :259-272) */
        const int s = mod->grid->elem1d[i].string;
        if (s >= 0 && s < mod->nstring && mod->str_values[s].ol_flow.bc_flag == BCT_NEU_LOAD) return 0;
    }
    return 1;
}

/* the constituents as the library takes them: property[0], MP DF per material string (the
 * library's material table, gpu_prepare), and per string the DB TRN / NB TRN flag and series */
static void transport_setup(SMODEL *mod) {
    const int n = mod->ntransport, S = gpu.nstring;
    int k, s;
    double *refc = malloc((n + 1) * sizeof(double)), *dm = malloc(((size_t) n * S + 1) * sizeof(double));
    int32_t *bc = malloc(((size_t) n * S + 1) * sizeof(int32_t)), *ser = malloc(((size_t) n * S + 1) * sizeof(int32_t));
    for (k = 0; k < n; k++) {
        refc[k] = mod->con[k].property[0];
        for (s = 0; s < S; s++) {
            const INPUT_DATA *in = &(mod->str_values[s].trans[k]);
            dm[(size_t) k * S + s] = gpu.mat_of[s] >= 0 ? mod->mat[gpu.mat_of[s]].trn[k].d_m : 0.0;
            bc[(size_t) k * S + s] = in->bc_flag == BCT_DIR ? SW2GPU_BCT_DIR : in->bc_flag == BCT_NEU ? SW2GPU_BCT_NEU : 0;
            ser[(size_t) k * S + s] = in->bc_flag == BCT_DIR ? in->iu_0 : in->bc_flag == BCT_NEU ? in->isigma : -1;
        }
    }
    sw2gpu_transport t = {n, refc, dm, bc, ser};
    if (sw2gpu_set_transport(gpu.ctx, &t) != SW2GPU_OK) gpu_fail("sw2gpu_set_transport");
    free(refc); free(dm); free(bc); free(ser);
    gpu.c = realloc(gpu.c, (gpu.nnodes + 1) * sizeof(double));
    gpu.tstats = realloc(gpu.tstats, (n + 1) * sizeof(sw2gpu_stats));
    gpu.trn_ready = 1;
}

int fe_transport_gpu(SSUPER_MODEL *sm, int isubModel) {
    SMODEL *mod = &(sm->submodel[isubModel]);
    const int V = gpu.nnodes;
    int k, i;
    if (!transport_on_device(mod)) return __real_fe_transport(sm, isubModel);
    if (!gpu.trn_ready) transport_setup(mod);
    mod->nsys = 1; sm->nsys = 1;                       /* fe_transport.c:40-44 */
    mod->nsys_sq = 1; sm->nsys_sq = 1;
    sm->solver_info.refresh = YES;
    sm->solver_info.LINEAR_PROBLEM = YES;
    /* the device shifts each constituent's levels itself: the host's current level goes in as the
     * device's current one and its old level as the device's old one */
    for (k = 0; k < mod->ntransport; k++) {
        if (sw2gpu_set_conc(gpu.ctx, k, 0, mod->con[k].concentration) != SW2GPU_OK ||
            sw2gpu_set_conc(gpu.ctx, k, 1, mod->con[k].old_concentration) != SW2GPU_OK)
            gpu_fail("sw2gpu_set_conc");
    }
    memset(gpu.tstats, 0, mod->ntransport * sizeof(sw2gpu_stats));
    const int rc = sw2gpu_transport_step(gpu.ctx, gpu.series, gpu.tstats);
    if (rc != SW2GPU_OK && rc != SW2GPU_E_NEWTON && rc != SW2GPU_E_LINEAR && rc != SW2GPU_E_NAN)
        gpu_fail("sw2gpu_transport_step");
    /* the constituents up to the first that failed were shifted and solved (or reset) on the
     * device, those after it not at all, as fe_transport returns at the first failure: the host
     * levels follow, older <- old, old <- current (fe_transport.c:60-61), then the new current */
    int last = mod->ntransport - 1;
    if (rc != SW2GPU_OK)
        for (k = 0; k < mod->ntransport; k++)
            if (gpu.tstats[k].status != SW2GPU_OK) { last = k; break; }
    for (k = 0; k <= last; k++) {
        sarray_copy_dbl(mod->con[k].older_concentration, mod->con[k].old_concentration, V);
        sarray_copy_dbl(mod->con[k].old_concentration, mod->con[k].concentration, V);
        if (sw2gpu_get_conc(gpu.ctx, k, 0, gpu.c) != SW2GPU_OK) gpu_fail("sw2gpu_get_conc");
        for (i = 0; i < V; i++) mod->con[k].concentration[i] = gpu.c[i];
        sm->solver_info.it_count_nonlin += gpu.tstats[k].newton_its;
    }
    sm->solver_info.PRN_NEWTON = OFF;
    if (rc == SW2GPU_OK) {
        /* the adaption error indicator of the constituents (fe_transport.c:83-88), host routine */
        SVECT2D *vel2d = mod->flag.SW_FLOW == ON ? mod->sw->d2->vel : mod->ns->d2->vel;
        scon_calculate_elem2d_error(mod->ntransport, mod->con, vel2d, mod->sw->d2->head, mod->grid, mod->mat, mod->dt);
        return YES;
    }
    /* a failed constituent (fe_newton.c:854-892): its current level already reset by the device
     * (fe_transport_init), dt * DT_REDUCE_FACTOR and every submodel told */
    sm->solver_info.it_count_nonlin_failed += gpu.tstats[last].newton_its;
    if (sm->solver_info.force_nonlin_it == YES) return YES;
    tc_scale(&sm->dt);
    for (i = 0; i < sm->nsubmodels; i++) {
        sm->submodel[i].dt = sm->dt;
        if (sm->submodel[i].proc_flag == 1) sm->submodel[i].flag.TIME_ADAPT_FAIL = YES;
    }
    return NO;
}

/* the linker's --wrap=fe_transport binding */
int __wrap_fe_transport(SSUPER_MODEL *sm, int isubModel) { return fe_transport_gpu(sm, isubModel); }

/* the linker's --wrap=fe_sw2_solve binding */
int __wrap_fe_sw2_solve(SSUPER_MODEL *sm, int isubModel) { return fe_sw2_solve_gpu(sm, isubModel); }

/* releases the device context (adh_finalize_func_) */
void fe_sw2_gpu_finalize(void) { gpu_release(); }
