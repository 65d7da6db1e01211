/* sw2gpu.h -- C ABI of the B200 SW2 (2D shallow-water) Newton step.
 *
 * Drop-in for the AdH SW2 solve path:
 *   fe_sw2_solve(SSUPER_MODEL*, int)            src/fe/sw2/fe_sw2_solve.c:30-57
 *     -> fe_newton(..., fe_sw2_init, fe_sw2_update, fe_sw2_resid, fe_sw2_load, fe_sw2_inc)
 *                                               src/fe/fe_newton.c:214-912
 *        -> fe_sw2_resid / fe_sw2_body_resid / fe_sw2_boundary_resid
 *                                               src/fe/sw2/fe_sw2_resid.c:29-216
 *        -> fe_sw2_load (FD Jacobian)           src/fe/sw2/fe_sw2_load.c:34-269
 *        -> solv_linear_sys_setup / _solve      src/solver/solv_linear_sys_setup.c:15,
 *                                               src/solver/solv_linear_sys_solve.c:16
 *
 * Plain pointers and sizes only.  Every entry point returns 0 on success and a
 * nonzero SW2GPU_E* code on failure; sw2gpu_last_error() gives the message.
 * Node unknowns are ordered [u, v, h] per node, Jacobian blocks are 3x3
 * row-major with rows (x-momentum, y-momentum, continuity) and columns (u, v, h)
 * (src/fe/fe_assemble_matrix.c:200-208).
 */
#ifndef SW2GPU_H
#define SW2GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SW2GPU_ABI_VERSION 1

/* status codes */
#define SW2GPU_OK            0
#define SW2GPU_E_ARG         1   /* bad argument / unsupported input */
#define SW2GPU_E_CUDA        2   /* CUDA runtime error */
#define SW2GPU_E_NOMEM       3   /* device allocation failed / admission refused */
#define SW2GPU_E_NEWTON      4   /* Newton did not converge: state reset, caller scales dt (tc_scale) */
#define SW2GPU_E_LINEAR      5   /* Krylov hit max_lin_it (solv_bcgstab.c:280-292) */
#define SW2GPU_E_NAN         6   /* NaN/Inf residual (fe_newton.c:119-124, 639-646) */
#define SW2GPU_E_TIMEOUT     7   /* a bounded device wait ran out */

/* boundary-condition flags (src/include/define.h) */
#define SW2GPU_NORMAL        (-1)
#define SW2GPU_BCT_OUTFLOW     4
#define SW2GPU_BCT_PRS_DIR     7
#define SW2GPU_BCT_VEL_DIR     8
#define SW2GPU_BCT_PRS_NEU     9   /* NB OTW: tailwater elevation */
#define SW2GPU_BCT_VEL_NEU    10   /* NB VEL: prescribed normal unit discharge */
#define SW2GPU_BCT_WATER_SOURCE 12
#define SW2GPU_BCT_VEL_PRS_DIR 16
#define SW2GPU_BCT_OVH_NEU    18   /* NB OVH: water elevation (str_isigma) + velocity (str_ivx, str_ivy) series */
/* lids on node strings (pressure under a lid in the body residual, fe_sw2_body_resid.c:154-177):
 * not built; sw2gpu_create rejects them with SW2GPU_E_ARG rather than ignore them */
#define SW2GPU_BCT_LID_DFT    20
#define SW2GPU_BCT_LID_ELV    21
#define SW2GPU_BCT_LID_DEP    22

/* precision modes */
#define SW2GPU_FP64          0   /* everything FP64 */
#define SW2GPU_MIXED         1   /* FP32 Jacobian storage, SpMV and preconditioner; FP64 Newton */

/* linear solve of every Newton iteration */
#define SW2GPU_PREC_BJACOBI  0   /* BiCGSTAB preconditioned with 3x3 block Jacobi */
#define SW2GPU_PREC_ILU0     1   /* block ILU(0): not built; sw2gpu_create rejects it with SW2GPU_E_ARG */
#define SW2GPU_PREC_BAND     2   /* exact LU of the Jacobi-scaled system in a band (nodes in reverse
                                  * Cuthill-McKee order, no pivoting), the direct solve the reference's
                                  * OP BLK 1 profile LU gives (solv_blk_set_profile,
                                  * src/solver/solv_blk_profile.c:5-79).  FP64 only; sw2gpu_create
                                  * rejects it with SW2GPU_E_ARG when the band would exceed 2 GiB.
                                  * Work n bw^2 per factorisation (n = 3 nnodes, bw the half-width in
                                  * unknowns): for the small and medium meshes of test decks, whose
                                  * time steps are too long for block Jacobi to converge */
#define SW2GPU_PREC_DILU     3   /* BiCGSTAB preconditioned with block D-ILU, the diagonal form of
                                  * block ILU(0) (L and U are the matrix's own strict block parts,
                                  * the diagonal blocks Dt_n = D_n - sum L_nk Dt_k^-1 U_kn), in a
                                  * greedy multicolour node order, applied on the split system with
                                  * Eisenstat's rearrangement (one SpMV's bytes per application).
                                  * About 3x fewer iterations than block Jacobi on the benchmark
                                  * basins, but each iteration waits at 4C - 1 grid barriers for C
                                  * colours (19 for 5) against block Jacobi's 3, so on a B200 it is
                                  * slower at every measured size (10k-1M triangles); block Jacobi
                                  * stays the default.  FP64 or MIXED (FP32 blocks); create rejects
                                  * a node graph that needs more than 16 colours, or a node with more
                                  * than 16 neighbours of lower or of higher colour, with SW2GPU_E_ARG */

/* Mesh and model data (what fe_sw2_* read from SGRID / SMODEL).  Host pointers;
 * the library copies what it needs at create time. */
typedef struct sw2gpu_mesh {
    int32_t nnodes, nelems2d, nelems1d, nstrings, nmats, nseries;
    const double  *x, *y, *z;          /* [nnodes] node coordinates and bed elevation */
    const int32_t *node_string;        /* [nnodes] SW2GPU_NORMAL or string id (NDS) */
    const int32_t *elem2d_nodes;       /* [3*nelems2d] counter-clockwise */
    const int32_t *elem2d_mat;         /* [nelems2d] material id; its string id is the same */
    const int32_t *elem1d_nodes;       /* [2*nelems1d] */
    const int32_t *elem1d_string;      /* [nelems1d] edge string */
    const int32_t *elem1d_parent;      /* [nelems1d] adjacent 2D element */
    const int32_t *str_bc_flag;        /* [nstrings] ol_flow.bc_flag */
    const int32_t *str_isigma;         /* [nstrings] series id or -1 */
    const int32_t *str_ivx, *str_ivy, *str_iu0;   /* [nstrings] Dirichlet (and NB OVH velocity) series ids or -1 */
    const double  *str_rough_height;   /* [nstrings] fterms.eqrheight (UNSET_FLT = no drag) */
    const int32_t *mat_eev_mode;       /* [nmats] 0: user eddy viscosity (EVS); 1..3: EEV mode */
    const double  *mat_ev;             /* [3*nmats] EVS xx, yy, xy */
    const double  *mat_eev_coef;       /* [nmats] */
    const double  *mat_coriolis;       /* [nmats] latitude, degrees */
} sw2gpu_mesh;

typedef struct sw2gpu_params {
    double  gravity, density, viscosity;
    double  drying_lower_limit, drying_upper_limit;
    double  tau_temporal, tau_pg;
    double  tol_nonlin, inc_nonlin;    /* IP NTL / IP ITL (UNSET_FLT = unset) */
    int32_t max_nonlin_it, max_lin_it, max_linesearch_cuts;
    int32_t precision;                 /* SW2GPU_FP64 / SW2GPU_MIXED */
    int32_t precond;                   /* SW2GPU_PREC_* */
    int32_t reserved;
    double  lin_rtol, lin_atol;        /* Krylov stop ||r||inf <= atol + rtol ||b||inf (ref: 1e-5, 1e-10) */
} sw2gpu_params;

typedef struct sw2gpu_stats {
    int32_t status;                    /* SW2GPU_OK or error code */
    int32_t newton_its;                /* nonlinear iterations of this call */
    int32_t linear_its;                /* total Krylov iterations of this call */
    int32_t linesearch_cuts;           /* total line-search halvings */
    double  resid_max, resid_l2, inc_max;   /* final norms (get_residual_norms) */
    double  device_ms;                 /* device time of the call (CUDA events) */
    int32_t kernel_launches;           /* kernels launched by the call */
    int32_t wd_elems;                  /* elements with wd_flag != 0 after the step */
    double  jac_ms;                    /* FD Jacobian element kernel (summed over Newton iterations) */
    double  krylov_ms;                 /* persistent BiCGSTAB kernel */
    double  resid_ms;                  /* residual element + gather kernels */
    double  other_ms;                  /* block gather, scaling, line search, init */
} sw2gpu_stats;

typedef struct sw2gpu_ctx sw2gpu_ctx;

/* Library / error info. */
int         sw2gpu_abi_version(void);
const char *sw2gpu_last_error(void);

/* Builds the device mesh, the BCSR pattern and the reference-order gather lists of the
 * atomic-free assembly (sw2gpu_prepare in the reference-side adapter; call again after every
 * mesh adaption).  `stream` is a cudaStream_t (NULL = a stream owned by the context). */
int sw2gpu_create(const sw2gpu_mesh *mesh, const sw2gpu_params *params, void *stream, sw2gpu_ctx **out);
int sw2gpu_destroy(sw2gpu_ctx *ctx);
/* After a mesh adaption (adpt_main, src/grid/adpt_main.c:17): the context of the adapted mesh,
 * made from `old`, which is released on success (*out replaces it; on failure `old` is kept and
 * still usable).  The adaption must keep node and triangle numbers (nodes and triangles
 * appended, some triangles' nodes changed, trailing triangles dropped, boundary edges changed),
 * as refinement does: then only the pattern rows of nodes that a changed, new or removed
 * element or edge touches are rebuilt and every other row is copied (a mesh with fewer nodes
 * is rebuilt from scratch), the tables equal those sw2gpu_create would make, and so do all
 * later results.  The new context keeps the stream, the parameters, dt, the launch variant, the
 * wait limits and the transport-output, mass-tracking and graph settings, and the three time
 * levels of the nodes both meshes have; new nodes start at 0 (set them with sw2gpu_set_state).
 * Wind and wave stresses are per node: set them again.  A context inside a batch, engine or
 * server is not remeshed. */
int sw2gpu_remesh(sw2gpu_ctx *old, const sw2gpu_mesh *mesh, sw2gpu_ctx **out);
/* Launch variants (no counterpart in the reference).  Two knobs change the speed of a step,
 * never its results: the register budget of the wet-Jacobian kernel (jac_minb: 1 or 2
 * resident CTAs per SM) and the depth of the Krylov kernel's shared-memory tile ring (stages:
 * 0 = sweeps read global memory, 2 or 3).  sw2gpu_autotune times every variant on the
 * context's own mesh and current state (which it leaves as it found it) and keeps the
 * fastest; a batch uses the variants of its instance with the most blocks. */
int sw2gpu_autotune(sw2gpu_ctx *ctx, int32_t *jac_minb, int32_t *stages);
int sw2gpu_set_variant(sw2gpu_ctx *ctx, int32_t jac_minb, int32_t stages);
int sw2gpu_get_variant(const sw2gpu_ctx *ctx, int32_t *jac_minb, int32_t *stages);
/* CUDA graphs for small meshes, where launches and host round trips are a large part of a
 * step (no counterpart in the reference).  enable = 1: sw2gpu_step replays the step start and
 * each Newton iteration as one graph launch each, the host reading the norms after each
 * iteration.  enable = 2: the whole step is one graph launch -- the Newton loop and the line
 * search are conditional WHILE nodes whose conditions single-thread control kernels set on the
 * device from the norms and the Krylov outcome (fe_newton's decisions, as direct stepping takes
 * them on the host), the failure reset an IF node -- and the host reads one status word per
 * step.  Graphs are captured at first use for each arrangement of the rotating state levels and
 * recaptured after a dt, variant or mass-tracking change.  Same kernels and results as direct
 * launches; phase times are not reported in graph mode.  0 = direct launches. */
int sw2gpu_set_graphs(sw2gpu_ctx *ctx, int32_t enable);
/* device memory the context holds (bytes); no counterpart in the reference */
int64_t sw2gpu_device_bytes(const sw2gpu_ctx *ctx);
/* Bounds of the device waits (no counterpart in the reference, whose solver runs on one CPU
 * thread): the Krylov kernel's grid barriers and its tile-copy waits give up after this many
 * polls, set SW2GPU_E_TIMEOUT and return; the step then resets the current level to the old
 * one, like a failed step, and the context stays usable.  0 = the library's defaults (2^23 and
 * 2^20 polls, a few seconds and about a second).  Failure-detection tests set a few polls to
 * make a wait run out without any fault. */
int sw2gpu_set_wait_limits(sw2gpu_ctx *ctx, int64_t barrier_polls, int64_t copy_polls);

/* State of time level `level` (0 = current t+dt iterate, 1 = old, 2 = older);
 * SW2 state is (head, vel.x, vel.y) as in src/structs/ssw_2d.h:13-18.  The library takes the
 * levels as given: a caller starting from a hot start passes levels with the Dirichlet node
 * values (DB OVH / OVL strings) already imposed on all three, as the reference's reader does
 * (src/structs/ssw.c:452-545); a raw hot start whose held depth differs from it gives results
 * that differ from the reference from the first Jacobian on. */
int sw2gpu_set_state(sw2gpu_ctx *ctx, int level, const double *h, const double *u, const double *v);
int sw2gpu_get_state(sw2gpu_ctx *ctx, int level, double *h, double *u, double *v);
int sw2gpu_get_wd_flag(sw2gpu_ctx *ctx, int32_t *wd_flag);
/* On-device output snapshot (for callers that keep their output on the GPU instead of writing
 * it through the host each step, as the reference's smodel_print_ts does,
 * src/structs/smodel.c:697): copies time level `level` into caller-owned DEVICE buffers of
 * nnodes doubles each (NULL skips a field).  The copies are ordered on the context's stream and
 * the call does not wait for them: they are complete once that stream has reached them (any
 * later blocking call of the library, or the caller's own synchronization of the stream). */
int sw2gpu_snapshot(sw2gpu_ctx *ctx, int level, double *d_h, double *d_u, double *d_v);
/* Overrides the element wet/dry flags (normally set by the step's fe_sw2_init). */
int sw2gpu_set_wd_flag(sw2gpu_ctx *ctx, const int32_t *wd_flag);

/* Wind surface stress (fe_sw2_body_resid.c:674-719 with swind_elem2d_get_local_stress,
 * src/structs/smeteor.c:241-306): stress_x / stress_y [nnodes] are the nodal wind values the
 * reference's meteor_update puts in winds[node].stress for the coming step; mat_flag[nmats] the
 * material's wind stress form (MP WND STR: 0 = the values are the stress, 1 = Wu's drag law of a
 * wind speed; the depth-dependent form 2 is not built and is rejected with SW2GPU_E_ARG) and
 * mat_windatt[nmats] its attenuation (MP WND ATT).  The element stress, the vertex average
 * scaled by windatt^2 / (3 density), enters the momentum residual of fully wet elements and
 * their SUPG strong momentum equations (:1049-1050).  Kept until the next call; stress_x = NULL
 * turns the term off (the default). */
int sw2gpu_set_wind(sw2gpu_ctx *ctx, const int32_t *mat_flag, const double *mat_windatt, const double *stress_x,
                    const double *stress_y);
/* Wave radiation stress (the same term, fe_sw2_body_resid.c:689-694, with
 * swave_elem2d_get_local_stress, src/structs/smeteor.c:312-327): rads_xx / rads_xy / rads_yy
 * [nnodes] are the nodal radiation stresses waves[node].rads the reference reads from the hot
 * file (WAVE_STRESS) or a wave station series.  The element stress is -sum_i grad(phi_i) . S_i and
 * adds to the wind stress.  The CSTORM coupled form (nodal stresses averaged) is not built.  Kept
 * until the next call; rads_xx = NULL turns the term off (the default). */
int sw2gpu_set_waves(sw2gpu_ctx *ctx, const double *rads_xx, const double *rads_xy, const double *rads_yy);

/* Mass-balance diagnostics (src/tools/tl_grid_mass.c), on the device.
 * sw2gpu_grid_mass: water mass of time level `level` times `density`
 * (tl_find_grid_mass_elem2d, :20-97; partially dry triangles by the h < 0 corner clip of
 * fe_3m2d_dry_wet_factornew, :289-346).
 * sw2gpu_mass_flux: the mass that entered the grid during the last step at the current level,
 * water sources minus boundary outflow (the per-step term tl_find_grid_mass_error_elem2d,
 * :102-159, adds to its running total; the caller keeps that total and forms
 * |mass - total - initial mass|).  Uses the last step's dt and series values.
 * Both add their terms in a fixed order: the same bits on every run and every GPU. */
int sw2gpu_grid_mass(sw2gpu_ctx *ctx, int level, double density, double *mass);
/* Adaption error indicator of the last step, on the device (ssw_2d_calculate_elem_error,
 * src/structs/ssw_2d.c:424-500, which fe_main calls after every accepted SW2 step and
 * adpt_main / error_main read, src/grid/error_main.c:2): per element the square root of the
 * summed squared steady continuity residuals at its vertices (current level against the old one,
 * the last step's dt) times its area, divided by refine_tol[material] (the reference's
 * refine_tolerance, MP SRT; one value per material id of the mesh), and 0.5 for elements with
 * wd_flag > 0.  elem_error[nelems2d]; node_error[nnodes] (may be NULL) the unscaled element
 * values averaged over each node's elements, the reference's sw->error. */
int sw2gpu_elem_error(sw2gpu_ctx *ctx, const double *refine_tol, double *elem_error, double *node_error);
int sw2gpu_mass_flux(sw2gpu_ctx *ctx, double density, double *flux);
/* The same two diagnostics for every accepted step, reduced inside sw2gpu_step (and a batch
 * step) on the step's stream after its Newton loop, with no launch or host round trip of their
 * own -- for callers that report mass every step, as the reference's SOUT MERROR does
 * (tl_find_grid_mass_error_elem2d after every step).  sw2gpu_step_mass returns the grid mass of
 * the new level and the step's flux, bitwise the values sw2gpu_grid_mass(ctx, 0, density) and
 * sw2gpu_mass_flux(ctx, density) give right after that step; SW2GPU_E_ARG if the last step was
 * not accepted or tracking is off.  Not part of the continuous-batching engine's ticks. */
int sw2gpu_set_mass_tracking(sw2gpu_ctx *ctx, int32_t enable, double density);
int sw2gpu_step_mass(sw2gpu_ctx *ctx, double *mass, double *flux);

/* Transport side output elem_rhs_dacont_extra_terms (src/fe/sw2/fe_sw2_body_resid.c:353-355,
 * :400, :1214): the continuity parts of shock capturing and SUPG per element vertex from the
 * last residual evaluation, which the reference keeps for its transport solve.  Off by default
 * (the residual kernel then skips it); sw2gpu_set_dacont(ctx, 1) allocates 24 B per element.
 * sw2gpu_get_dacont copies it vertex-major like the reference's [3][nelems2d] array:
 * out[i * nelems2d + e]; SW2GPU_E_ARG while it is off. */
int sw2gpu_set_dacont(sw2gpu_ctx *ctx, int32_t enable);
int sw2gpu_get_dacont(sw2gpu_ctx *ctx, double *out);

/* Constituent transport (fe_transport, src/fe/transport/fe_transport.c:31-113): general
 * constituents (CN CON, src/initio/read_bc_CN.c:14-18) carried by the flow, solved after every
 * accepted flow step on the flow's new, old and older levels, wd_flag and side output
 * elem_rhs_dacont_extra_terms (switched on by sw2gpu_set_transport).  Per constituent and Newton
 * iteration: the triangle and boundary-edge residuals (fe_2d_transport_body_resid.c:50-676,
 * fe_2d_transport_boundary_resid.c:37-300: wrapped wet/dry temporal and advection terms,
 * diffusion by MP DF or the estimated eddy viscosity, SUPG, the flow's extra continuity terms),
 * the scalar FD Jacobian (fe_transport_load.c:41-340), a Jacobi-preconditioned BiCGSTAB on the
 * device run to ||r||inf <= lin_atol + min(lin_rtol, 1e-12) ||b||inf (the reference solves each
 * transport system exactly with its profile LU), and the reference's Newton rules for a linear
 * problem (iterate while the residual max norm exceeds tol_nonlin).  Salinity and temperature (baroclinic coupling), the vorticity
 * constituent, sediment and quadrilaterals are not built.
 *   ref_conc[k]                  property[0]: boundary series values are divided by it
 *   diffusion[k * nmats + m]     MP DF d_m of material m
 *   str_bc_flag[k * nstrings + s] 0, SW2GPU_BCT_DIR (DB TRN: node string s holds the value of
 *                                series str_series[..] / ref_conc) or SW2GPU_BCT_NEU (NB TRN: water
 *                                entering through edge string s carries that value); DB TRN on an
 *                                edge string is rejected with SW2GPU_E_ARG (the reference's
 *                                boundary residual would read the string's unset NB TRN series)
 * sw2gpu_set_transport copies the description (NULL or ntransport = 0 turns transport off) and
 * starts every level at 0; sw2gpu_set_conc / sw2gpu_get_conc move a constituent's level
 * (0 current, 1 old, 2 older) as stored, i.e. as the hot start's ICON data set gives it. */
#define SW2GPU_BCT_DIR 1
#define SW2GPU_BCT_NEU 3
typedef struct sw2gpu_transport {
    int32_t ntransport;
    const double  *ref_conc;       /* [ntransport] */
    const double  *diffusion;      /* [ntransport * nmats] */
    const int32_t *str_bc_flag;    /* [ntransport * nstrings] */
    const int32_t *str_series;     /* [ntransport * nstrings] series id or -1 */
} sw2gpu_transport;
int sw2gpu_set_transport(sw2gpu_ctx *ctx, const sw2gpu_transport *transport);
int sw2gpu_set_conc(sw2gpu_ctx *ctx, int32_t itrn, int32_t level, const double *conc);
int sw2gpu_get_conc(sw2gpu_ctx *ctx, int32_t itrn, int32_t level, double *conc);
/* fe_transport after an accepted sw2gpu_step: every constituent in order (levels shifted, then
 * its Newton solve); `series` are the step values the flow step used, stats[ntransport] (may be
 * NULL).  Stops at the first constituent that fails with SW2GPU_E_NEWTON, _LINEAR, _NAN or
 * _TIMEOUT, its current level reset to the old one (fe_transport_init); the reference then
 * retries the whole time step with dt / 4, flow and transport shifting their levels again. */
int sw2gpu_transport_step(sw2gpu_ctx *ctx, const double *series, sw2gpu_stats *stats);
/* Hot-path pieces, for parity checks against the reference units: fe_transport_init of
 * constituent itrn at the current levels (current level from the old one, dry nodes 0, DB TRN
 * values); the residual resid[nnodes] (fe_transport_resid) and the scalar FD Jacobian
 * val[nnzb] over the context's pattern (fe_transport_load) at the current state. */
int sw2gpu_transport_init(sw2gpu_ctx *ctx, int32_t itrn, const double *series);
int sw2gpu_transport_load(sw2gpu_ctx *ctx, int32_t itrn, double *resid, double *val);
/* The constituents' adaption error indicator of the last step (scon_calculate_elem2d_error,
 * src/structs/scon.c:282-361, which fe_main calls right after the flow's indicator,
 * src/fe/fe_main.c:625-628): per element and constituent the steady transport residual at each
 * vertex less its element mean, as a root sum of squares times the area.  elem_error[nelems2d]
 * is in/out: each element keeps the largest of its value (pass the flow's, sw2gpu_elem_error)
 * and every constituent's error over refine_tol[itrn * nmats + material] (MP TRT);
 * node_error[ntransport * nnodes] (may be NULL) the constituents' element errors averaged over
 * each node's elements, the reference's con[itrn].error. */
int sw2gpu_transport_elem_error(sw2gpu_ctx *ctx, const double *refine_tol, double *elem_error, double *node_error);

/* One implicit time step: time-level shift (fe_sw2, src/fe/sw2/fe_sw2.c:43-50) then the
 * damped Newton loop (fe_newton).  `series` holds the step-averaged value of every BC
 * series over [t, t+dt] (sseries_setall_ts_valuesAVG).  On SW2GPU_E_NEWTON the current
 * state is reset to the old level (fe_sw2_init) and the caller retries with dt * 0.25. */
int sw2gpu_step(sw2gpu_ctx *ctx, double dt, const double *series, sw2gpu_stats *stats);

/* Hot-path pieces, for parity checks against the reference units:
 *   sw2gpu_resid: fe_sw2_init-free residual at the current state (fe_sw2_resid);
 *                 writes resid[3*nnodes] and applies the dry-node velocity zeroing.
 *   sw2gpu_load:  FD Jacobian (fe_sw2_load incl. the tiny-diagonal fix) in BCSR form:
 *                 row_ptr[nnodes+1], col[nnzb], val[9*nnzb] (sorted columns), and the
 *                 residual after the fix in resid[3*nnodes].  Pass NULL to query nnzb. */
int sw2gpu_set_dt(sw2gpu_ctx *ctx, double dt, const double *series);
int sw2gpu_resid(sw2gpu_ctx *ctx, double *resid);
int sw2gpu_load(sw2gpu_ctx *ctx, int32_t *nnzb, int32_t *row_ptr, int32_t *col, double *val, double *resid);

/* Linear solve of a given BCSR system with the device Krylov solver (solv_linear_sys_setup
 * + solv_linear_sys_solve): Jacobi scaling, preconditioned BiCGSTAB, unscaling.  The matrix
 * uses the pattern of the context. */
int sw2gpu_linear_solve(sw2gpu_ctx *ctx, const double *val, const double *rhs, double *x, int32_t *iterations);

/* Allocation-free linear solve.  No counterpart in the reference: it exists for callers
 * that own all of their GPU memory (a fixed arena sized at start-up, as a coupled model's
 * time loop or a serving process has) and cannot let a library call cudaMalloc during a
 * step, since that can synchronize the device, fail mid-run and escape their accounting.
 * Solves the 3x3-block CSR system (row_ptr[nnodes+1], col[nnzb], val[9*nnzb], rhs[3*nnodes]
 * -> x[3*nnodes], all DEVICE pointers owned by the caller) with the same Jacobi scaling and
 * block-Jacobi BiCGSTAB as sw2gpu_linear_solve; the stopping test is
 * ||r||inf <= atol + rtol ||M^-1 S rhs||inf.  Its only work memory is one file-scope device
 * array of about 16.7 MB that every GPU loading the library keeps until exit, so systems
 * above SW2GPU_NOALLOC_MAX_NODES rows or SW2GPU_NOALLOC_MAX_BLOCKS blocks are rejected with
 * SW2GPU_E_ARG.  The block structure is checked before the array is written: row_ptr[0] = 0,
 * row_ptr[nnodes] = nnzb, ordered row ranges, column indices in [0, nnodes) and exactly one
 * diagonal block per row, else SW2GPU_E_ARG.  The first call on a device looks up that array's device address (make it
 * before any stream capture).  All calls share the array: calls that overlap on the GPU
 * race and corrupt each other.  Returns SW2GPU_E_LINEAR if max_it is reached. */
#define SW2GPU_NOALLOC_MAX_NODES  16384
#define SW2GPU_NOALLOC_MAX_BLOCKS 131072
int sw2gpu_bcsr_solve_noalloc(int32_t nnodes, int32_t nnzb, const int32_t *row_ptr, const int32_t *col,
                              const double *val, const double *rhs, double *x, double rtol, double atol,
                              int32_t max_it, void *stream, int32_t *iterations);

/* Batched ensemble: many independent contexts stepped together, each Newton phase one
 * launch over all of them (element kernels: per group of up to 30 instances; the Krylov
 * solve: one cooperative launch, each instance on its own range of CTAs); every context
 * keeps its own data and gets bitwise the results it gets alone.  Steps launched directly
 * spread a Krylov solve over up to 4 launches as the engine does by default (see
 * sw2gpu_engine_set_rebalance); steps replayed from CUDA graphs keep one. */
typedef struct sw2gpu_batch sw2gpu_batch;
int sw2gpu_batch_create(sw2gpu_ctx **ctxs, int32_t n, void *stream, sw2gpu_batch **out);
int sw2gpu_batch_step(sw2gpu_batch *b, const double *dt, const double *const *series, sw2gpu_stats *stats);
int sw2gpu_batch_destroy(sw2gpu_batch *b);
/* Replay the batch's step start and every Newton iteration in which all instances iterate from
 * CUDA graphs, captured per arrangement of the instances' time levels, dt and launch variant
 * (the three most recent kept); iterations of a subset launch directly.  Each instance's Krylov
 * tolerance is read from device memory.  Bitwise the same as direct stepping; worth it for
 * batches of small meshes, whose steps are launch-bound. */
int sw2gpu_batch_set_graphs(sw2gpu_batch *b, int32_t enable);

/* Continuous batching (no counterpart in the reference, whose time loop runs one model).
 * Instances of uneven size join and leave an engine between ticks.  A tick starts a time
 * step for every instance between steps (step-averaged series, level shift, fe_sw2_init,
 * residual) and runs one Newton iteration for every instance inside a step, each phase as
 * one launch over all of them.  A failed step is retried with dt / 4 and dt doubles again
 * after every accepted step, up to the base dt, as the reference's time loop does (tc_scale,
 * tc_end); an instance computes exactly what sw2gpu_step computes for it alone.
 * The engine does not own the contexts; an instance that finished leaves the engine and is
 * reported by the tick. */
typedef struct sw2gpu_engine sw2gpu_engine;
typedef struct {
    int64_t id;
    int32_t status;      /* 0: nsteps completed; else the failure code of the last attempt (gave up) */
    int32_t steps;       /* completed time steps */
    int32_t failures;    /* failed step attempts (each retried with dt / 4) */
    int32_t newton_its;
    int32_t linear_its;
    int32_t ticks;       /* ticks the instance was in the engine */
    double t;            /* model time reached */
    double dt;           /* time step at the end */
} sw2gpu_run_stats;
int sw2gpu_engine_create(int32_t precision, void *stream, sw2gpu_engine **out);
/* nseries piecewise-linear series (the instance's BC series, ids as in the mesh): series_len[s]
 * points each, times and values concatenated in series order; averaged over every step.
 * max_retries: consecutive failed attempts allowed before the instance gives up. */
int sw2gpu_engine_add(sw2gpu_engine *e, sw2gpu_ctx *ctx, int64_t id, double t0, double dt, int32_t nsteps,
                      int32_t max_retries, int32_t nseries, const int32_t *series_len, const double *series_t,
                      const double *series_v);
/* finished: room for at least sw2gpu_engine_active(e) records */
int sw2gpu_engine_tick(sw2gpu_engine *e, sw2gpu_run_stats *finished, int32_t max_finished, int32_t *nfinished);
int32_t sw2gpu_engine_active(const sw2gpu_engine *e);
/* the last tick: device_ms and the phase times of sw2gpu_stats, kernel_launches, and in
 * newton_its the instances that ran a Newton iteration, in linear_its the largest Krylov
 * iteration count among them, in linesearch_cuts the instances that started a time step,
 * in wd_elems the instances in the engine */
int sw2gpu_engine_last_tick(const sw2gpu_engine *e, sw2gpu_stats *out);
/* Krylov rebalancing of the engine's launches (default 4 rounds, fraction 0.5): a batched
 * Krylov launch lasts as long as its slowest instance, so in every launch but the last of
 * `rounds`, once `fraction` of its CTAs have finished their instances, the instances still
 * iterating pause at an iteration boundary and the next launch shares all CTAs among them.
 * Results do not change (an instance's reductions depend only on its own partition, not on
 * its CTAs); rounds = 1 turns it off.  rounds in [1, 8], fraction in [0, 1]. */
int sw2gpu_engine_set_rebalance(sw2gpu_engine *e, int32_t rounds, double fraction);
int sw2gpu_engine_destroy(sw2gpu_engine *e);

/* Request server (no counterpart in the reference): a request loop in the library.  Each
 * submitted solve -- mesh, parameters, initial state, series, number of steps -- is copied,
 * queued and admitted in arrival order when its device bytes fit the budget (a fraction of
 * the device memory free at creation; a request that fits no budget is admitted alone).
 * Loader threads build admitted requests' contexts while a worker thread ticks a
 * continuous-batching engine, so requests that arrive while others run share their launches
 * and every solve keeps its state on the device between steps.  Results and per-request
 * times are collected with sw2gpu_server_wait.  One precision per server. */
typedef struct sw2gpu_server sw2gpu_server;
#define SW2GPU_PENDING 100   /* sw2gpu_server_wait: not finished within the timeout */
typedef struct {
    int64_t id;
    int32_t status;       /* 0: all steps done */
    int32_t steps, failures, newton_its, linear_its;
    int32_t reserved;
    double t;             /* model time reached */
    double queue_ms;      /* submit -> admitted */
    double run_ms;        /* admitted -> finished (context build, steps, result copy) */
    double latency_ms;    /* submit -> finished */
    int64_t device_bytes; /* device memory the request held */
} sw2gpu_request_stats;
int sw2gpu_server_create(int32_t precision, double hbm_fraction, int32_t max_active, sw2gpu_server **out);
/* series as for sw2gpu_engine_add; *id receives the request id */
int sw2gpu_server_submit(sw2gpu_server *s, const sw2gpu_mesh *mesh, const sw2gpu_params *params,
                         const double *h0, const double *u0, const double *v0, double t0, double dt,
                         int32_t nsteps, int32_t nseries, const int32_t *series_len, const double *series_t,
                         const double *series_v, int64_t *id);
/* waits up to timeout_s; on completion fills st and the final state (nnodes each, may be NULL)
 * and forgets the request; SW2GPU_PENDING if still running */
int sw2gpu_server_wait(sw2gpu_server *s, int64_t id, double timeout_s, sw2gpu_request_stats *st, double *h,
                       double *u, double *v);
int sw2gpu_server_status(sw2gpu_server *s, int32_t *queued, int32_t *active, int64_t *bytes_in_use,
                         int64_t *budget);
/* stops both threads; requests not finished are dropped */
int sw2gpu_server_destroy(sw2gpu_server *s);

#ifdef __cplusplus
}
#endif
#endif /* SW2GPU_H */
