// trn_kernels.cuh -- the kernels of one constituent's transport Newton iteration (fe_transport,
// src/fe/transport/fe_transport.c:31-113) on the flow's mesh:
//
//   k_trn_init           fe_transport_init: current level from the old one, dry nodes 0, held
//                        nodes at their series value, bc_mask
//   k_trn_elem<JAC>      per triangle and boundary edge: the residual (JAC = false) or the
//                        scalar FD Jacobian (JAC = true, 2 evaluations per vertex) into per-element
//                        slots, numbered as the flow's (triangle e, vertex i: 3 e + i; block (a, b):
//                        9 e + 3 a + b; edges after the triangles)
//   k_trn_resid_gather   per node: slots summed in reference element order, held rows 0, entries
//                        below SMALL zeroed, and the residual norms of get_residual_norms
//   k_trn_jac_gather     per row: blocks summed in reference element order, the tiny-diagonal fix,
//                        and the Jacobi-folded operator D^-1 A (unit diagonal) for the Krylov solve
//   k_trn_bicgstab       persistent cooperative BiCGSTAB on the folded operator
//   k_trn_inc            fe_transport_inc and the line search's half steps
#pragma once
#include "trn_physics.cuh"

namespace sw2 {

struct TrnArgs {
    DevMesh m;                          // the flow's mesh, gather lists and pattern
    const double *h, *u, *v, *ho, *hoo; // the flow's levels after its step
    const int* wd;
    const double* dac;                  // [3][T] the flow's side output, vertex-major
    double* c;                          // the constituent's current level
    const double *co, *coo;             // its old and older levels
    const int* node_str;                // [V] node string or -1
    const int* tbc;                     // [S] the constituent's bc flag per string
    const double* tsval;                // [S] step value of the string's series over property[0]
    const double* tdm;                  // [M] MP DF d_m
    double refc;                        // property[0]
    unsigned char* mask;                // [V] bc_mask (held nodes)
    double *rslot, *jslot;              // [3T + 2E], [9T + 4E]
    double *R, *sol;                    // [V]
    double *aoff, *dinv, *val;          // [nnzb - V], [V], [nnzb] (val may be null)
    Norms *npart, *norms;
    unsigned* ncounter;
    TrnParams P;
};

constexpr int kTrnThreads = 128;

__device__ __forceinline__ bool trn_held(const TrnArgs& A, int n) {
    const int s = A.node_str[n];
    return s >= 0 && A.tbc[s] == kTrnBctDir;
}

__global__ void __launch_bounds__(kTrnThreads) k_trn_init(const __grid_constant__ TrnArgs A) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.m.V) return;
    double c = A.co[n];
    if (A.h[n] <= kNotQuiteSmall) c = 0.0;
    unsigned char held = 0;
    if (trn_held(A, n)) {
        held = 1;
        c = A.tsval[A.node_str[n]];
    }
    A.c[n] = c;
    A.mask[n] = held;
}

__device__ __forceinline__ void trn_load_elem(const TrnArgs& A, int e, TrnElem& E, int* n) {
    const DevMesh& m = A.m;
    n[0] = m.en0[e];
    n[1] = m.en1[e];
    n[2] = m.en2[e];
    E.dir = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int k = n[i];
        E.x[i] = m.x[k];
        E.y[i] = m.y[k];
        E.h[i] = A.h[k];
        E.ho[i] = A.ho[k];
        E.hoo[i] = A.hoo[k];
        E.u[i] = A.u[k];
        E.v[i] = A.v[k];
        E.co[i] = A.co[k];
        E.coo[i] = A.coo[k];
        E.dac[i] = A.dac[(size_t)i * m.T + e];
        if (trn_held(A, k)) E.dir |= 1u << i;
    }
    E.djac = m.djac[e];
    E.gx[0] = m.gx0[e]; E.gy[0] = m.gy0[e];
    E.gx[1] = m.gx1[e]; E.gy[1] = m.gy1[e];
    E.gx[2] = m.gx2[e]; E.gy[2] = m.gy2[e];
    const int mat = m.emat[e];
    const MatParams M = m.mats[mat];
    E.ks = M.ks;
    E.eev_coef = M.eev_coef;
    E.eev_mode = M.eev_mode;
    E.dm = A.tdm[mat];
    E.wd = A.wd[e];
}

__device__ __forceinline__ void trn_load_edge(const TrnArgs& A, int j, TrnEdge& B, int* n) {
    const DevMesh& m = A.m;
    n[0] = m.bn0[j];
    n[1] = m.bn1[j];
    B.dir = 0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int k = n[i];
        B.h[i] = A.h[k];
        B.u[i] = A.u[k];
        B.v[i] = A.v[k];
        if (trn_held(A, k)) B.dir |= 1u << i;
    }
    B.djac = m.bdjac[j];
    B.nx = m.bnx[j];
    B.ny = m.bny[j];
    const int s = m.bstr[j];
    B.kind = m.bkind[j];
    B.cflag = A.tbc[s];
    B.flux_in = m.str_value[s];
    B.c_user = A.tsval[s];
}

// residual (JAC = false) or Jacobian (JAC = true) of one triangle or boundary edge per thread;
// the residual skips triangles whose wd_flag is neither 0 nor 1 (their slots hold 0), the
// Jacobian covers them all (fe_transport_resid.c:131-133, fe_transport_load.c:79-81)
template <bool JAC>
__global__ void __launch_bounds__(kTrnThreads) k_trn_elem(const __grid_constant__ TrnArgs A) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    const int T = A.m.T, E = A.m.E;
    if (w < T) {
        TrnElem el;
        int n[3];
        trn_load_elem(A, w, el, n);
        double c[3];
#pragma unroll
        for (int i = 0; i < 3; i++) c[i] = A.c[n[i]];
        if (!JAC) {
            double er[3] = {0, 0, 0};
            if (el.wd == 0 || el.wd == 1) {
                TrnPre pre;
                trn_prepare(el, A.P, pre);
                trn_elem_resid(el, pre, c, A.P, er);
            }
#pragma unroll
            for (int i = 0; i < 3; i++) A.rslot[3 * (size_t)w + i] = er[i];
        } else {
            TrnPre pre;
            trn_prepare(el, A.P, pre);
            double M[9];
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const double eps = trn_eps(c[i], A.refc);
                double cp[3] = {c[0], c[1], c[2]}, cm[3] = {c[0], c[1], c[2]};
                cp[i] += 1 * eps;
                cm[i] += -1 * eps;
                double rp[3], rm[3];
                trn_elem_resid(el, pre, cp, A.P, rp);
                trn_elem_resid(el, pre, cm, A.P, rm);
#pragma unroll
                for (int k = 0; k < 3; k++) M[i + 3 * k] = (rp[k] - rm[k]) / (2.0 * eps);   // elem_matrix_deriv_1dof
            }
#pragma unroll
            for (int q = 0; q < 9; q++) A.jslot[9 * (size_t)w + q] = fabs(M[q]) > kSmall ? M[q] : 0.0;
        }
    } else if (w < T + E) {
        const int j = w - T;
        TrnEdge B;
        int n[2];
        trn_load_edge(A, j, B, n);
        double c[2] = {A.c[n[0]], A.c[n[1]]};
        if (!JAC) {
            double er[2];
            trn_edge_resid(B, c, A.P.dt, er);
            A.rslot[3 * (size_t)T + 2 * j] = er[0];
            A.rslot[3 * (size_t)T + 2 * j + 1] = er[1];
        } else {
            double M[4];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const double eps = trn_eps(c[i], A.refc);
                double cp[2] = {c[0], c[1]}, cm[2] = {c[0], c[1]};
                cp[i] += 1 * eps;
                cm[i] += -1 * eps;
                double rp[2], rm[2];
                trn_edge_resid(B, cp, A.P.dt, rp);
                trn_edge_resid(B, cm, A.P.dt, rm);
#pragma unroll
                for (int k = 0; k < 2; k++) M[i + 2 * k] = (rp[k] - rm[k]) / (2.0 * eps);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) A.jslot[9 * (size_t)T + 4 * j + q] = fabs(M[q]) > kSmall ? M[q] : 0.0;
        }
    }
}

// fixed-order block reduction of (max, sum, max, count) (the flow's block_reduce3)
__global__ void __launch_bounds__(kGatherThreads) k_trn_resid_gather(const __grid_constant__ TrnArgs A) {
    const DevMesh& m = A.m;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = gridDim.x;
    double rmax = 0.0, l2 = 0.0, imax = 0.0;
    int nan = 0;
    if (n < m.V) {
        double acc = 0.0;
        for (int k = m.slot_ptr[n]; k < m.slot_ptr[n + 1]; k++) acc += A.rslot[m.slot_idx[k]];
        double r = A.mask[n] ? 0.0 : -acc;
        if (fabs(r) < kSmall) r = 0.0;
        A.R[n] = r;
        if (fmin(A.h[n], A.ho[n]) > 0) {   // include_node_in_residual (fe_newton.c:177-188)
            rmax = fabs(r);
            imax = fabs(A.sol[n]);
        }
        l2 = r * r;
        nan = isnan(r) ? 1 : 0;
    }
    block_reduce3<kGatherThreads>(rmax, l2, imax, nan);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        A.npart[blockIdx.x] = Norms{rmax, l2, imax, nan, 0};
        __threadfence();
        last = (atomicAdd(A.ncounter, 1u) == (unsigned)nb - 1u);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double a = 0.0, b = 0.0, c = 0.0;
        int d = 0;
        for (int k = threadIdx.x; k < nb; k += blockDim.x) {
            a = fmax(a, __ldcg(&A.npart[k].rmax));
            b += __ldcg(&A.npart[k].l2sum);
            c = fmax(c, __ldcg(&A.npart[k].imax));
            d += __ldcg(&A.npart[k].nan);
        }
        block_reduce3<kGatherThreads>(a, b, c, d);
        if (threadIdx.x == 0) {
            *A.norms = Norms{a, b, c, d, 0};
            *A.ncounter = 0u;
        }
    }
}

// one row per thread: the pattern's values (element blocks in reference order), the diagonal
// raised to NOT_QUITE_SMALL when below it (check_matrix_diagonal_for_nonexistant_entries,
// tl_matrix.c:59-67), and the row of D^-1 A without its unit diagonal
__global__ void __launch_bounds__(kTrnThreads) k_trn_jac_gather(const __grid_constant__ TrnArgs A) {
    const DevMesh& m = A.m;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.V) return;
    const int k0 = m.rowptr[i], k1 = m.rowptr[i + 1], kd = m.dpos[i];
    double d = 0.0;
    for (int c = m.blk_ptr[kd]; c < m.blk_ptr[kd + 1]; c++) d += A.jslot[m.blk_src[c]];
    if (fabs(d) < kNotQuiteSmall) d = kNotQuiteSmall;
    const double di = 1.0 / d;
    A.dinv[i] = di;
    if (A.val) A.val[kd] = d;
    for (int k = k0; k < k1; k++) {
        if (k == kd) continue;
        double a = 0.0;
        for (int c = m.blk_ptr[k]; c < m.blk_ptr[k + 1]; c++) a += A.jslot[m.blk_src[c]];
        if (A.val) A.val[k] = a;
        A.aoff[k - i - (k > kd ? 1 : 0)] = a * di;
    }
}

// mode 0: c += sol, then sol = -sol (fe_newton.c:563-590); mode 1: the line search's
// sol *= 0.5, c += sol (:668-672)
__global__ void __launch_bounds__(kTrnThreads) k_trn_inc(double* __restrict__ c, double* __restrict__ sol, int V,
                                                         int mode) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= V) return;
    double s = sol[n];
    if (mode == 1) s *= 0.5;
    c[n] += s;
    sol[n] = mode == 0 ? -s : s;
}

// the constituents' adaption error indicator (scon_calculate_elem2d_error, src/structs/scon.c:
// 282-361), one constituent per launch: per element the steady transport residual at each vertex
// less its element mean, as a root sum of squares times the area (raw[e]), and elem[e] raised to
// raw / refine_tol of the element's material where that is larger (max over the constituents and
// whatever elem held before, the flow's indicator in fe_main's order, src/fe/fe_main.c:625-628)
__global__ void __launch_bounds__(kTrnThreads) k_trn_elem_error(const __grid_constant__ DevMesh m,
                                                                const double* __restrict__ h,
                                                                const double* __restrict__ u,
                                                                const double* __restrict__ v,
                                                                const double* __restrict__ c,
                                                                const double* __restrict__ co, double dt,
                                                                const double* __restrict__ tol,
                                                                double* __restrict__ raw,
                                                                double* __restrict__ elem) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.T) return;
    const int n[3] = {m.en0[e], m.en1[e], m.en2[e]};
    const double gx[3] = {m.gx0[e], m.gx1[e], m.gx2[e]}, gy[3] = {m.gy0[e], m.gy1[e], m.gy2[e]};
    double hh[3], uu[3], vv[3], cc[3], cp[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        hh[i] = h[n[i]];
        uu[i] = u[n[i]];
        vv[i] = v[n[i]];
        cc[i] = c[n[i]];
        cp[i] = co[n[i]];
    }
    double dudx = 0., dvdy = 0., dcdx = 0., dcdy = 0.;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        dudx += gx[i] * uu[i];
        dvdy += gy[i] * vv[i];
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        dcdx += gx[i] * cc[i];
        dcdy += gy[i] * cc[i];
    }
    double coef[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
        coef[i] = hh[i] * (cc[i] - cp[i]) / dt + uu[i] * hh[i] * dcdx + hh[i] * cc[i] * dudx + hh[i] * vv[i] * dcdy +
                  hh[i] * cc[i] * dvdy;
    double err = (1. / 3.) * (coef[0] + coef[1] + coef[2]);
#pragma unroll
    for (int i = 0; i < 3; i++) {
        coef[i] -= err;
        coef[i] = coef[i] * coef[i];
    }
    err = sqrt(coef[0] + coef[1] + coef[2]) * m.djac[e];
    raw[e] = err;
    const double scaled = err / tol[m.emat[e]];
    if (scaled > elem[e]) elem[e] = scaled;
}

// ---------------------------------------------------------------------------------
// Persistent cooperative BiCGSTAB on the folded operator A' = D^-1 A (unit diagonal) with
// b' = D^-1 R, from x = 0; stops when ||r||inf <= atol + rtol ||b'||inf or after max_it
// iterations.  CTA b owns a contiguous range of rows.  Every dot product and norm is reduced in
// a fixed order: per-CTA partials (a fixed warp tree) to global slots, then after the grid
// barrier every CTA sums the slots in CTA order with one warp, so all CTAs hold the same bits.
// Three grid barriers per iteration, one per reduction, and none for a product's input alone:
//   sweep 1  p = r + beta q, Ar = A'r, v = Ar + beta A'q   (A'p without p complete; q = p - omega v)
//            rhat.v                                         -- barrier
//   sweep 2  s = r - alpha v, t = Ar - alpha A'v            (A's without s complete)
//            t.s, t.t, rhat.s, rhat.t                       -- barrier
//   update   x += alpha p + omega s, r = s - omega t, q = p - omega v, max |r|
//            (rhat.r_new = rhat.s - omega rhat.t comes with the sweep-2 sums)  -- barrier
// The barriers are bounded (grid_sync): a wait that runs out sets ctl->err and every CTA returns.
// one CTA of 1024 threads per SM (measured on the 1M-triangle basin: 43 us per iteration, against
// 47-52 us for 256- and 512-thread CTAs at one to four per SM)
constexpr int kTrnKThreads = 1024;
constexpr double kTrnKrylovRtol = 1e-12;   // relative stop of the transport Krylov solve (at most)
constexpr int kTrnKVectors = 8;   // r, rhat, p, v, s, t, q, Ar

struct TrnKrylovArgs {
    int V;
    const int *orowptr, *ocol;
    const double *aoff, *dinv, *R;
    double* x;                    // the solution (the Newton increment)
    double* vec[kTrnKVectors];
    double* part;                 // [3][4][nblocks] reduction slots
    KrylovCtl* ctl;
    double rtol, atol;
    int max_it;
    long long spin_limit;
};

// A'y at row i: unit diagonal plus the folded off-diagonal row
__device__ __forceinline__ double trn_amult(const TrnKrylovArgs& K, const double* __restrict__ y, int i) {
    double s = y[i];
    for (int k = K.orowptr[i]; k < K.orowptr[i + 1]; k++) s += K.aoff[k] * y[K.ocol[k]];
    return s;
}
// A'y and A'z at row i in one pass over the row
__device__ __forceinline__ void trn_amult2(const TrnKrylovArgs& K, const double* __restrict__ y,
                                           const double* __restrict__ z, int i, double& ay, double& az) {
    double a = y[i], b = z[i];
    for (int k = K.orowptr[i]; k < K.orowptr[i + 1]; k++) {
        const double w = K.aoff[k];
        const int j = K.ocol[k];
        a += w * y[j];
        b += w * z[j];
    }
    ay = a;
    az = b;
}

// fixed-order CTA reduction of up to four values into slot[q][blockIdx.x] (max for `ismax`)
template <int THREADS, int NV>
__device__ __forceinline__ void trn_cta_reduce(double (&a)[NV], const bool (&ismax)[NV], double* slot, int nb) {
    __shared__ double red[THREADS / 32][4];
#pragma unroll
    for (int q = 0; q < NV; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_xor_sync(0xffffffffu, a[q], o);
            a[q] = ismax[q] ? fmax(a[q], t) : a[q] + t;
        }
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) red[wid][q] = a[q];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double s = red[0][q];
            for (int w = 1; w < THREADS / 32; w++) s = ismax[q] ? fmax(s, red[w][q]) : s + red[w][q];
            slot[(size_t)q * nb + blockIdx.x] = s;
        }
    }
}

// every CTA: the global values of the slots (lane-strided partial sums, then a fixed xor tree)
template <int NV>
__device__ __forceinline__ void trn_grid_values(const double* slot, const bool (&ismax)[NV], int nb, double (&g)[NV]) {
    __shared__ double out[4];
    if (threadIdx.x < 32) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double s = 0.0;
            for (int k = threadIdx.x; k < nb; k += 32) {
                const double v = __ldcg(slot + (size_t)q * nb + k);
                s = ismax[q] ? fmax(s, v) : s + v;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double t = __shfl_xor_sync(0xffffffffu, s, o);
                s = ismax[q] ? fmax(s, t) : s + t;
            }
            if (threadIdx.x == 0) out[q] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) g[q] = out[q];
    __syncthreads();
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_trn_bicgstab(const __grid_constant__ TrnKrylovArgs K) {
    const int nb = gridDim.x;
    const int V = K.V;
    const int r0 = (int)((long long)V * blockIdx.x / nb), r1 = (int)((long long)V * (blockIdx.x + 1) / nb);
    double *r = K.vec[0], *rh = K.vec[1], *p = K.vec[2], *v = K.vec[3], *s = K.vec[4], *t = K.vec[5],
           *q = K.vec[6], *ar = K.vec[7];
    double* slotA = K.part;                    // rhat . v
    double* slotB = K.part + 4 * (size_t)nb;   // t . s, t . t, rhat . s, rhat . t
    double* slotC = K.part + 8 * (size_t)nb;   // max |r| (at the start: rhat . r, max |b'|)
    const long long lim = K.spin_limit > 0 ? K.spin_limit : kBarrierSpinLimit;
    unsigned epoch = 0;
    // start: r = b' = D^-1 R, rhat = r, x = 0, q = 0
    {
        double acc[2] = {0.0, 0.0};
        const bool m0[2] = {false, true};
        for (int i = r0 + threadIdx.x; i < r1; i += THREADS) {
            const double b = K.dinv[i] * K.R[i];
            r[i] = b;
            rh[i] = b;
            K.x[i] = 0.0;
            q[i] = 0.0;
            acc[0] += b * b;
            acc[1] = fmax(acc[1], fabs(b));
        }
        trn_cta_reduce<THREADS, 2>(acc, m0, slotC, nb);
    }
    if (!grid_sync(K.ctl, nb, epoch, lim)) return;
    double rho, bnorm;
    {
        double g0[2];
        const bool m0[2] = {false, true};
        trn_grid_values<2>(slotC, m0, nb, g0);
        rho = g0[0];
        bnorm = g0[1];
    }
    double rnorm = bnorm, beta = 0.0;
    const double stop = K.atol + bnorm * K.rtol;
    int it = 0, conv = rnorm <= stop ? 1 : 0;
    const bool mS1[1] = {false}, mS4[4] = {false, false, false, false}, mM1[1] = {true};
    while (!conv && it < K.max_it) {
        // sweep 1
        double a1[1] = {0.0};
        for (int i = r0 + threadIdx.x; i < r1; i += THREADS) {
            double av, aq = 0.0;
            if (beta != 0.0) trn_amult2(K, r, q, i, av, aq);
            else av = trn_amult(K, r, i);
            const double vv = beta != 0.0 ? av + beta * aq : av;
            p[i] = r[i] + beta * q[i];
            ar[i] = av;
            v[i] = vv;
            a1[0] += rh[i] * vv;
        }
        trn_cta_reduce<THREADS, 1>(a1, mS1, slotA, nb);
        if (!grid_sync(K.ctl, nb, epoch, lim)) return;
        double g1[1];
        trn_grid_values<1>(slotA, mS1, nb, g1);
        if (!(g1[0] != 0.0)) break;
        const double alpha = rho / g1[0];
        // sweep 2
        double a2[4] = {0.0, 0.0, 0.0, 0.0};
        for (int i = r0 + threadIdx.x; i < r1; i += THREADS) {
            const double ss = r[i] - alpha * v[i];
            const double tt = ar[i] - alpha * trn_amult(K, v, i);
            s[i] = ss;
            t[i] = tt;
            const double rr = rh[i];
            a2[0] += tt * ss;
            a2[1] += tt * tt;
            a2[2] += rr * ss;
            a2[3] += rr * tt;
        }
        trn_cta_reduce<THREADS, 4>(a2, mS4, slotB, nb);
        if (!grid_sync(K.ctl, nb, epoch, lim)) return;
        double g2[4];
        trn_grid_values<4>(slotB, mS4, nb, g2);
        if (!(g2[1] > 0.0)) break;
        const double omega = g2[0] / g2[1];
        const double rho_new = g2[2] - omega * g2[3];
        // update
        double a3[1] = {0.0};
        for (int i = r0 + threadIdx.x; i < r1; i += THREADS) {
            const double pi = p[i], si = s[i], ti = t[i];
            K.x[i] += alpha * pi + omega * si;
            const double rr = si - omega * ti;
            r[i] = rr;
            q[i] = pi - omega * v[i];
            a3[0] = fmax(a3[0], fabs(rr));
        }
        trn_cta_reduce<THREADS, 1>(a3, mM1, slotC, nb);
        if (!grid_sync(K.ctl, nb, epoch, lim)) return;
        double g3[1];
        trn_grid_values<1>(slotC, mM1, nb, g3);
        it++;
        rnorm = g3[0];
        conv = rnorm <= stop ? 1 : 0;
        if (!(rho_new != 0.0) || !(omega != 0.0)) break;
        beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        K.ctl->iterations = it;
        K.ctl->converged = conv;
        K.ctl->rnorm = rnorm;
        K.ctl->bnorm = bnorm;
    }
}

}  // namespace sw2
