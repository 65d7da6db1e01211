// newton_ctl.cuh -- the Newton loop's control on the device, for a time step replayed as one CUDA
// graph whose loops are conditional WHILE nodes (sw2gpu_set_graphs(ctx, 2)).
//
// The decisions are fe_newton's (src/fe/fe_newton.c:426-912) as the host takes them in direct
// stepping (newton_begin / newton_eta / newton_finish / newton_status of sw2gpu.cu), moved into
// single-thread kernels that read the residual norms and the Krylov outcome from device memory and
// set the loops' conditions with cudaGraphSetConditional:
//
//   k_ctl_begin   after the step's first residual: norms, state reset     -> Newton loop condition
//   k_ctl_eta     the iteration's Krylov tolerance (inexact Newton) into the device slot the Krylov
//                 kernel reads, and the l2 norm the line search compares against
//   k_ctl_after   after Jacobian, Krylov, update and residual: the solve's outcome, the norms
//                                                                       -> line-search condition
//   k_ctl_ls      after a halved increment and its residual             -> line-search condition
//   k_ctl_end     the convergence test                                  -> Newton loop condition
//   k_ctl_final   the step's status                                     -> reset condition
//
// Same arithmetic, same order as the host's, so a step replayed this way gives the bits of a
// direct step; the host reads one status word (and the statistics) per step.
#pragma once
#include <cuda_runtime.h>

namespace sw2 {

struct NewtonParams {
    double tol_nonlin, inc_nonlin, lin_rtol, eta_ntl, accept_rel;
    int max_nonlin_it, max_ls_cuts, mixed, V;
};

struct NewtonCtl {              // fe_newton's state of one step (NState of the host loop)
    double rmax, l2, imax, old_l2, eta;
    int it, lin, cuts, cuts_total;
    int ok, nan, done, timeout, status;
    int its_at[8];              // Krylov iterations of each Newton iteration (batch CTA shares)
};

__device__ __forceinline__ void ctl_norms(NewtonCtl* s, const Norms* nm, int V) {
    s->rmax = nm->rmax;
    s->l2 = sqrt(nm->l2sum / (3.0 * V));
    s->imax = nm->imax;
}

__device__ __forceinline__ bool ctl_ls_go(const NewtonCtl* s, const NewtonParams& P) {
    return s->rmax > P.tol_nonlin && s->l2 > s->old_l2 && s->cuts < P.max_ls_cuts;
}

__global__ void k_ctl_begin(NewtonCtl* s, const NewtonParams P, const Norms* nm, cudaGraphConditionalHandle hN) {
    NewtonCtl z = {};
    *s = z;
    ctl_norms(s, nm, P.V);
    s->ok = 1;
    if (nm->nan) {
        s->nan = 1;
        s->ok = 0;
        s->done = 1;
    }
    cudaGraphSetConditional(hN, s->done ? 0u : 1u);
}

__global__ void k_ctl_eta(NewtonCtl* s, const NewtonParams P, double* eta_dev) {
    const double eta = fmin(1e-5, fmax(P.lin_rtol, P.eta_ntl * P.tol_nonlin / fmax(s->rmax, 1e-300)));
    s->eta = eta;
    *eta_dev = eta;
    s->old_l2 = s->l2;
}

__global__ void k_ctl_after(NewtonCtl* s, const NewtonParams P, const Norms* nm, const KrylovCtl* kc,
                            cudaGraphConditionalHandle hL) {
    if (kc->err) {   // a Krylov wait ran out: the step ends with SW2GPU_E_TIMEOUT
        s->timeout = 1;
        s->ok = 0;
        s->done = 1;
        cudaGraphSetConditional(hL, 0u);
        return;
    }
    s->lin += kc->iterations;
    s->its_at[min(s->it, 7)] = max(kc->iterations, 1);
    // the plain path fails the step when BiCGSTAB hits max_lin_it without a useful reduction
    // (solv_bcgstab.c:280-292); the mixed path accepts its last iterate
    if (!kc->converged && !P.mixed && !(kc->rnorm <= P.accept_rel * kc->bnorm)) s->ok = 0;
    ctl_norms(s, nm, P.V);
    if (nm->nan || isnan(s->l2) || isinf(s->l2)) {
        s->ok = 0;
        s->nan = 1;
    }
    s->cuts = 0;
    cudaGraphSetConditional(hL, ctl_ls_go(s, P) ? 1u : 0u);   // line search (fe_newton.c:692-747)
}

__global__ void k_ctl_ls(NewtonCtl* s, const NewtonParams P, const Norms* nm, cudaGraphConditionalHandle hL) {
    ctl_norms(s, nm, P.V);
    s->cuts++;
    cudaGraphSetConditional(hL, ctl_ls_go(s, P) ? 1u : 0u);
}

__global__ void k_ctl_end(NewtonCtl* s, const NewtonParams P, cudaGraphConditionalHandle hN) {
    s->cuts_total += s->cuts;
    if (!s->timeout) s->it++;
    const bool keep = !s->timeout && s->ok && s->it < P.max_nonlin_it && s->rmax < 1.0E+20 &&
                      (s->rmax > P.tol_nonlin && s->imax > P.inc_nonlin);
    if (!keep) s->done = 1;
    cudaGraphSetConditional(hN, keep ? 1u : 0u);
}

// the step's status (newton_status; SW2GPU_E_TIMEOUT after a Krylov wait ran out) and whether the
// current level goes back to the old one
__global__ void k_ctl_final(NewtonCtl* s, const NewtonParams P, int e_nan, int e_linear, int e_newton, int e_timeout,
                            cudaGraphConditionalHandle hF) {
    int st = 0;
    if (s->timeout) st = e_timeout;
    else if (!s->ok || (s->rmax > P.tol_nonlin && s->imax > P.inc_nonlin) || s->rmax >= 1.0E+20)
        st = s->nan ? e_nan : (!s->ok ? e_linear : e_newton);
    s->status = st;
    cudaGraphSetConditional(hF, st != 0 ? 1u : 0u);
}

}  // namespace sw2
