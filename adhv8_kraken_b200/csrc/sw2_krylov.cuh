// sw2_krylov.cuh -- the linear solve of one Newton iteration as ONE persistent kernel.
//
// Restates solv_bcgstab (src/solver/solv_bcgstab.c:39-301) on the Jacobi-scaled
// system A' = S A S, b' = S R (spv_jacobi), left-preconditioned by M^-1, with the
// reference's stopping test ||r||inf <= atol + rtol ||M^-1 b'||inf and its initial
// guess u = M^-1 b'.  M is the 3x3 block-Jacobi inverse (the reference factors
// OP BLK node blocks exactly; any M that converges gives the same Newton result).
//
// One cooperative launch runs the whole iteration: phases are grid-stride loops over
// node rows separated by a bounded grid barrier; every dot product / norm is a
// per-block partial reduced by every block in the same fixed order, so all blocks
// take identical control decisions and reruns are bitwise identical.  s = r - alpha Ap
// is never stored: the second SpMV forms it on the fly from r and Ap.
// On exit the kernel applies the Newton increment: x = S u, state += x (fe_sw2_inc),
// sol = -x (fe_newton.c:561-585).
#pragma once
#include <cuda_runtime.h>

namespace sw2 {

constexpr int kKrylovThreads = 256;
constexpr long long kBarrierSpinLimit = 1ll << 26;   // bounded wait (~seconds), then error
constexpr int kStall = 40;                           // iterations without a new best residual

struct KrylovCtl {
    unsigned count;       // barrier arrival counter
    unsigned gen;         // barrier generation
    int err;              // 1 = a barrier wait ran out
    int iterations;
    int converged;        // 1 = stopping test met, 0 = hit max_lin_it
    int pad;
    double rnorm, bnorm;
};

// Grid barrier with a bounded spin.  Returns false (and sets ctl->err) if any block
// gave up; the caller then returns, so the kernel always terminates.
__device__ __forceinline__ bool grid_sync(KrylovCtl* ctl) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &ctl->gen;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&ctl->count, 1u) + 1u;
        if (arrived == gridDim.x) {
            ctl->count = 0u;
            __threadfence();
            atomicAdd(&ctl->gen, 1u);
        } else {
            long long spins = 0;
            while (*vgen == g) {
                if (++spins > kBarrierSpinLimit || *(volatile int*)&ctl->err) {
                    atomicExch(&ctl->err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int*)&ctl->err == 0;
}

// deterministic all-reduce of up to 4 per-block partials: every block sums the partials
// of all blocks in block order (sum or max per slot)
template <int NV>
__device__ __forceinline__ void grid_allreduce(const double* part, const int* is_max, double* out) {
    __shared__ double red[NV][kKrylovThreads];
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double a = 0.0;
        for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
            const double p = __ldcg(part + (size_t)k * 4 + q);
            a = is_max[q] ? fmax(a, p) : a + p;
        }
        red[q][threadIdx.x] = a;
    }
    __syncthreads();
    for (int w = kKrylovThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
#pragma unroll
            for (int q = 0; q < NV; q++)
                red[q][threadIdx.x] = is_max[q] ? fmax(red[q][threadIdx.x], red[q][threadIdx.x + w])
                                                : red[q][threadIdx.x] + red[q][threadIdx.x + w];
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < NV; q++) out[q] = red[q][0];
    __syncthreads();
}

// block partials: thread values reduced in a fixed tree, written by thread 0
template <int NV>
__device__ __forceinline__ void block_partial(double* vals, const int* is_max, double* part) {
    __shared__ double red[NV][kKrylovThreads];
#pragma unroll
    for (int q = 0; q < NV; q++) red[q][threadIdx.x] = vals[q];
    __syncthreads();
    for (int w = kKrylovThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
#pragma unroll
            for (int q = 0; q < NV; q++)
                red[q][threadIdx.x] = is_max[q] ? fmax(red[q][threadIdx.x], red[q][threadIdx.x + w])
                                                : red[q][threadIdx.x] + red[q][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) part[(size_t)blockIdx.x * 4 + q] = red[q][0];
    }
    __syncthreads();
}

template <typename T>
__device__ __forceinline__ T ldv(const T* p) { return __ldcg(p); }

struct KrylovArgs {
    int V;
    const int *rowptr, *col;
    const double* S;          // scale vector [3V]
    const double* bs;         // scaled rhs S R [3V]
    double rtol, atol;
    int maxit;
    double *h, *u, *v;        // state, incremented on exit
    double* sol;              // -x on exit (x itself when apply_inc == 0)
    int apply_inc;            // 1: Newton increment of the state; 0: plain solve
    double* part;             // [2][grid][4] partials (ping-pong: a slot is rewritten only two reductions later)
    KrylovCtl* ctl;
};

// y = Dinv_i * sum_j A'_ij x_j for node row i, with x_j = xa_j - alpha * xb_j when xb != null.
// Eight lanes share a row: lane l takes the row's values l, l+8, ... (the row's blocks are
// contiguous, so every load instruction of the 8 lanes reads 64 consecutive bytes), and the
// three row sums are combined with xor shuffles in a fixed order.  Products and sums are
// formed in the matrix type MT (FP32 accumulation on the mixed path).  The result is valid
// on lane 0 of the group; `active` false contributes zeros so the whole warp can shuffle.
constexpr int kRowLanes = 8;
template <typename MT, typename VT>
__device__ __forceinline__ void row_apply8(int i, bool active, int lane8, const int* rowptr, const int* col,
                                           const MT* A, const MT* Dinv, const VT* xa, const VT* xb, VT alpha,
                                           VT y[3]) {
    MT a0 = 0, a1 = 0, a2 = 0;
    if (active) {
        const int v1 = __ldg(rowptr + i + 1) * 9;
        for (int v = __ldg(rowptr + i) * 9 + lane8; v < v1; v += kRowLanes) {
            const int kb = v / 9, q = v - 9 * kb, r = q / 3, c = q - 3 * r;
            const int j = __ldg(col + kb);
            VT x = ldv(xa + 3 * j + c);
            if (xb) x -= alpha * ldv(xb + 3 * j + c);
            const MT prod = __ldg(A + v) * (MT)x;
            a0 += (r == 0) ? prod : (MT)0;
            a1 += (r == 1) ? prod : (MT)0;
            a2 += (r == 2) ? prod : (MT)0;
        }
    }
#pragma unroll
    for (int o = kRowLanes / 2; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o, kRowLanes);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o, kRowLanes);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o, kRowLanes);
    }
    if (active && lane8 == 0) {
        const MT* d = Dinv + (size_t)i * 9;
        y[0] = (VT)(__ldg(d + 0) * a0 + __ldg(d + 1) * a1 + __ldg(d + 2) * a2);
        y[1] = (VT)(__ldg(d + 3) * a0 + __ldg(d + 4) * a1 + __ldg(d + 5) * a2);
        y[2] = (VT)(__ldg(d + 6) * a0 + __ldg(d + 7) * a1 + __ldg(d + 8) * a2);
    } else {
        y[0] = y[1] = y[2] = (VT)0;
    }
}

// MT: matrix / preconditioner storage and SpMV accumulation type; VT: Krylov vector type
// (FP64 on both paths: FP32 vectors let the recursively updated residual drift away from
// the true one and the iteration stagnates).
template <typename MT, typename VT>
__global__ void __launch_bounds__(kKrylovThreads) k_bicgstab(KrylovArgs K, const MT* __restrict__ A,
                                                            const MT* __restrict__ Dinv, VT* __restrict__ b,
                                                            VT* __restrict__ uu, VT* __restrict__ r,
                                                            VT* __restrict__ q, VT* __restrict__ p, VT* __restrict__ Ap,
                                                            VT* __restrict__ As, VT* __restrict__ ubest) {
    const int V = K.V;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    // SpMV phases: groups of kRowLanes lanes per row; a warp covers 32 / kRowLanes rows
    const int lane8 = threadIdx.x % kRowLanes;
    const int warp_g = t0 / 32;
    const int grp_off = (threadIdx.x % 32) / kRowLanes;
    const int g0 = warp_g * (32 / kRowLanes);
    const int gstride = (stride / 32) * (32 / kRowLanes);
    const int SUM = 0, MAX = 1;
    KrylovCtl* ctl = K.ctl;
    int nred = 0;   // reductions so far; selects the partial buffer
    auto pbuf = [&]() { return K.part + (size_t)(nred & 1) * gridDim.x * 4; };

    // b <- M^-1 b'
    for (int i = t0; i < V; i += stride) {
        const MT* d = Dinv + (size_t)i * 9;
        const double b0 = K.bs[3 * i], b1 = K.bs[3 * i + 1], b2 = K.bs[3 * i + 2];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const VT y = (VT)((double)d[3 * c] * b0 + (double)d[3 * c + 1] * b1 + (double)d[3 * c + 2] * b2);
            b[3 * i + c] = y;
            uu[3 * i + c] = y;
        }
    }
    if (!grid_sync(ctl)) return;
    // r = b - M^-1 A u, q = r, p = r; norms and rho
    {
        double vals[4] = {0, 0, 0, 0};
        const int ism[4] = {MAX, MAX, SUM, SUM};
        for (int base = g0; base < V; base += gstride) {
            const int i = base + grp_off;
            const bool act = i < V;
            VT y[3];
            row_apply8<MT, VT>(i, act, lane8, K.rowptr, K.col, A, Dinv, uu, (const VT*)nullptr, (VT)0, y);
            if (act && lane8 == 0) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const VT bb = ldv(b + 3 * i + c);
                    const VT rr = bb - y[c];
                    r[3 * i + c] = rr;
                    q[3 * i + c] = rr;
                    p[3 * i + c] = rr;
                    Ap[3 * i + c] = 0;
                    vals[0] = fmax(vals[0], fabs((double)rr));
                    vals[1] = fmax(vals[1], fabs((double)bb));
                    vals[2] += (double)rr * (double)rr;
                }
            }
        }
        block_partial<4>(vals, ism, pbuf());
        if (!grid_sync(ctl)) return;
        double red[4];
        grid_allreduce<4>(pbuf(), ism, red);
        nred++;
        double rnorm = red[0];
        const double bnorm = red[1];
        double rho = red[2], rhop = 1.0, alpha = 1.0, omega = 1.0;
        int it = 0;
        const double tol = K.atol + bnorm * K.rtol;
        // best iterate so far: past its attainable accuracy BiCGSTAB's residual drifts back up,
        // so on stagnation (no new best for kStall iterations) or at max_lin_it the best one is used
        double best = rnorm;
        int best_it = 0;
        for (int i = t0; i < V; i += stride)
#pragma unroll
            for (int c = 0; c < 3; c++) ubest[3 * i + c] = uu[3 * i + c];
        while (rnorm > tol && it < K.maxit && it - best_it < kStall) {
            it++;
            // (d)-(e): Ap = M^-1 A p, gamma = q . Ap
            {
                double g[4] = {0, 0, 0, 0};
                const int gm[4] = {SUM, SUM, SUM, SUM};
                for (int base = g0; base < V; base += gstride) {
                    const int i = base + grp_off;
                    const bool act = i < V;
                    VT y[3];
                    row_apply8<MT, VT>(i, act, lane8, K.rowptr, K.col, A, Dinv, p, (const VT*)nullptr, (VT)0, y);
                    if (act && lane8 == 0) {
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            Ap[3 * i + c] = y[c];
                            g[0] += (double)ldv(q + 3 * i + c) * (double)y[c];
                        }
                    }
                }
                block_partial<1>(g, gm, pbuf());
                if (!grid_sync(ctl)) return;
                grid_allreduce<1>(pbuf(), gm, g);
                nred++;
                alpha = rho / g[0];
            }
            // (f)-(g): As = M^-1 A (r - alpha Ap); omega, next rho
            {
                double w[4] = {0, 0, 0, 0};
                const int wm[4] = {SUM, SUM, SUM, SUM};
                const VT al = (VT)alpha;
                for (int base = g0; base < V; base += gstride) {
                    const int i = base + grp_off;
                    const bool act = i < V;
                    VT y[3];
                    row_apply8<MT, VT>(i, act, lane8, K.rowptr, K.col, A, Dinv, r, Ap, al, y);
                    if (act && lane8 == 0) {
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            const VT s = ldv(r + 3 * i + c) - al * ldv(Ap + 3 * i + c);
                            As[3 * i + c] = y[c];
                            w[0] += (double)y[c] * (double)s;
                            w[1] += (double)y[c] * (double)y[c];
                            w[2] += (double)y[c] * (double)ldv(q + 3 * i + c);
                        }
                    }
                }
                block_partial<3>(w, wm, pbuf());
                if (!grid_sync(ctl)) return;
                grid_allreduce<3>(pbuf(), wm, w);
                nred++;
                omega = w[0] / w[1];
                rhop = rho;
                rho = -1.0 * omega * w[2];
            }
            // (h)-(i) and the next search direction (c): u += alpha p + omega s; r = s - omega As;
            // p = beta (p - omega Ap) + r with beta = (rho alpha) / (rhop omega)
            {
                double mx[4] = {0, 0, 0, 0};
                const int mm[4] = {MAX, MAX, MAX, MAX};
                const double beta = (rho * alpha) / (rhop * omega);
                const VT al = (VT)alpha, om = (VT)omega, be = (VT)beta;
                for (int i = t0; i < V; i += stride) {
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const int k = 3 * i + c;
                        const VT s = ldv(r + k) - al * ldv(Ap + k);
                        VT uk = ldv(uu + k);
                        uk += al * ldv(p + k);
                        uk += om * s;
                        uu[k] = uk;
                        const VT rk = s - om * ldv(As + k);
                        r[k] = rk;
                        p[k] = (ldv(p + k) - om * ldv(Ap + k)) * be + rk;
                        mx[0] = fmax(mx[0], fabs((double)rk));
                    }
                }
                block_partial<1>(mx, mm, pbuf());
                if (!grid_sync(ctl)) return;
                grid_allreduce<1>(pbuf(), mm, mx);
                nred++;
                rnorm = mx[0];
                if (rnorm < best) {   // identical decision in every block; own rows only
                    best = rnorm;
                    best_it = it;
                    for (int i = t0; i < V; i += stride)
#pragma unroll
                        for (int c = 0; c < 3; c++) ubest[3 * i + c] = uu[3 * i + c];
                }
            }
        }
        const bool conv = rnorm <= tol;
        // x = S u; state += x; sol = -x
        const VT* ux = conv ? uu : ubest;
        for (int i = t0; i < V; i += stride) {
            const double x0 = (double)ldv(ux + 3 * i) * K.S[3 * i];
            const double x1 = (double)ldv(ux + 3 * i + 1) * K.S[3 * i + 1];
            const double x2 = (double)ldv(ux + 3 * i + 2) * K.S[3 * i + 2];
            if (K.apply_inc) {
                K.u[i] += x0;
                K.v[i] += x1;
                K.h[i] += x2;
                K.sol[3 * i] = -x0;
                K.sol[3 * i + 1] = -x1;
                K.sol[3 * i + 2] = -x2;
            } else {
                K.sol[3 * i] = x0;
                K.sol[3 * i + 1] = x1;
                K.sol[3 * i + 2] = x2;
            }
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ctl->iterations = it;
            ctl->converged = conv ? 1 : 0;
            ctl->rnorm = conv ? rnorm : best;
            ctl->bnorm = bnorm;
        }
    }
}

}  // namespace sw2
