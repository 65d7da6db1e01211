// sw2_band.cuh -- the exact banded LU solve of one Newton iteration's linear system.
//
// The reference's default linear solver factors the whole Jacobi-scaled system exactly
// (OP BLK 1: one node block, profile LU of solv_blk_set_profile, src/solver/solv_blk_profile.c:5-79,
// applied by solv_blk_solve, src/solver/solv_blk_solve.c:5-62) and runs BiCGSTAB on top of it,
// which then stops at its first test: the solution is LU^-1 b to round-off.  Block-Jacobi
// BiCGSTAB stalls on systems whose time step is many wave-crossings of an element (the QA decks
// the reference ships run at CFL numbers of tens), so a context may ask for this path instead
// (SW2GPU_PREC_BAND): the nodes are renumbered in reverse Cuthill-McKee order on the host, the
// scaled system S A S is scattered into a row-major band of half-width bw (dofs), factored in
// place without pivoting (as the reference's profile LU), and the two triangular solves give the
// increment directly.  One CTA walks the n = 3V pivots in order; the threads share the rank-1
// update of each pivot's bw x bw trailing block and each triangular solve's row updates.  The
// work is n bw^2 for the factor and n bw for a solve, so the path is for the small and medium
// systems of the reference's test decks, not for the 1M-triangle meshes (where the band does not
// fit in the limit sw2gpu_create applies).
#pragma once
#include <cuda_runtime.h>

#include "sw2_krylov.cuh"   // KrylovCtl

namespace sw2 {

constexpr int kBandThreads = 1024;

struct BandArgs {
    int V, n, bw, width;        // nodes, 3V dofs, half-width (dofs), row stride 2 bw + 1
    const int* perm;            // [V] new position of node i
    const int *rowptr, *col;    // BCSR pattern (sorted columns, diagonal included)
    const double* val;          // BCSR values [nnzb][9]
    const double* S;            // Jacobi scale [3V]
    const double* bs;           // scaled right-hand side S R [3V]
    double* band;               // [n][width], a(i, j) at i * width + (j - i + bw)
    double* y;                  // [n] permuted right-hand side, then the solution
};

// a(i, j) of the band (callers keep |i - j| <= bw)
__device__ __forceinline__ double& band_at(const BandArgs& B, int i, int j) {
    return B.band[(size_t)i * B.width + (j - i + B.bw)];
}

// S A S of one BCSR block into the band (thread k: block k of row `row[k]`), the band zeroed before
__global__ void k_band_fill(const __grid_constant__ BandArgs B, const int* __restrict__ blk_row, int nnzb) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnzb) return;
    const int i = blk_row[k], j = B.col[k];
    const int pi = 3 * B.perm[i], pj = 3 * B.perm[j];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++)
            band_at(B, pi + r, pj + c) = B.val[(size_t)k * 9 + 3 * r + c] * (B.S[3 * i + r] * B.S[3 * j + c]);
}

// the right-hand side in the band's order
__global__ void k_band_rhs(const __grid_constant__ BandArgs B) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.V) return;
#pragma unroll
    for (int r = 0; r < 3; r++) B.y[3 * B.perm[i] + r] = B.bs[3 * i + r];
}

// In-place LU without pivoting, one CTA: for every pivot k the multipliers l(i, k) = a(i, k) /
// a(k, k) of the rows below it within the band, then the rank-1 update a(i, j) -= l(i, k) a(k, j)
// of the trailing bw x bw block.  A zero pivot gives an infinite or NaN solution, which the Newton
// loop's norms report (the reference's profile LU does not pivot either).
__global__ void __launch_bounds__(kBandThreads) k_band_factor(const __grid_constant__ BandArgs B) {
    const int n = B.n, bw = B.bw;
    for (int k = 0; k < n; k++) {
        const int m = min(bw, n - 1 - k);   // rows (and columns) of the trailing block
        const double piv = band_at(B, k, k);
        for (int t = threadIdx.x; t < m; t += blockDim.x) band_at(B, k + 1 + t, k) /= piv;
        __syncthreads();
        for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
            const int i = k + 1 + t / m, j = k + 1 + t % m;
            band_at(B, i, j) -= band_at(B, i, k) * band_at(B, k, j);
        }
        __syncthreads();
    }
}

// Forward (unit lower) and backward (upper) substitution in place in y, one CTA; every step
// updates the rows the pivot reaches within the band.
__global__ void __launch_bounds__(kBandThreads) k_band_solve(const __grid_constant__ BandArgs B) {
    const int n = B.n, bw = B.bw;
    for (int k = 0; k < n; k++) {
        const double yk = B.y[k];
        const int m = min(bw, n - 1 - k);
        for (int t = threadIdx.x; t < m; t += blockDim.x) B.y[k + 1 + t] -= band_at(B, k + 1 + t, k) * yk;
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; k--) {
        if (threadIdx.x == 0) B.y[k] = B.y[k] / band_at(B, k, k);
        __syncthreads();
        const double xk = B.y[k];
        const int m = min(bw, k);
        for (int t = threadIdx.x; t < m; t += blockDim.x) B.y[k - 1 - t] -= band_at(B, k - 1 - t, k) * xk;
        __syncthreads();
    }
}

// The increment in node order, unscaled (x = S y), as the Krylov kernel's exit applies it: the
// state advances by x and sol = -x (fe_sw2_inc, fe_newton.c:561-585), or sol = x for a plain solve;
// the control record reports one converged iteration.
__global__ void k_band_apply(const __grid_constant__ BandArgs B, double* __restrict__ h, double* __restrict__ u,
                             double* __restrict__ v, double* __restrict__ sol, int apply_inc, KrylovCtl* ctl) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        ctl->iterations = 1;
        ctl->converged = 1;
        ctl->rnorm = 0.0;
        ctl->bnorm = 0.0;
    }
    if (i >= B.V) return;
    const int p = 3 * B.perm[i];
    const double x0 = B.y[p] * B.S[3 * i], x1 = B.y[p + 1] * B.S[3 * i + 1], x2 = B.y[p + 2] * B.S[3 * i + 2];
    if (apply_inc) {
        u[i] += x0;
        v[i] += x1;
        h[i] += x2;
        sol[3 * i] = -x0;
        sol[3 * i + 1] = -x1;
        sol[3 * i + 2] = -x2;
    } else {
        sol[3 * i] = x0;
        sol[3 * i + 1] = x1;
        sol[3 * i + 2] = x2;
    }
}

}  // namespace sw2
