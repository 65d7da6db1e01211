// sw2_dilu.cuh -- the linear solve of one Newton iteration with a block D-ILU preconditioner.
//
// The reference preconditions BiCGSTAB with an exact LU of its node blocks (OP BLK,
// solv_blk_set_profile, src/solver/solv_blk_profile.c:5-79); with one block (the default) that
// is the whole system and BiCGSTAB stops at once.  A 3x3 block Jacobi M (sw2_krylov.cuh) needs
// some 20 iterations per solve on the benchmark basins.  Block D-ILU is the ILU(0) family's
// diagonal form: with A' = S A S = L + D + U (strict block lower part, block diagonal, strict
// block upper part in the order below),
//
//     M = (Dt + L) Dt^-1 (Dt + U),   Dt_n = D_n - sum_{k < n, k ~ n} L_nk Dt_k^-1 U_kn,
//
// i.e. L and U are A's own blocks and only the diagonal blocks are modified (so that M and A'
// agree on the diagonal and on the pattern's lower and upper parts' products through the
// diagonal).  On the benchmark generator's basins it needs as many BiCGSTAB iterations as a
// full block ILU(0) (6 against block Jacobi's 20 to 1e-8, 4 against 9 to 1e-5), and it is
// applied without the factors: with M = M1 M2, M1 = (Dt + L) Dt^-1, M2 = Dt + U, BiCGSTAB runs
// on the split system
//
//     Ah y = bh,   Ah = Dt (Dt + L)^-1 A' (Dt + U)^-1,   bh = Dt (Dt + L)^-1 S R,   x' = (Dt + U)^-1 y,
//
// and Eisenstat's rearrangement A' = (Dt + L) + (Dt + U) + (D - 2 Dt) gives
//
//     Ah v = Dt t + Dt (Dt + L)^-1 g,   t = (Dt + U)^-1 v,   g = v + (D - 2 Dt) t:
//
// one backward sweep over the upper blocks and one forward sweep over the lower blocks, the
// bytes of one SpMV per operator application.  Both Dt products come free: the backward sweep
// forms w = v - U t = Dt t before its inverse, the forward sweep y = g - L s = Dt s before its
// inverse (s = (Dt + L)^-1 g), so Ah v = w + y, and (D - 2 Dt) t = D t - 2 w.
//
// Parallel order.  The nodes are coloured on the host so that no two neighbours share a colour
// and renumbered colour by colour; a node's lower neighbours are then exactly its neighbours of
// lower colours.  A sweep runs colour by colour (backward: last colour first), each colour's
// rows in parallel, with a bounded grid barrier between colours; the backward sweep's first
// colour and the forward sweep's first colour run in one phase.  One persistent cooperative
// kernel runs the whole BiCGSTAB: per iteration two operator applications and an update pass,
// 4C - 1 barriers for C colours (C is 5 on the benchmark basins).  Every CTA is one virtual CTA of the instance (the instance
// always gets the same CTAs, alone or in a batch); warp w of CTA p owns the 32-row tiles
// p + (w + 8 k) * ncta of every colour, one thread per row, so every dot product is the same
// fixed-order sum of per-CTA partials alone, in a batch and on reruns.
//
// The iterate is kept as x' = (Dt + U)^-1 y directly: y advances by alpha p + omega s, and the
// two applications already formed t1 = (Dt + U)^-1 p and t2 = (Dt + U)^-1 s, so x' advances by
// alpha t1 + omega t2 and no closing sweep is needed.  On exit x = S x' in the natural node
// order, state += x and sol = -x (fe_sw2_inc, fe_newton.c:561-585), or sol = x for a plain solve.
#pragma once
#include <cuda_runtime.h>

#include "sw2_krylov.cuh"   // KrylovCtl, grid_sync, block_partial, grid_allreduce, inv3, LaunchMap

namespace sw2 {

constexpr int kDiluThreads = 256;                   // = kKrylovRowThreads: the reduction helpers' CTA
constexpr int kDiluWarps = kDiluThreads / 32;
constexpr int kMaxColours = 16;
constexpr int kDiluVectors = 11;                    // x', r, r0, p, nu, t, t1, g, s, w, t2 (new order, [3V])
constexpr int kDiluChunk = 4;                       // blocks of a row whose gathers are issued together
constexpr int kDiluMinBlocks = 2;                   // co-resident CTAs per SM the registers are cut for
constexpr int kDiluMaxSlots = 16;                   // lower (or upper) blocks of a row, at most

struct DiluArgs {
    int V, N, ncol;                 // nodes; new rows (colours padded to 32-row tiles); colours
    int nlo, nup;                   // lower / upper block slots
    int ncta;                       // CTAs of the instance's solve (fixed per instance)
    int cstart[kMaxColours + 1];    // new rows of colour c: cstart[c] .. cstart[c+1]-1 (whole tiles),
    int cend[kMaxColours + 1];      // the real ones cstart[c] .. cend[c]-1
    // ELL blocks per colour: the k-th lower block of row n of colour c is slot
    // lbase[c] + k L_c + (n - cstart[c]), L_c = cstart[c+1] - cstart[c], for k < lkn[c] (the
    // colour's longest row; upper: ubase, ukn); element e of slot s is at
    // (s / 32) * 288 + 32 e + s % 32, so a warp reads element e of 32 rows' blocks at once.
    // Lower slots come first in blk, upper slots from 9 * nlo on.
    int lbase[kMaxColours + 1], ubase[kMaxColours + 1], lkn[kMaxColours + 1], ukn[kMaxColours + 1];
    const int *lcol, *ucol;         // [nlo], [nup] new column, -1 in padding slots
    const int *lsrc, *usrc;         // natural BCSR block of a slot, -1 in padding slots
    const int* tslot;               // [nlo] for a lower block (n, j): the slot of (j, n) among j's upper blocks
    const int* old;                 // [N] natural node of new row n, -1 for padding rows
    void* blk;                      // [9 (nlo + nup)] S A S, MT, sliced
    double* Dti;                    // [9 N] Dt_n^-1, sliced by tile like the blocks
    double* Dd;                     // [9 N] D_n = S_n A_nn S_n, sliced
    // natural-order inputs: BCSR pattern and values, scale, scaled right-hand side
    const int *blk_row, *bcol, *dpos;
    const double *val, *S, *bs;
    int* singular;                  // set when a Dt block is singular
    double atol;
    int maxit;
    double *h, *u, *v, *sol;
    int apply_inc;
    double* part;                   // [2][ncta][4] partials (ping-pong)
    KrylovCtl* ctl;
    long long spin_limit;           // polls of a grid-barrier wait (0: kBarrierSpinLimit)
    double* vec[kDiluVectors];      // [3 N] each
};

// element e of sliced slot (or row) s
__device__ __forceinline__ size_t dl_idx(int s, int e) { return (size_t)(s >> 5) * 288 + 32 * e + (s & 31); }

// Setup kernels over a batch: instance ids[j] of the device table owns blocks boff[j] .. .
struct DiluMap {
    const DiluArgs* tab;
    LaunchMap mp;
    __device__ __forceinline__ const DiluArgs& get(int& lb, int& nb) const { return tab[map_block(mp, lb, nb)]; }
};
// The solve: one instance by value, or a batch (device table, map, per-instance tolerance).
struct DiluOne {
    DiluArgs K;
    double rtol;
    const double* rtol_dev;         // graph replays read the tolerance here
    __device__ __forceinline__ const DiluArgs& get(int& pl, int& np, double& rt) const {
        pl = blockIdx.x;
        np = gridDim.x;
        rt = rtol_dev ? __ldcg(rtol_dev) : rtol;
        return K;
    }
};
struct DiluTab {
    const DiluArgs* tab;
    LaunchMap mp;
    double rtol[kMaxBatch];
    const double* rtol_dev;         // when set, instance k's tolerance is read at rtol_dev[k] (graph replays)
    // the instance's descriptor is copied to shared memory once (called by the whole CTA)
    __device__ __forceinline__ const DiluArgs& get(int& pl, int& np, double& rt) const {
        __shared__ DiluArgs sk;
        int nb;
        const int b = blockIdx.x;
        int lo = 0, hi = mp.n;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (mp.boff[mid] <= b) lo = mid;
            else hi = mid;
        }
        pl = b - mp.boff[lo];
        nb = mp.boff[lo + 1] - mp.boff[lo];
        np = nb;
        rt = rtol_dev ? __ldcg(rtol_dev + mp.ids[lo]) : rtol[lo];
        if (threadIdx.x == 0) sk = tab[mp.ids[lo]];
        __syncthreads();
        return sk;
    }
};

// S A S of every off-diagonal block into its sliced slot, and the scaled diagonal blocks (after
// k_rowscale: S and the tiny-diagonal fix).  One thread per lower slot, upper slot, then row.
template <typename MT>
__global__ void k_dilu_scatter(const __grid_constant__ DiluMap m) {
    int lb, nb;
    const DiluArgs& K = m.get(lb, nb);
    int t = lb * blockDim.x + threadIdx.x;
    if (t < K.nlo + K.nup) {
        const bool lower = t < K.nlo;
        const int s = lower ? t : t - K.nlo;
        const int k = lower ? K.lsrc[s] : K.usrc[s];
        if (k < 0) return;
        const int i = K.blk_row[k], j = K.bcol[k];
        MT* o = (MT*)K.blk + (lower ? 0 : (size_t)9 * K.nlo);
        const double* a = K.val + (size_t)k * 9;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) o[dl_idx(s, 3 * r + c)] = (MT)(a[3 * r + c] * (K.S[3 * i + r] * K.S[3 * j + c]));
        return;
    }
    t -= K.nlo + K.nup;
    if (t >= K.N) return;
    const int i = K.old[t];
    if (i < 0) return;
    const double* a = K.val + (size_t)K.dpos[i] * 9;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) K.Dd[dl_idx(t, 3 * r + c)] = a[3 * r + c] * (K.S[3 * i + r] * K.S[3 * i + c]);
}

// c = a b (3x3 row-major), FP64
__device__ __forceinline__ void dl_mm3(const double* a, const double* b, double* c) {
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int q = 0; q < 3; q++) c[3 * r + q] = fmadd(a[3 * r + 2], b[6 + q], fmadd(a[3 * r + 1], b[3 + q], a[3 * r] * b[q]));
}

// The modified diagonal blocks of colour c: Dt_n = D_n - sum over n's lower blocks (in column
// order) of L_nj Dt_j^-1 U_jn, and their inverses.  Colours run in separate launches, lowest
// first, so the Dt_j^-1 of lower colours are complete.
template <typename MT>
__global__ void k_dilu_diag(const __grid_constant__ DiluMap m, int c) {
    int lb, nb;
    const DiluArgs& K = m.get(lb, nb);
    if (c >= K.ncol) return;
    const int n = K.cstart[c] + lb * blockDim.x + threadIdx.x;
    if (n >= K.cend[c]) return;
    const MT* BL = (const MT*)K.blk;
    const MT* BU = BL + (size_t)9 * K.nlo;
    double d[9];
#pragma unroll
    for (int e = 0; e < 9; e++) d[e] = K.Dd[dl_idx(n, e)];
    const int base = K.lbase[c] + n - K.cstart[c], stride = K.cstart[c + 1] - K.cstart[c];
    for (int k = 0; k < K.lkn[c]; k++) {
        const int s = base + k * stride;
        const int j = K.lcol[s];
        if (j < 0) break;   // a row's blocks fill its first slots
        const int su = K.tslot[s];
        double l[9], di[9], uu[9], ld[9], p[9];
#pragma unroll
        for (int e = 0; e < 9; e++) {
            l[e] = (double)BL[dl_idx(s, e)];
            di[e] = K.Dti[dl_idx(j, e)];
            uu[e] = (double)BU[dl_idx(su, e)];
        }
        dl_mm3(l, di, ld);
        dl_mm3(ld, uu, p);
#pragma unroll
        for (int e = 0; e < 9; e++) d[e] -= p[e];
    }
    double inv[9];
    if (!inv3(d, inv)) atomicExch(K.singular, 1);
#pragma unroll
    for (int e = 0; e < 9; e++) K.Dti[dl_idx(n, e)] = inv[e];
}

// w -= B x for a 3x3 block stored as MT, FP64 arithmetic in a fixed order
template <typename MT>
__device__ __forceinline__ void dl_sub_bx(const MT* __restrict__ b, const double x[3], double w[3]) {
#pragma unroll
    for (int r = 0; r < 3; r++)
        w[r] -= fmadd((double)b[3 * r + 2], x[2], fmadd((double)b[3 * r + 1], x[1], (double)b[3 * r] * x[0]));
}
// y = A x for an FP64 3x3 block
__device__ __forceinline__ void dl_mv3(const double* __restrict__ a, const double x[3], double y[3]) {
#pragma unroll
    for (int r = 0; r < 3; r++) y[r] = fmadd(a[3 * r + 2], x[2], fmadd(a[3 * r + 1], x[1], a[3 * r] * x[0]));
}
__device__ __forceinline__ void dl_ld3(const double* p, int n, double x[3]) {
    x[0] = __ldcg(p + 3 * n);
    x[1] = __ldcg(p + 3 * n + 1);
    x[2] = __ldcg(p + 3 * n + 2);
}
__device__ __forceinline__ void dl_st3(double* p, int n, const double x[3]) {
    p[3 * n] = x[0];
    p[3 * n + 1] = x[1];
    p[3 * n + 2] = x[2];
}
__device__ __forceinline__ double dl_dot3(const double a[3], const double b[3]) {
    return fmadd(a[2], b[2], fmadd(a[1], b[1], a[0] * b[0]));
}

// w -= sum of B_k x_col(k) over a row's blocks k, slots base + k stride for k < kn (the
// colour's longest row; padding slots have column -1), in k order.  All column indices are
// loaded at once, then the vector gathers of kDiluChunk blocks are issued together: about three
// dependent memory round trips per row.  A warp reads each block element of 32 rows at once.
template <typename MT>
__device__ __forceinline__ void dl_row_sub(const MT* __restrict__ B, const int* __restrict__ cix, const double* xv,
                                           int base, int stride, int kn, double w[3]) {
    int j[kDiluMaxSlots];
#pragma unroll
    for (int k = 0; k < kDiluMaxSlots; k++) j[k] = k < kn ? __ldg(cix + base + k * stride) : -1;
#pragma unroll
    for (int k0 = 0; k0 < kDiluMaxSlots; k0 += kDiluChunk) {
        if (k0 >= kn) break;
        double x[kDiluChunk][3];
#pragma unroll
        for (int u = 0; u < kDiluChunk; u++) {
            if (j[k0 + u] >= 0) {
                dl_ld3(xv, j[k0 + u], x[u]);
            } else {
                x[u][0] = 0.0;
                x[u][1] = 0.0;
                x[u][2] = 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < kDiluChunk; u++)
            if (j[k0 + u] >= 0) {
                const MT* b = B + dl_idx(base + (k0 + u) * stride, 0);
#pragma unroll
                for (int r = 0; r < 3; r++)
                    w[r] -= fmadd((double)b[32 * (3 * r + 2)], x[u][2],
                                  fmadd((double)b[32 * (3 * r + 1)], x[u][1], (double)b[32 * (3 * r)] * x[u][0]));
            }
    }
}

template <typename MT, class SRC>
__global__ void __launch_bounds__(kDiluThreads, kDiluMinBlocks) k_dilu_bicgstab(const __grid_constant__ SRC srcs) {
    __shared__ double red[4 * kKrylovWarps];
    int pl, np;
    double rtol;
    const DiluArgs& K = srcs.get(pl, np, rtol);
    const int C = K.ncol;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const MT* __restrict__ BL = (const MT*)K.blk;
    const MT* __restrict__ BU = BL + (size_t)9 * K.nlo;
    const int* __restrict__ lcol = K.lcol;
    const int* __restrict__ ucol = K.ucol;
    const double* __restrict__ Dti = K.Dti;
    const double* __restrict__ Dd = K.Dd;
    double* xv = K.vec[0];   // x' = (Dt + U)^-1 y, kept up to date
    double* rv = K.vec[1];
    double* r0 = K.vec[2];
    double* pv = K.vec[3];
    double* nu = K.vec[4];
    double* tv = K.vec[5];
    double* t1 = K.vec[6];   // backward-sweep vectors of the first and second application:
    double* t2 = K.vec[10];  // t1 = (Dt + U)^-1 p, t2 = (Dt + U)^-1 s
    double* gv = K.vec[7];
    double* ss = K.vec[8];
    double* wv = K.vec[9];
    KrylovCtl* ctl = K.ctl;
    unsigned epoch = 0;
    int nred = 0;
    const long long lim = K.spin_limit > 0 ? K.spin_limit : kBarrierSpinLimit;
    const int SUM = 0, MAX = 1;
    auto gsync = [&]() { return grid_sync(ctl, np, epoch, lim); };
    // the rows of colour c this thread owns, in a fixed order (a warp takes whole tiles)
    auto rows = [&](int c, auto&& f) {
        const int c0 = K.cstart[c], c1 = K.cend[c];
        const int nt = (K.cstart[c + 1] - c0) / 32;
        for (int m = pl + warp * np; m < nt; m += kDiluWarps * np) {
            const int n = c0 + m * 32 + lane;
            if (n < c1) f(n);
        }
    };
    auto lower = [&](const double* xv, int c, int n, double* w) {
        dl_row_sub(BL, lcol, xv, K.lbase[c] + n - K.cstart[c], K.cstart[c + 1] - K.cstart[c], K.lkn[c], w);
    };
    auto upper = [&](const double* xv, int c, int n, double* w) {
        dl_row_sub(BU, ucol, xv, K.ubase[c] + n - K.cstart[c], K.cstart[c + 1] - K.cstart[c], K.ukn[c], w);
    };
    // per-CTA partials of NV values, then the grid-wide fixed-order combination
    auto reduce = [&](auto nvc, double* vals, const int* kinds, double* out) -> bool {
        constexpr int NV = decltype(nvc)::value;
        double* part = K.part + (size_t)(nred & 1) * np * 4;
        nred++;
        block_partial<NV>(vals, kinds, part, pl, red);
        if (!gsync()) return false;
        grid_allreduce<NV>(part, np, kinds, out, red);
        return true;
    };
    auto ld9 = [](const double* __restrict__ a, int n, double* o) {
#pragma unroll
        for (int e = 0; e < 9; e++) o[e] = __ldg(a + dl_idx(n, e));
    };
    // Eisenstat application out = Ah v = w + y, colour phase by colour phase; vin(n, v) gives
    // row n's input, vout(n, o) takes its output; tt receives t = (Dt + U)^-1 v.  The backward
    // sweep keeps t (its recursion), w and g; the forward sweep keeps s (its recursion).  Each
    // row's diagonal blocks are loaded before its gathers, so their latency overlaps.  The last
    // phase ends without a barrier (the caller's reduction closes it).
    auto apply = [&](double* tt, auto&& vin, auto&& vout) -> bool {
        for (int c = C - 1; c >= 0; c--) {
            rows(c, [&](int n) {
                double di[9], dd[9], vn[3], w[3], t[3], g[3];
                ld9(Dti, n, di);
                ld9(Dd, n, dd);
                vin(n, vn);
                w[0] = vn[0]; w[1] = vn[1]; w[2] = vn[2];
                upper(tt, c, n, w);
                dl_mv3(di, w, t);
                dl_st3(tt, n, t);
                dl_mv3(dd, t, g);
#pragma unroll
                for (int r = 0; r < 3; r++) g[r] = vn[r] + g[r] - 2.0 * w[r];
                if (c == 0) {   // no lower neighbours: the forward sweep's first colour, y = g
                    double s[3], o[3];
                    dl_mv3(di, g, s);
                    dl_st3(ss, n, s);
#pragma unroll
                    for (int r = 0; r < 3; r++) o[r] = w[r] + g[r];
                    vout(n, o);
                } else {
                    dl_st3(gv, n, g);
                    dl_st3(wv, n, w);
                }
            });
            if (!gsync()) return false;
        }
        for (int c = 1; c < C; c++) {
            rows(c, [&](int n) {
                double di[9], y[3], s[3], w[3], o[3];
                ld9(Dti, n, di);
                dl_ld3(gv, n, y);
                dl_ld3(wv, n, w);
                lower(ss, c, n, y);
                dl_mv3(di, y, s);
                dl_st3(ss, n, s);
#pragma unroll
                for (int r = 0; r < 3; r++) o[r] = w[r] + y[r];
                vout(n, o);
            });
            if (c + 1 < C && !gsync()) return false;
        }
        return true;
    };

    // ---- bh = Dt (Dt + L)^-1 S R in the coloured order: a forward sweep (recursion on s in ss),
    // bh its values before the inverse; r = r0 = bh, x' = 0
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = 0; c < C; c++) {
        rows(c, [&](int n) {
            const int i = K.old[n];
            double di[9];
            ld9(Dti, n, di);
            double y[3] = {K.bs[3 * i], K.bs[3 * i + 1], K.bs[3 * i + 2]}, s[3];
            lower(ss, c, n, y);
            dl_mv3(di, y, s);
            dl_st3(ss, n, s);
            dl_st3(rv, n, y);
            dl_st3(r0, n, y);
            const double z[3] = {0.0, 0.0, 0.0};
            dl_st3(xv, n, z);
            acc[0] += dl_dot3(y, y);
            acc[1] = fmax(acc[1], fmax(fabs(y[0]), fmax(fabs(y[1]), fabs(y[2]))));
        });
        if (c + 1 < C && !gsync()) return;
    }
    double out[4];
    {
        const int kinds[2] = {SUM, MAX};
        if (!reduce(IntC<2>{}, acc, kinds, out)) return;
    }
    double rho = out[0];
    const double bnorm = out[1];
    const double tol = K.atol + rtol * bnorm;
    double rnorm = bnorm;
    bool conv = !(rnorm > tol);   // also stops on a NaN right-hand side
    int it = 0;
    double alpha = 0.0, omega = 0.0, beta = 0.0;
    while (!conv && it < K.maxit) {
        it++;
        // nu = Ah p, p = r + beta (p - omega nu) (p = r on the first iteration); t1 = (Dt + U)^-1 p
        const bool first = it == 1;
        double a1[1] = {0.0};
        if (!apply(
                t1,
                [&](int n, double* p) {
                    double r[3];
                    dl_ld3(rv, n, r);
                    if (first) {
                        p[0] = r[0]; p[1] = r[1]; p[2] = r[2];
                    } else {
                        double po[3], no[3];
                        dl_ld3(pv, n, po);
                        dl_ld3(nu, n, no);
#pragma unroll
                        for (int q = 0; q < 3; q++) p[q] = r[q] + beta * (po[q] - omega * no[q]);
                    }
                    dl_st3(pv, n, p);
                },
                [&](int n, const double* o) {
                    double z[3];
                    dl_st3(nu, n, o);
                    dl_ld3(r0, n, z);
                    a1[0] += dl_dot3(z, o);
                }))
            return;
        {
            const int kinds[1] = {SUM};
            if (!reduce(IntC<1>{}, a1, kinds, out)) return;
        }
        const double r0nu = out[0];
        if (!(r0nu != 0.0) || !isfinite(r0nu)) break;   // breakdown: keep the iterate so far
        alpha = rho / r0nu;
        // t = Ah s, s = r - alpha nu; t2 = (Dt + U)^-1 s
        double a2[2] = {0.0, 0.0};
        if (!apply(
                t2,
                [&](int n, double* s) {
                    double r[3], no[3];
                    dl_ld3(rv, n, r);
                    dl_ld3(nu, n, no);
#pragma unroll
                    for (int q = 0; q < 3; q++) s[q] = r[q] - alpha * no[q];
                },
                [&](int n, const double* o) {
                    double r[3], no[3], s[3];
                    dl_st3(tv, n, o);
                    dl_ld3(rv, n, r);
                    dl_ld3(nu, n, no);
#pragma unroll
                    for (int q = 0; q < 3; q++) s[q] = r[q] - alpha * no[q];
                    a2[0] += dl_dot3(o, s);
                    a2[1] += dl_dot3(o, o);
                }))
            return;
        {
            const int kinds[2] = {SUM, SUM};
            if (!reduce(IntC<2>{}, a2, kinds, out)) return;
        }
        omega = out[1] > 0.0 ? out[0] / out[1] : 0.0;
        // y += alpha p + omega s, kept as x' += alpha t1 + omega t2; r = s - omega t
        double a3[2] = {0.0, 0.0};
        for (int c = 0; c < C; c++)
            rows(c, [&](int n) {
                double r[3], no[3], t[3], x[3], ta[3], tb[3];
                dl_ld3(rv, n, r);
                dl_ld3(nu, n, no);
                dl_ld3(tv, n, t);
                dl_ld3(xv, n, x);
                dl_ld3(t1, n, ta);
                dl_ld3(t2, n, tb);
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const double s = r[q] - alpha * no[q];
                    x[q] = x[q] + alpha * ta[q] + omega * tb[q];
                    r[q] = s - omega * t[q];
                }
                dl_st3(xv, n, x);
                dl_st3(rv, n, r);
                double z[3];
                dl_ld3(r0, n, z);
                a3[0] = fmax(a3[0], fmax(fabs(r[0]), fmax(fabs(r[1]), fabs(r[2]))));
                a3[1] += dl_dot3(z, r);
            });
        {
            const int kinds[2] = {MAX, SUM};
            if (!reduce(IntC<2>{}, a3, kinds, out)) return;
        }
        rnorm = out[0];
        conv = !(rnorm > tol) && isfinite(rnorm);
        if (conv) break;
        const double rho1 = out[1];
        if (!(omega != 0.0) || !(rho != 0.0) || !isfinite(rho1)) break;
        beta = (rho1 / rho) * (alpha / omega);
        rho = rho1;
    }
    // ---- x = S x' in the natural order (the last update pass's values are this thread's own rows)
    for (int c = 0; c < C; c++)
        rows(c, [&](int n) {
            double x[3];
            dl_ld3(xv, n, x);
            const int i = K.old[n];
            const double x0 = x[0] * K.S[3 * i], x1 = x[1] * K.S[3 * i + 1], x2 = x[2] * K.S[3 * i + 2];
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
        });
    if (pl == 0 && threadIdx.x == 0) {
        ctl->iterations = it;
        ctl->converged = conv ? 1 : 0;
        ctl->rnorm = rnorm;
        ctl->bnorm = bnorm;
    }
}

}  // namespace sw2
