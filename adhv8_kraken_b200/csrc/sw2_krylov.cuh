// sw2_krylov.cuh -- the linear solve of one Newton iteration as ONE persistent kernel.
//
// Restates solv_bcgstab (src/solver/solv_bcgstab.c:39-301) on the Jacobi-scaled
// system A' = S A S, b' = S R (spv_jacobi), left-preconditioned by M^-1, with the
// reference's stopping test ||r||inf <= atol + rtol ||M^-1 b'||inf and its initial
// guess u = M^-1 b'.  M is the 3x3 block-Jacobi inverse (the reference factors
// OP BLK node blocks exactly; any M that converges gives the same Newton result).
//
// One cooperative launch runs the whole iteration for every instance of a batch: each
// instance owns a contiguous range of CTAs with its own bounded barrier.  Its work is cut
// into a fixed number of virtual CTAs (the grid the instance would get alone); a physical
// CTA runs virtual CTAs pl, pl + np, ... in turn.  Every dot product / norm is a per-virtual-
// CTA partial reduced in the same fixed order by every CTA, so all CTAs of an instance take
// identical control decisions, and an instance's results are bitwise the same alone, in any
// batch and on reruns.  s = r - alpha Ap is never stored: the second SpMV forms it on the
// fly from r and Ap.
// A batch launch may stop the instances still iterating at an iteration boundary once enough
// CTAs have finished theirs (KrylovTab::done_ctas), keeping the loop scalars in each
// instance's KrylovCtl; the next launch resumes them with all CTAs shared among them.  The
// partial structure stays that of the instance's virtual grid, so the bits do not change.
// On exit the kernel applies the Newton increment: x = S u, state += x (fe_sw2_inc),
// sol = -x (fe_newton.c:561-585).
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

namespace sw2 {

// 8 row warps (SpMV rows, vector passes, partials) and one copy warp that fills the tile ring
constexpr int kKrylovRowThreads = 256;
constexpr int kKrylovThreads = kKrylovRowThreads + 32;
constexpr long long kBarrierSpinLimit = 1ll << 23;   // polls (a few seconds: each is an L2 round trip), then error
constexpr long long kMbarSpinLimit = 1ll << 20;      // polls (about a second) of one tile mbarrier, then error
// a launch may bound its waits more tightly (KrylovArgs::spin_limit / copy_limit, 0 = these
// defaults): failure-detection tests make a wait run out that way, without a fault
constexpr int kStall = 40;                           // iterations without a new best residual
constexpr int kRowLanes = 8;                         // lanes per node row in the SpMV sweeps
constexpr int kTileRows = kKrylovRowThreads / kRowLanes;   // node rows per CTA tile (32)
constexpr int kMaxStages = 3;                        // deepest shared-memory tile ring of the staged sweeps
constexpr int kVirtualPerSM = 3;                     // virtual CTAs per SM of a large instance (fixed:
                                                     // it sets the reduction order, so no tuning knob may)

// Blocks of one launch over a batch: instance ids[j] owns blocks boff[j] .. boff[j+1]-1.
// Passed by value (kernel parameter space), so lookups are uniform constant-bank reads.
constexpr int kMaxBatch = 256;
struct LaunchMap {
    int n;
    int boff[kMaxBatch + 1];
    int ids[kMaxBatch];
};
// instance id of this block; lb = block index inside the instance, nb = its block count
__device__ __forceinline__ int map_block(const LaunchMap& mp, int& lb, int& nb) {
    const int b = blockIdx.x;
    int lo = 0, hi = mp.n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (mp.boff[mid] <= b) lo = mid;
        else hi = mid;
    }
    lb = b - mp.boff[lo];
    nb = mp.boff[lo + 1] - mp.boff[lo];
    return mp.ids[lo];
}

struct KrylovCtl {
    unsigned count;       // barrier arrivals since the launch (zeroed before it)
    unsigned pad0;
    int err;              // 1 = a barrier or tile-copy wait ran out
    int iterations;
    int converged;        // 1 = stopping test met, 0 = hit max_lin_it
    int pad;
    double rnorm, bnorm;
    // A batch launch may pause an instance at the top of an iteration so that a later launch,
    // with the CTAs of the instances that have finished, resumes it (KrylovTab::done_ctas).  The
    // instance's first CTA sets pause_at (the iteration at whose top it stops) before the
    // iteration's second grid barrier; every CTA reads it at the next loop top.  The loop's
    // scalars are kept here; the vectors stay where they are.
    int pause_at;         // 0: no pause requested
    int paused;           // 1: the launch ended at a pause, the solve resumes in the next one
    int s_it, s_best_it, s_pending, s_upd, s_cur, s_nred;
    double s_rnorm, s_tol, s_rho, s_alpha, s_omega, s_beta, s_best;
};

// Grid barrier with a bounded spin.  Arrivals only ever add to one counter, so the b-th
// barrier of a launch is passed once the counter reaches b * nblocks (`epoch`, per CTA): the
// last arrival releases everyone without a second atomic.  Returns false (and sets ctl->err)
// if any block gave up; the caller then returns, so the kernel always terminates.  The error
// word is read once, by thread 0, and the decision reaches the whole CTA through shared
// memory: another CTA may set the word at any moment, and threads reading it one by one could
// disagree, some returning while the rest of the CTA waits for them at its next barrier.
__device__ __forceinline__ bool grid_sync(KrylovCtl* ctl, unsigned nblocks, unsigned& epoch, long long limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        epoch += nblocks;
        __threadfence();
        atomicAdd(&ctl->count, 1u);
        // tight bounded poll (acquire loads, no sleep: a wake-up later than the last arrival
        // would be paid at every barrier)
        long long spins = 0;
        for (;;) {
            unsigned cur;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(&ctl->count) : "memory");
            if ((int)(cur - epoch) >= 0) break;
            if (++spins > limit || *(volatile int*)&ctl->err) {
                atomicExch(&ctl->err, 1);
                break;
            }
        }
        // no trailing fence: the acquire load orders this thread's later accesses, and the
        // __syncthreads below orders the rest of the CTA's after it
        s_ok = *(volatile int*)&ctl->err == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

constexpr int kKrylovWarps = kKrylovRowThreads / 32;   // warps that hold partials
// named barrier of the Krylov CTA's row warps alone (0 is __syncthreads')
constexpr int kBarRows = 1;
__device__ __forceinline__ void bar_sync_n(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive_n(int id, int count) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// fixed-order warp tree (xor shuffles): every lane ends with the same value
__device__ __forceinline__ double warp_combine(double a, bool is_max) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, a, o);
        a = is_max ? fmax(a, t) : a + t;
    }
    return a;
}

// deterministic all-reduce of up to 4 per-block partials: every block combines the partials
// of all blocks in the same fixed order (sum or max per slot); red = shared [4][kKrylovWarps].
// The row warps read the partials; every thread of the CTA (the copy warp too, which needs
// the loop decisions) ends with the result.  Called by the whole CTA.
template <int NV>
__device__ __forceinline__ void grid_allreduce(const double* part, int nparts, const int* is_max, double* out,
                                               double* red) {
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (threadIdx.x < kKrylovRowThreads) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double a = 0.0;
            for (int k = threadIdx.x; k < nparts; k += kKrylovRowThreads) {
                const double p = __ldcg(part + (size_t)k * 4 + q);
                a = is_max[q] ? fmax(a, p) : a + p;
            }
            a = warp_combine(a, is_max[q]);
            if (lane == 0) red[q * kKrylovWarps + warp] = a;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double a = red[q * kKrylovWarps];
#pragma unroll
        for (int w = 1; w < kKrylovWarps; w++) a = is_max[q] ? fmax(a, red[q * kKrylovWarps + w]) : a + red[q * kKrylovWarps + w];
        out[q] = a;
    }
    __syncthreads();
}

// block partials: the row threads' values combined in a fixed order, written by thread 0 to
// slot `slot`.  Called by the row warps only (the copy warp may be ahead in the tile sequence).
template <int NV>
__device__ __forceinline__ void block_partial(double* vals, const int* is_max, double* part, int slot, double* red) {
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
#pragma unroll
    for (int q = 0; q < NV; q++) {
        const double a = warp_combine(vals[q], is_max[q]);
        if (lane == 0) red[q * kKrylovWarps + warp] = a;
    }
    bar_sync_n(kBarRows, kKrylovRowThreads);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double a = red[q * kKrylovWarps];
#pragma unroll
            for (int w = 1; w < kKrylovWarps; w++)
                a = is_max[q] ? fmax(a, red[q * kKrylovWarps + w]) : a + red[q * kKrylovWarps + w];
            part[(size_t)slot * 4 + q] = a;
        }
    }
    bar_sync_n(kBarRows, kKrylovRowThreads);
}

template <typename T>
__device__ __forceinline__ T ldv(const T* p) { return __ldcg(p); }

// inverse of a 3x3 block (cofactors over the determinant); false (and the identity) when
// the block is singular or not finite
__device__ __forceinline__ bool inv3(const double* a, double* out) {
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (det == 0.0 || !isfinite(det)) {
#pragma unroll
        for (int q = 0; q < 9; q++) out[q] = (q % 4 == 0) ? 1.0 : 0.0;
        return false;
    }
    const double id = 1.0 / det;
    out[0] = c00 * id;
    out[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    out[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    out[3] = c01 * id;
    out[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    out[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    out[6] = c02 * id;
    out[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    out[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return true;
}

// o = d * b for 3x3 blocks (row-major), formed in FP64 and stored as MT
template <typename MT>
__device__ __forceinline__ void fold_block(const double* d, const double* b, MT* o) {
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++)
            o[3 * r + c] = (MT)(d[3 * r] * b[c] + d[3 * r + 1] * b[3 + c] + d[3 * r + 2] * b[6 + c]);
}

struct KrylovArgs {
    int V;
    const int *rowptr, *col;  // off-diagonal block structure of the folded operator M^-1 A'
    const double* S;          // scale vector [3V]
    const double* bs;         // scaled rhs S R [3V]
    double atol;              // absolute Krylov tolerance (the relative one is per launch)
    int maxit;
    double *h, *u, *v;        // state, incremented on exit
    double* sol;              // -x on exit (x itself when apply_inc == 0)
    int apply_inc;            // 1: Newton increment of the state; 0: plain solve
    double* part;             // [2][vgrid][4] partials (ping-pong: a slot is rewritten only two reductions later)
    KrylovCtl* ctl;
    int vgrid;                // virtual CTAs: the partial structure, fixed per instance
    int fuse_update;          // 1: an iteration's update is applied by the next iteration's first
                              // sweep (one grid barrier and one vector pass fewer per iteration,
                              // more vectors live: for launches whose vectors stay in L2); a batch
                              // launch decides for all its instances (KrylovTab::fuse)
    long long spin_limit;     // polls of a grid-barrier wait before it gives up (0: kBarrierSpinLimit)
    long long copy_limit;     // polls of a tile-copy wait before it gives up (0: kMbarSpinLimit)
};

// one instance of a Krylov launch
struct KrylovInst {
    KrylovArgs K;
    const void* A;            // folded off-diagonal blocks, MT
    const double* Dinv;       // FP64 block-Jacobi inverses (b = M^-1 b' only)
    double* vec[12];          // b, u, r, q, p, Ap, As, best u, and the second copies of u, r, p, Ap
};
constexpr int kKrylovVectors = 12;
// The fused update keeps all 12 vectors live within one sweep and gathers four of them; it pays
// while the vectors of every instance of a launch stay in L2 together (126 MB on B200), i.e.
// up to ~170k nodes in total.
constexpr long long kFuseUpdateMaxBytes = 48ll << 20;
inline int krylov_fuse_update(long long nodes) { return kKrylovVectors * 24ll * nodes <= kFuseUpdateMaxBytes ? 1 : 0; }

// Stage layout of the staged sweeps: byte offsets inside one stage of the tile's column
// indices, row pointers and epilogue vectors (the blocks start at 0), and the stage stride.
struct StageLayout {
    unsigned c_off, r_off, v_off, stage_bytes;
};

// Where a Krylov launch finds its instances.  KrylovOne: one instance, its record and
// tolerance kernel parameters; KrylovTab: a batch, records in a device table, the map and
// each mapped instance's relative tolerance in the parameters.
struct KrylovOne {
    KrylovInst Q;
    double rtol;
    const double* rtol_dev;   // when set, the tolerance is read here (a launch replayed from a
                              // CUDA graph takes each Newton iteration's tolerance from memory)
    StageLayout lay;
    __device__ __forceinline__ const KrylovInst& get(int& pl, int& np, double& rt) const {
        pl = blockIdx.x;
        np = gridDim.x;
        rt = rtol_dev ? __ldcg(rtol_dev) : rtol;
        return Q;
    }
    __device__ __forceinline__ bool fuse_update(const KrylovInst& KI) const { return KI.K.fuse_update != 0; }
    __device__ __forceinline__ unsigned* done_counter() const { return nullptr; }
    __device__ __forceinline__ unsigned pause_threshold() const { return 0u; }
    __device__ __forceinline__ bool resuming() const { return false; }
};
struct KrylovTab {
    const KrylovInst* tab;
    LaunchMap mp;
    double rtol[kMaxBatch];
    StageLayout lay;
    int fuse;                 // fused update for every instance of the launch (their vectors together)
    const double* rtol_dev;   // when set, instance k's tolerance is read at rtol_dev[k] (graph replays)
    // Rebalancing (host-driven launches only): every CTA whose instance finished adds one to
    // *done_ctas (zeroed before the launch); once it reaches pause_after, the instances still
    // running pause at their next iteration top.  resume = 1: every instance of the launch
    // continues a paused solve from the scalars in its KrylovCtl.  An instance's partial
    // structure depends on its virtual grid alone, so its bits do not depend on where it paused
    // nor on how many CTAs each launch gave it.
    unsigned* done_ctas;      // nullptr: no pausing
    unsigned pause_after;
    int resume;
    __device__ __forceinline__ unsigned* done_counter() const { return done_ctas; }
    __device__ __forceinline__ unsigned pause_threshold() const { return pause_after; }
    __device__ __forceinline__ bool resuming() const { return resume != 0; }
    __device__ __forceinline__ const KrylovInst& get(int& pl, int& np, double& rt) const {
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
        return tab[mp.ids[lo]];
    }
    __device__ __forceinline__ bool fuse_update(const KrylovInst&) const { return fuse != 0; }
};

// the control words of the instances a launch resumes: a fresh barrier, no pause pending (the
// saved scalars stay)
static __global__ void k_krylov_rearm(KrylovCtl* ctl, const __grid_constant__ LaunchMap mp) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= mp.n) return;
    KrylovCtl* c = ctl + mp.ids[j];
    c->count = 0;
    c->pause_at = 0;
    c->paused = 0;
}

// bytes of one epilogue vector's slice for a full tile (3 components per row)
template <typename VT>
__host__ __device__ constexpr unsigned tile_vec_bytes() { return kTileRows * 3 * sizeof(VT); }
constexpr int kMaxEpilogue = 6;   // epilogue vectors a sweep stages per tile

// ---- tile staging: one bulk copy per tile, completion on an mbarrier -------------------------
// Tile m = node rows [m kTileRows, (m+1) kTileRows); its blocks and column indices are contiguous.
// The copied ranges are rounded out to 16 bytes (the bulk-copy rule); the arrays are allocated
// with 16 spare bytes and start on 256-byte boundaries, so the rounded ranges stay inside them.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// the same with an L2 eviction policy (evict_first for data streamed once per sweep)
__device__ __forceinline__ void bulk_load_hint(void* dst, const void* src, unsigned bytes, unsigned long long* bar,
                                               unsigned long long policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// orders this thread's view of global data written through the generic proxy (other CTAs'
// stores before the last grid barrier) before its following bulk copies (async proxy)
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
// bounded wait (at most `limit` polls) for the completion of the phase with the given parity.
// A try_wait poll may itself suspend the thread for a hardware time window, long enough for a
// tile copy to land; a limit below kShortWait polls with the non-blocking test_wait instead, so
// that a short limit really bounds the wait (failure-detection tests).
constexpr long long kShortWait = 64;
constexpr unsigned kWaitHintNs = 1000;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long limit) {
    const unsigned a = smem_addr(bar);
    if (limit < kShortWait) {
        for (long long k = 0; k < limit; k++) {
            unsigned done;
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                : "=r"(done)
                : "r"(a), "r"(parity)
                : "memory");
            if (done) return true;
        }
        return false;
    }
    for (long long k = 0; k < limit; k++) {
        unsigned done;
        // the suspend-time hint (ns) caps how long one poll may park the thread, so `limit` polls
        // bound the wait to about limit microseconds; a completed phase wakes the thread at once
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity), "r"(kWaitHintNs)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ unsigned long long lo16(const void* p) { return (unsigned long long)p & ~15ull; }
__device__ __forceinline__ unsigned long long hi16(const void* p) { return ((unsigned long long)p + 15ull) & ~15ull; }

// One bulk copy group per tile m: its off-diagonal blocks and column indices (16-byte-rounded
// ranges), its kTileRows + 1 row pointers and the slices of up to three epilogue vectors (these
// start on 16-byte boundaries: tile offsets are multiples of 128 and 768 bytes).  All
// completions land on one mbarrier.
template <typename MT, typename VT>
__device__ __forceinline__ void issue_tile(int m, int V, const int* rowptr, const int* col, const MT* A, int nvec,
                                           const VT* const* vecs, unsigned char* stage, const StageLayout& K,
                                           unsigned long long* bar, unsigned long long pol) {
    const int r0 = m * kTileRows, nr = min(kTileRows, V - r0);
    const int k0 = __ldg(rowptr + r0), k1 = __ldg(rowptr + r0 + nr);
    const unsigned long long alo = lo16(A + (size_t)k0 * 9), ahi = hi16(A + (size_t)k1 * 9);
    const unsigned long long clo = lo16(col + k0), chi = hi16(col + k1);
    const unsigned ab = (unsigned)(ahi - alo), cb = (unsigned)(chi - clo);
    const unsigned rb = ((unsigned)(nr + 1) * 4u + 15u) & ~15u;
    const unsigned vb = ((unsigned)nr * 3u * (unsigned)sizeof(VT) + 15u) & ~15u;
    mbar_arrive_expect_tx(bar, ab + cb + rb + (unsigned)nvec * vb);
    if (ab) bulk_load_hint(stage, (const void*)alo, ab, bar, pol);
    if (cb) bulk_load_hint(stage + K.c_off, (const void*)clo, cb, bar, pol);
    bulk_load_hint(stage + K.r_off, rowptr + r0, rb, bar, pol);
    for (int v = 0; v < nvec; v++)
        bulk_load(stage + K.v_off + v * tile_vec_bytes<VT>(), vecs[v] + (size_t)r0 * 3, vb, bar);
}

// explicit fused multiply-add, a * b + c rounded once (the library is built without implicit
// contraction so that every kernel instantiation rounds alike; hot loops state their FMAs)
__device__ __forceinline__ double fmadd(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmadd(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <int N>
struct IntC {
    static constexpr int value = N;
};

// Off-diagonal row sum y = sum_j B_ij x_j of the folded operator (B_ij = D_i^-1 A'_ij, blocks
// kb..ke-1) for node row i, with x_j formed by gat(j, x) from the vectors at node j; the caller
// adds the identity diagonal block's x_i.  Eight lanes share a row and each lane takes whole 3x3 blocks
// (lane l: the row's blocks l, l+8, ...); the column index and the three x components are loaded
// once per block.  blk(k) / cix(k) give block k's values and column index (from the staged tile
// in shared memory, or from global memory).  The three sums are combined with xor shuffles in a
// fixed order, so staged and direct sweeps give bitwise identical results.  Products and sums
// are formed in the matrix type MT (FP32 accumulation on the mixed path).  The result is valid
// on lane 0 of the group; `active` false contributes zeros so the whole warp can shuffle.
template <typename MT, typename VT, class BLK, class CIX, class GAT>
__device__ __forceinline__ void row_apply(bool active, int lane8, int kb, int ke, BLK blk, CIX cix, GAT gat, VT y[3]) {
    MT a0 = 0, a1 = 0, a2 = 0;
    if (active) {
        for (int k = kb + lane8; k < ke; k += kRowLanes) {
            const MT* bk = blk(k);
            MT m[9];
#pragma unroll
            for (int q = 0; q < 9; q++) m[q] = bk[q];
            const int j = cix(k);
            VT x[3];
            gat(j, x);
            const MT c0 = (MT)x[0], c1 = (MT)x[1], c2 = (MT)x[2];
            a0 = fmadd(m[2], c2, fmadd(m[1], c1, fmadd(m[0], c0, a0)));
            a1 = fmadd(m[5], c2, fmadd(m[4], c1, fmadd(m[3], c0, a1)));
            a2 = fmadd(m[8], c2, fmadd(m[7], c1, fmadd(m[6], c0, a2)));
        }
    }
#pragma unroll
    for (int o = kRowLanes / 2; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o, kRowLanes);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o, kRowLanes);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o, kRowLanes);
    }
    y[0] = (VT)a0;
    y[1] = (VT)a1;
    y[2] = (VT)a2;
}

// MT: matrix storage and SpMV accumulation type; VT: Krylov vector type (FP64 on both paths:
// FP32 vectors let the recursively updated residual drift away from the true one and the
// iteration stagnates).  Per instance, A holds the folded off-diagonal blocks D_i^-1 A'_ij
// (rowptr / col of K) and Dinv the FP64 inverses (used once, for b = M^-1 b').  STAGED: the
// SpMV sweeps read each tile's blocks, column indices, row pointers and epilogue vectors from
// a STAGES-deep shared-memory ring filled by bulk copies (the copy warp issues them up to
// STAGES tiles ahead of the row warps, completion on an mbarrier per stage), so a row's only
// global loads are its x gathers; the streamed matrix data carry an L2 evict-first hint, which keeps
// the Krylov vectors in L2.  The dynamic shared memory is STAGES * L.stage_bytes.  STAGES = 0:
// the lanes load everything from global memory.  Every variant computes the same bits.
template <typename MT, typename VT, int STAGES, class KS>
__global__ void __launch_bounds__(kKrylovThreads, 3) k_bicgstab(const __grid_constant__ KS src) {
    __shared__ double red[4 * kKrylovWarps];
    __shared__ int s_pause;                     // the instance's pause_at, read at a loop top
    constexpr bool STAGED = STAGES > 0;
    constexpr int NST = STAGES > 0 ? STAGES : 1;
    __shared__ unsigned long long bar[NST];     // per ring stage: its tile copy has landed ("full")
    __shared__ unsigned long long ebar[NST];    // per ring stage: every row warp is done with it ("empty")
    extern __shared__ __align__(128) unsigned char stage_mem[];
    int pl, np;   // this CTA's index among the instance's np CTAs
    double rtol;
    const KrylovInst& KI = src.get(pl, np, rtol);
    const StageLayout& L = src.lay;
    const KrylovArgs K = KI.K;
    const MT* __restrict__ A = (const MT*)KI.A;
    const double* __restrict__ Dinv = KI.Dinv;
    VT* __restrict__ b = KI.vec[0];
    VT* __restrict__ q = KI.vec[3];
    VT* __restrict__ As = KI.vec[6];
    VT* __restrict__ ubest = KI.vec[7];
    // u, r, p, Ap in two copies: the sweep that applies an iteration's update reads the old
    // copy (its gathers at neighbour rows too) and writes the new one
    VT* const U2[2] = {KI.vec[1], KI.vec[8]};
    VT* const R2[2] = {KI.vec[2], KI.vec[9]};
    VT* const P2[2] = {KI.vec[4], KI.vec[10]};
    VT* const AP2[2] = {KI.vec[5], KI.vec[11]};
    const int V = K.V;
    const int VG = K.vgrid;
    const bool rows = threadIdx.x < kKrylovRowThreads;   // row warp (else: the copy warp)
    const int pstride = np * kKrylovRowThreads;           // reduction-free loops: physical CTAs
    const int pt0 = pl * kKrylovRowThreads + threadIdx.x;
    const int lane8 = threadIdx.x % kRowLanes;
    const int li = threadIdx.x / kRowLanes;   // row of the tile this lane group works on
    const int ntiles = (V + kTileRows - 1) / kTileRows;   // >= VG: every virtual CTA has a tile
    const int SUM = 0, MAX = 1;
    KrylovCtl* ctl = K.ctl;
    int nred = 0;      // reductions so far; selects the partial buffer
    unsigned epoch = 0;   // barrier arrivals this CTA waits for (grid_sync)
    unsigned tc = 0;   // tiles consumed by this CTA: stage tc % NST, mbarrier parity (tc / NST) & 1
    unsigned issued = 0;   // tile copies issued (the copy warp's issuing lane)
    bool copy_stop = false;   // the issuing lane gave up a wait: no more copies
    bool wait_failed = false;
    unsigned long long pol = 0;
    auto pbuf = [&]() { return K.part + (size_t)(nred & 1) * VG * 4; };
    auto stage = [&](unsigned c) { return stage_mem + (c % NST) * L.stage_bytes; };
    const long long bar_limit = K.spin_limit > 0 ? K.spin_limit : kBarrierSpinLimit;
    const long long copy_limit = K.copy_limit > 0 ? K.copy_limit : kMbarSpinLimit;
    // Before a CTA leaves on an error, the bulk copies it issued must have landed in its shared
    // memory: the issuing lane waits (bounded by the default limit) for its last copy into every
    // ring stage.
    auto drain = [&]() {
        if (STAGED && threadIdx.x == kKrylovRowThreads)
            for (unsigned it = issued > (unsigned)NST ? issued - NST : 0u; it < issued; it++)
                mbar_wait(&bar[it % NST], (it / NST) & 1u, kMbarSpinLimit);
    };
    // grid barrier; false (after draining the tile ring) when some CTA gave up: return at once
    auto gsync = [&]() -> bool {
        if (grid_sync(ctl, np, epoch, bar_limit)) return true;
        drain();
        return false;
    };

    if (STAGED) {
        if (threadIdx.x == 0) {
            for (int s = 0; s < NST; s++) {
                mbar_init(&bar[s], 1);
                mbar_init(&ebar[s], kKrylovWarps);
            }
            mbar_init_fence();
        }
        if (threadIdx.x == kKrylovRowThreads) pol = policy_evict_first();
        __syncthreads();
    }

    // One SpMV sweep: this CTA runs virtual CTAs v = pl, pl + np, ... < VG, each over tiles
    // m = v, v + VG, ... < ntiles.  y = sum_j B_ij x_j over the off-diagonal blocks of each row,
    // x_j = gat(j) from the vectors at node j; lane 0 of each row group calls epi(i, y, ev) with
    // ev(v, c) = component c of epilogue vector v at row i (NV vectors; read from the staged tile
    // or from global memory), from which the epilogue forms the diagonal term; fin(v) closes
    // virtual CTA v (its partial).
    // STAGED: the copy warp's issuing lane walks the same tile sequence up to NST tiles ahead,
    // filling ring stage (item % NST) once every row warp has released the stage's previous item
    // (its "empty" mbarrier: one arrival per row warp and item) and that item's copy has landed;
    // the row warps wait on the stage's "full" mbarrier, so each warp proceeds at its own pace.
    // Every wait is bounded: a row warp whose wait runs out flags the error and stops reading the
    // ring for the rest of the sweep (still waiting for and releasing every item, so the issuing
    // lane never waits on a release that cannot come); an issuing lane whose wait runs out flags
    // the error and issues nothing more; the next grid barrier then ends the kernel.
    // Called by the whole CTA.
    auto sweep = [&](auto nvc, const VT* const* vecs, auto&& gat, auto&& epi, auto&& fin) {
        constexpr int NV = decltype(nvc)::value;
        int nitems = 0;   // tiles of this CTA in this sweep
        for (int v = pl; v < VG; v += np) nitems += (ntiles - v + VG - 1) / VG;
        if (!rows) {
            if (STAGED) {
                // the whole warp walks the items (it stays converged for the CTA barriers that
                // follow); its first lane waits and issues, the stop decision is broadcast
                const bool issuer = threadIdx.x == kKrylovRowThreads;
                if (issuer) fence_proxy_async_global();
                for (int v = pl; v < VG; v += np)
                    for (int m = v; m < ntiles; m += VG) {
                        if (!copy_stop) {
                            bool stop = false;
                            if (issuer) {
                                const unsigned item = issued;
                                if (item >= (unsigned)NST) {
                                    // the stage's previous item: released by every row warp, and
                                    // its copy landed (the row warps waited for it)
                                    const unsigned par = ((item - NST) / NST) & 1u;
                                    stop = !mbar_wait(&ebar[item % NST], par, kMbarSpinLimit) ||
                                           !mbar_wait(&bar[item % NST], par, kMbarSpinLimit);
                                }
                                if (stop) atomicExch(&ctl->err, 1);
                                else issue_tile<MT, VT>(m, V, K.rowptr, K.col, A, NV, vecs, stage(item), L,
                                                        &bar[item % NST], pol);
                            }
                            copy_stop = __shfl_sync(0xffffffffu, stop, 0);
                            if (!copy_stop) issued++;
                        }
                        __syncwarp();
                    }
            }
            tc += nitems;
            return;
        }
        for (int v = pl; v < VG; v += np) {
            for (int m = v; m < ntiles; m += VG) {
                const int i = m * kTileRows + li;
                const bool act = i < V;
                VT y[3];
                if (STAGED) {
                    // a wait that runs out flags the error once; the warp then treats the rest of
                    // the sweep's rows as absent (a stage that may not have landed is never read,
                    // so no index comes from stale shared memory) and the next barrier returns.
                    // It still waits (with the default bound) for every tile before releasing
                    // it, so it never runs ahead of the copies: the ring stays in step and every
                    // copy has landed before the kernel returns.
                    {
                        const unsigned par = (tc / NST) & 1u;
                        const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar[tc % NST], par,
                                                                          wait_failed ? kMbarSpinLimit : copy_limit));
                        if (!ok && !wait_failed) {
                            wait_failed = true;
                            if ((threadIdx.x & 31) == 0) atomicExch(&ctl->err, 1);
                            __syncwarp();
                            (void)mbar_wait(&bar[tc % NST], par, kMbarSpinLimit);
                        }
                    }
                    const bool use = act && !wait_failed;
                    const unsigned char* st = stage(tc);
                    const int* sR = (const int*)(st + L.r_off);
                    const int k0 = wait_failed ? 0 : sR[0];
                    const MT* sA = (const MT*)(st + ((unsigned long long)(A + (size_t)k0 * 9) & 15ull));
                    const int* sC = (const int*)(st + L.c_off + ((unsigned long long)(K.col + k0) & 15ull));
                    const VT* sV = (const VT*)(st + L.v_off);
                    const int kb = use ? sR[li] : 0, ke = use ? sR[li + 1] : 0;
                    row_apply<MT, VT>(
                        use, lane8, kb, ke, [&](int k) { return sA + (size_t)(k - k0) * 9; },
                        [&](int k) { return sC[k - k0]; }, gat, y);
                    if (use && lane8 == 0)
                        epi(i, y, [&](int w, int c) { return sV[w * (tile_vec_bytes<VT>() / sizeof(VT)) + 3 * li + c]; });
                } else {
                    const int kb = act ? __ldg(K.rowptr + i) : 0, ke = act ? __ldg(K.rowptr + i + 1) : 0;
                    row_apply<MT, VT>(
                        act, lane8, kb, ke, [&](int k) { return A + (size_t)k * 9; },
                        [&](int k) { return __ldg(K.col + k); }, gat, y);
                    if (act && lane8 == 0) epi(i, y, [&](int w, int c) { return ldv(vecs[w] + 3 * i + c); });
                }
                if (STAGED) {
                    // this warp is done with the stage: one arrival per warp releases it
                    __syncwarp();
                    if ((threadIdx.x & 31) == 0) mbar_arrive(&ebar[tc % NST]);
                    tc++;
                }
            }
            fin(v);
        }
    };

    int cur = 0;   // the copy of u, r, p, Ap that holds the current iterate
    const bool resume = src.resuming();
    // b <- M^-1 b'
    for (int i = pt0; !resume && rows && i < V; i += pstride) {
        const double* d = Dinv + (size_t)i * 9;
        const double b0 = K.bs[3 * i], b1 = K.bs[3 * i + 1], b2 = K.bs[3 * i + 2];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const VT y = (VT)(d[3 * c] * b0 + d[3 * c + 1] * b1 + d[3 * c + 2] * b2);
            b[3 * i + c] = y;
            U2[0][3 * i + c] = y;
        }
    }
    if (!resume && !gsync()) return;
    // r = b - M^-1 A u, q = r, p = r; norms and rho
    {
        double rnorm, rho, rhop, alpha, omega, beta, tol, best;
        int it, best_it;
        bool pending, upd;
        if (resume) {   // the scalars of the paused solve (written by the previous launch)
            rnorm = ctl->s_rnorm;
            tol = ctl->s_tol;
            rho = ctl->s_rho;
            rhop = 1.0;   // dead at a loop top (set from rho before its use)
            alpha = ctl->s_alpha;
            omega = ctl->s_omega;
            beta = ctl->s_beta;
            best = ctl->s_best;
            it = ctl->s_it;
            best_it = ctl->s_best_it;
            pending = ctl->s_pending != 0;
            upd = ctl->s_upd != 0;
            cur = ctl->s_cur;
            nred = ctl->s_nred;
        } else {
        double vals[4] = {0, 0, 0, 0};
        const int ism[4] = {MAX, MAX, SUM, SUM};
        const VT* ev2[2] = {b, U2[0]};
        const VT* x0 = U2[0];
        VT* const r = R2[0];
        VT* const p = P2[0];
        VT* const Ap = AP2[0];
        sweep(
            IntC<2>{}, ev2,
            [&](int j, VT (&x)[3]) {
                x[0] = ldv(x0 + 3 * j);
                x[1] = ldv(x0 + 3 * j + 1);
                x[2] = ldv(x0 + 3 * j + 2);
            },
            [&](int i, const VT* y, auto&& ev) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const VT bb = ev(0, c);
                    const VT rr = bb - (ev(1, c) + y[c]);
                    r[3 * i + c] = rr;
                    q[3 * i + c] = rr;
                    p[3 * i + c] = rr;
                    Ap[3 * i + c] = 0;
                    vals[0] = fmax(vals[0], fabs((double)rr));
                    vals[1] = fmax(vals[1], fabs((double)bb));
                    vals[2] += (double)rr * (double)rr;
                }
            },
            [&](int v) {
                block_partial<4>(vals, ism, pbuf(), v, red);
                vals[0] = vals[1] = vals[2] = vals[3] = 0.0;
            });
        if (!gsync()) return;
        double rd[4];
        grid_allreduce<4>(pbuf(), VG, ism, rd, red);
        nred++;
        rnorm = rd[0];
        const double bnorm = rd[1];
        if (pl == 0 && threadIdx.x == 0) ctl->bnorm = bnorm;   // read back with the outcome
        rho = rd[2], rhop = 1.0, alpha = 1.0, omega = 1.0, beta = 0.0;
        it = 0;
        tol = K.atol + bnorm * rtol;
        // best iterate so far: past its attainable accuracy BiCGSTAB's residual drifts back up,
        // so on stagnation (no new best for kStall iterations) or at max_lin_it the best one is
        // used.  It is saved lazily: when an iteration sets a new best (`pending`), the next
        // update, which reads u anyway, writes that u to ubest.
        best = rnorm;
        best_it = 0;
        pending = true;
        upd = false;
        }
        // An iteration's update (u += alpha p + omega s, r = s - omega As, p = beta (p - omega Ap)
        // + r) is either its own vector pass with a grid barrier (fuse_update 0) or applied by the
        // first sweep of the next iteration (fuse_update 1): that sweep's epilogue updates its own
        // rows into the other copy, and its gathers form the new p of the neighbour rows from the
        // old copies, with the same arithmetic, so the bits are those of the separate pass.  The
        // stopping test of the updated residual then follows that sweep; when it stops the solve,
        // the product A p that sweep formed is not used.
        const bool fuse = src.fuse_update(KI);
        while (upd || (rnorm > tol && it < K.maxit && it - best_it < kStall)) {
            if (src.done_counter()) {   // a pause requested before the last iteration's second barrier
                if (threadIdx.x == 0) s_pause = *(volatile int*)&ctl->pause_at;
                __syncthreads();
                if (s_pause != 0 && it >= s_pause) {
                    if (pl == 0 && threadIdx.x == 0) {
                        ctl->s_rnorm = rnorm;
                        ctl->s_tol = tol;
                        ctl->s_rho = rho;
                        ctl->s_alpha = alpha;
                        ctl->s_omega = omega;
                        ctl->s_beta = beta;
                        ctl->s_best = best;
                        ctl->s_it = it;
                        ctl->s_best_it = best_it;
                        ctl->s_pending = pending ? 1 : 0;
                        ctl->s_upd = upd ? 1 : 0;
                        ctl->s_cur = cur;
                        ctl->s_nred = nred;
                        ctl->paused = 1;
                    }
                    return;
                }
            }
            // [update of iteration it] and Ap = M^-1 A p, gamma = q . Ap
            {
                double g[4] = {0, 0, 0, 0};
                const int gm[4] = {SUM, MAX, SUM, SUM};
                if (!upd) {
                    const VT* const p = P2[cur];
                    VT* const Ap = AP2[cur];
                    const VT* ev2[2] = {q, p};
                    sweep(
                        IntC<2>{}, ev2,
                        [&](int j, VT (&x)[3]) {
                            x[0] = ldv(p + 3 * j);
                            x[1] = ldv(p + 3 * j + 1);
                            x[2] = ldv(p + 3 * j + 2);
                        },
                        [&](int i, const VT* y, auto&& ev) {
#pragma unroll
                            for (int c = 0; c < 3; c++) {
                                const VT apc = ev(1, c) + y[c];
                                Ap[3 * i + c] = apc;
                                g[0] += (double)ev(0, c) * (double)apc;
                            }
                        },
                        [&](int v) {
                            block_partial<1>(g, gm, pbuf(), v, red);
                            g[0] = 0.0;
                        });
                } else {
                    const VT al = (VT)alpha, om = (VT)omega, be = (VT)beta;
                    const VT* const uo = U2[cur];
                    const VT* const ro = R2[cur];
                    const VT* const po = P2[cur];
                    const VT* const apo = AP2[cur];
                    VT* const un = U2[cur ^ 1];
                    VT* const rn = R2[cur ^ 1];
                    VT* const pn = P2[cur ^ 1];
                    VT* const apn = AP2[cur ^ 1];
                    const bool save = pending;
                    const VT* ev6[6] = {q, uo, po, apo, As, ro};
                    sweep(
                        IntC<6>{}, ev6,
                        [&](int j, VT (&x)[3]) {   // the new p at node j
#pragma unroll
                            for (int c = 0; c < 3; c++) {
                                const VT apk = ldv(apo + 3 * j + c);
                                const VT s = fmadd(-al, apk, ldv(ro + 3 * j + c));
                                const VT rk = fmadd(-om, ldv(As + 3 * j + c), s);
                                x[c] = fmadd(fmadd(-om, apk, ldv(po + 3 * j + c)), be, rk);
                            }
                        },
                        [&](int i, const VT* y, auto&& ev) {
#pragma unroll
                            for (int c = 0; c < 3; c++) {
                                const int k = 3 * i + c;
                                const VT apk = ev(3, c), pk = ev(2, c);
                                const VT s = fmadd(-al, apk, ev(5, c));
                                VT uk = ev(1, c);
                                if (save) ubest[k] = uk;
                                uk = fmadd(al, pk, uk);
                                uk = fmadd(om, s, uk);
                                un[k] = uk;
                                const VT rk = fmadd(-om, ev(4, c), s);
                                rn[k] = rk;
                                const VT pnk = fmadd(fmadd(-om, apk, pk), be, rk);
                                pn[k] = pnk;
                                g[1] = fmax(g[1], fabs((double)rk));
                                const VT apc = pnk + y[c];
                                apn[k] = apc;
                                g[0] += (double)ev(0, c) * (double)apc;
                            }
                        },
                        [&](int v) {
                            block_partial<2>(g, gm, pbuf(), v, red);
                            g[0] = g[1] = 0.0;
                        });
                }
                if (!gsync()) return;
                if (!upd) {
                    grid_allreduce<1>(pbuf(), VG, gm, g, red);
                } else {
                    grid_allreduce<2>(pbuf(), VG, gm, g, red);
                    cur ^= 1;
                    rnorm = g[1];
                    pending = rnorm < best;   // identical decision in every CTA of the instance
                    if (pending) {
                        best = rnorm;
                        best_it = it;
                    }
                    if (!(rnorm > tol && it < K.maxit && it - best_it < kStall)) break;
                }
                nred++;
                it++;
                alpha = rho / g[0];
            }
            // (f)-(g): As = M^-1 A (r - alpha Ap); omega, next rho
            {
                double w[4] = {0, 0, 0, 0};
                const int wm[4] = {SUM, SUM, SUM, SUM};
                const VT al = (VT)alpha;
                const VT* const r = R2[cur];
                const VT* const Ap = AP2[cur];
                const VT* ev3[3] = {r, Ap, q};
                sweep(
                    IntC<3>{}, ev3,
                    [&](int j, VT (&x)[3]) {   // the s the epilogue forms
#pragma unroll
                        for (int c = 0; c < 3; c++) x[c] = fmadd(-al, ldv(Ap + 3 * j + c), ldv(r + 3 * j + c));
                    },
                    [&](int i, const VT* y, auto&& ev) {
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            const VT s = fmadd(-al, ev(1, c), ev(0, c));   // the s the gathers form
                            const VT asc = s + y[c];
                            As[3 * i + c] = asc;
                            w[0] += (double)asc * (double)s;
                            w[1] += (double)asc * (double)asc;
                            w[2] += (double)asc * (double)ev(2, c);
                        }
                    },
                    [&](int v) {
                        block_partial<3>(w, wm, pbuf(), v, red);
                        w[0] = w[1] = w[2] = 0.0;
                    });
                // the pause request: after this iteration's first barrier (which every CTA
                // reaches after its last loop-top read) and before its second one (which every
                // CTA passes before its next loop-top read)
                if (src.done_counter() && pl == 0 && threadIdx.x == 0 && *(volatile int*)&ctl->pause_at == 0 &&
                    *(volatile unsigned*)src.done_counter() >= src.pause_threshold())
                    *(volatile int*)&ctl->pause_at = it;
                if (!gsync()) return;
                grid_allreduce<3>(pbuf(), VG, wm, w, red);
                nred++;
                omega = w[0] / w[1];
                rhop = rho;
                rho = -1.0 * omega * w[2];
                beta = (rho * alpha) / (rhop * omega);
                upd = fuse;
            }
            if (fuse) continue;
            // (h)-(i) and the next search direction (c) as a pass of its own, in place
            {
                double mx[4] = {0, 0, 0, 0};
                const int mm[4] = {MAX, MAX, MAX, MAX};
                const VT al = (VT)alpha, om = (VT)omega, be = (VT)beta;
                VT* const uu = U2[cur];
                VT* const r = R2[cur];
                VT* const p = P2[cur];
                const VT* const Ap = AP2[cur];
                auto upd1 = [&](int k) {
                    const VT apk = ldv(Ap + k), pk = ldv(p + k);
                    const VT s = fmadd(-al, apk, ldv(r + k));
                    VT uk = ldv(uu + k);
                    if (pending) ubest[k] = uk;
                    uk = fmadd(al, pk, uk);
                    uk = fmadd(om, s, uk);
                    uu[k] = uk;
                    const VT rk = fmadd(-om, ldv(As + k), s);
                    r[k] = rk;
                    p[k] = fmadd(fmadd(-om, apk, pk), be, rk);
                    mx[0] = fmax(mx[0], fabs((double)rk));
                };
                // two elements per thread with 16-byte accesses (the vectors start on 256-byte
                // boundaries); the arithmetic is that of upd1, element by element
                auto upd2 = [&](int k2) {
                    using V2 = typename std::conditional<sizeof(VT) == 8, double2, float2>::type;
                    const V2 a2 = __ldcg(reinterpret_cast<const V2*>(Ap) + k2);
                    const V2 p2 = __ldcg(reinterpret_cast<const V2*>(p) + k2);
                    const V2 r2 = __ldcg(reinterpret_cast<const V2*>(r) + k2);
                    const V2 u2 = __ldcg(reinterpret_cast<const V2*>(uu) + k2);
                    const V2 s2 = __ldcg(reinterpret_cast<const V2*>(As) + k2);
                    if (pending) reinterpret_cast<V2*>(ubest)[k2] = u2;
                    V2 un, rn, pn;
                    {
                        const VT s = fmadd(-al, (VT)a2.x, (VT)r2.x);
                        VT uk = fmadd(al, (VT)p2.x, (VT)u2.x);
                        uk = fmadd(om, s, uk);
                        const VT rk = fmadd(-om, (VT)s2.x, s);
                        un.x = uk;
                        rn.x = rk;
                        pn.x = fmadd(fmadd(-om, (VT)a2.x, (VT)p2.x), be, rk);
                        mx[0] = fmax(mx[0], fabs((double)rk));
                    }
                    {
                        const VT s = fmadd(-al, (VT)a2.y, (VT)r2.y);
                        VT uk = fmadd(al, (VT)p2.y, (VT)u2.y);
                        uk = fmadd(om, s, uk);
                        const VT rk = fmadd(-om, (VT)s2.y, s);
                        un.y = uk;
                        rn.y = rk;
                        pn.y = fmadd(fmadd(-om, (VT)a2.y, (VT)p2.y), be, rk);
                        mx[0] = fmax(mx[0], fabs((double)rk));
                    }
                    reinterpret_cast<V2*>(uu)[k2] = un;
                    reinterpret_cast<V2*>(r)[k2] = rn;
                    reinterpret_cast<V2*>(p)[k2] = pn;
                };
                for (int v = pl; rows && v < VG; v += np) {
                    // element pairs (16-byte accesses), virtual CTA v's share; each element is
                    // updated on its own, the pairing only widens the loads
                    const int n2 = (3 * V) / 2;
                    for (int k2 = v * kKrylovRowThreads + threadIdx.x; k2 < n2; k2 += VG * kKrylovRowThreads) upd2(k2);
                    if ((3 * V) % 2 && v == 0 && threadIdx.x == 0) upd1(3 * V - 1);
                    block_partial<1>(mx, mm, pbuf(), v, red);
                    mx[0] = 0.0;
                }
                if (!gsync()) return;
                grid_allreduce<1>(pbuf(), VG, mm, mx, red);
                nred++;
                rnorm = mx[0];
                pending = rnorm < best;   // identical decision in every CTA of the instance
                if (pending) {
                    best = rnorm;
                    best_it = it;
                }
            }
        }
        const bool conv = rnorm <= tol;
        // x = S u; state += x; sol = -x.  Without convergence the best iterate is u itself when
        // the last iteration set it (not saved yet), else ubest.
        const VT* ux = (conv || pending) ? U2[cur] : ubest;
        for (int i = pt0; rows && i < V; i += pstride) {
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
        if (pl == 0 && threadIdx.x == 0) {
            ctl->iterations = it;
            ctl->converged = conv ? 1 : 0;
            ctl->rnorm = conv ? rnorm : best;
        }
        if (src.done_counter() && threadIdx.x == 0) atomicAdd(src.done_counter(), 1u);   // this CTA's instance is done
    }
}

}  // namespace sw2
