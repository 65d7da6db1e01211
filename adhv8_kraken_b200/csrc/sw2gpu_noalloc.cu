// sw2gpu_noalloc.cu -- the allocation-free variant of the device linear solve.
//
// Some callers cannot let a library allocate GPU memory during a solve: applications
// that own all device memory themselves (a fixed arena sized once at start-up, as a
// coupled model's time loop or a long-running serving process does) and must not have
// a call inside their step run cudaMalloc, which can synchronize the device, can fail
// half-way through a run, and is invisible to their memory accounting.  For them,
// sw2gpu_bcsr_solve_noalloc() solves a 3x3-block CSR system that lives entirely in the
// caller's device buffers, using as its only work memory the file-scope array below.
//
// The array is a static __device__ allocation of kScratchDoubles doubles (16.7 MB, checked
// below): every GPU that loads this library holds it until the process exits.  Its size
// bounds the problem: at most SW2GPU_NOALLOC_MAX_NODES node rows and
// SW2GPU_NOALLOC_MAX_BLOCKS blocks; larger systems are rejected.  All calls share the one
// array and it keeps the previous call's contents, so the barrier/control words are cleared
// on every call, and two calls that overlap on the GPU (different streams, or different host
// threads at once) race on it and corrupt each other's results.
//
// The caller's block structure is checked before anything is written into the array:
// row_ptr[0] = 0 and row_ptr[nnodes] = nnzb on the host (8 bytes read back), then on the
// device every row range inside [0, nnzb], every column index inside [0, nnodes) and exactly
// one diagonal block per row; a system that fails is rejected with SW2GPU_E_ARG and no
// further kernel runs, so the fold's packed positions (which assume one diagonal block per
// row) always stay inside their region.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/sw2gpu.h"
#include "sw2_krylov.cuh"

using namespace sw2;

namespace {

constexpr double kSmall = 2.220446049250313e-16;   // DBL_EPSILON, the spv_jacobi floor
constexpr int kMaxNodes = SW2GPU_NOALLOC_MAX_NODES;
constexpr int kMaxBlocks = SW2GPU_NOALLOC_MAX_BLOCKS;
constexpr int kMaxGrid = (kMaxNodes + kKrylovThreads - 1) / kKrylovThreads;   // persistent-kernel blocks
constexpr size_t kAlign = 32;                                                 // doubles = 256 bytes
constexpr size_t al(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }
// layout (in doubles): control word, partials, S, b', Dinv, folded off-diagonal blocks, their
// row pointers and column indices (int32, two per double), the Krylov vectors
constexpr size_t kOffCtl = 0;
constexpr size_t kOffPart = kOffCtl + al((sizeof(KrylovCtl) + 7) / 8);
constexpr size_t kOffS = kOffPart + al(2ull * kMaxGrid * 4);
constexpr size_t kOffB = kOffS + al(3ull * kMaxNodes);
constexpr size_t kOffDinv = kOffB + al(3ull * kMaxNodes);
constexpr size_t kOffA = kOffDinv + al(9ull * kMaxNodes);
constexpr size_t kOffRp = kOffA + al(9ull * kMaxBlocks);
constexpr size_t kOffCol = kOffRp + al((kMaxNodes + 2) / 2);
constexpr size_t kOffVec = kOffCol + al((kMaxBlocks + 1) / 2);
constexpr size_t kScratchDoubles = kOffVec + kKrylovVectors * al(3ull * kMaxNodes);
static_assert(kScratchDoubles * sizeof(double) > 16650000 && kScratchDoubles * sizeof(double) < 16750000,
              "the work array is documented as 16.7 MB");
// the structure-check word sits in the control region, after the KrylovCtl record
constexpr size_t kCheckByte = 192;
static_assert(sizeof(KrylovCtl) <= kCheckByte && kCheckByte + sizeof(int) <= kAlign * sizeof(double),
              "control region layout");
constexpr int kBadRowRange = 1, kBadColumn = 2, kBadDiagonal = 4;   // bits of the check word

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_setup_mutex;
double* g_scratch_dev[128] = {nullptr};   // device address of the array, per device ordinal

}  // namespace

// error text shared with sw2gpu_last_error() (defined in sw2gpu.cu, not exported)
void sw2gpu_internal_set_error(const char* msg);

namespace {

int na_fail(int code, const char* msg) {
    sw2gpu_internal_set_error(msg);
    return code;
}

// Structure check, one thread per node row: the row's range inside [0, nnzb] and ordered,
// its column indices inside [0, V), exactly one diagonal block.  Reads only inside the
// caller's arrays (row_ptr[V + 1], col[nnzb]): a column index is read only once its row range
// is known to be in bounds.  Failures set bits of *bad.
__global__ void k_na_check(int V, int nnzb, const int* __restrict__ rowptr, const int* __restrict__ col,
                           int* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const int kb = rowptr[i], ke = rowptr[i + 1];
    if (kb < 0 || kb > ke || ke > nnzb) {
        atomicOr(bad, kBadRowRange);
        return;
    }
    int ndiag = 0, badcol = 0;
    for (int k = kb; k < ke; k++) {
        const int j = col[k];
        if (j < 0 || j >= V) badcol = 1;
        ndiag += (j == i) ? 1 : 0;
    }
    if (badcol) atomicOr(bad, kBadColumn);
    if (ndiag != 1) atomicOr(bad, kBadDiagonal);
}

// S = 1/sqrt(max |row entry|) (spv_jacobi) and b' = S rhs, one thread per node row
__global__ void k_na_rowscale(int V, const int* __restrict__ rowptr, const double* __restrict__ val,
                              const double* __restrict__ rhs, double* __restrict__ S, double* __restrict__ bs) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= V) return;
    double mx[3] = {0.0, 0.0, 0.0};
    for (int k = rowptr[n]; k < rowptr[n + 1]; k++)
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) mx[r] = fmax(mx[r], fabs(val[(size_t)k * 9 + 3 * r + c]));
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const double sv = (mx[r] < kSmall) ? 1.0 / sqrt(kSmall) : 1.0 / sqrt(fabs(mx[r]));
        S[3 * n + r] = sv;
        bs[3 * n + r] = rhs[3 * n + r] * sv;
    }
}

// The Krylov operator with the block-Jacobi inverse folded in, one thread per node row: the
// inverse D_i^-1 of the scaled diagonal block S_i A_ii S_i, and the row's off-diagonal blocks
// D_i^-1 S_i A_ij S_j with their column indices, packed without the diagonal (position k - i
// for blocks before it, k - i - 1 after it).  Runs only on a structure k_na_check accepted
// (one diagonal block per row), so the positions of row i are [row_ptr[i] - i,
// row_ptr[i + 1] - i - 1), inside the region of nnzb - V blocks; a singular diagonal block
// sets `singular`.
__global__ void k_na_fold(int V, const int* __restrict__ rowptr, const int* __restrict__ col,
                          const double* __restrict__ val, const double* __restrict__ S, double* __restrict__ dinv,
                          double* __restrict__ aoff, int* __restrict__ orp, int* __restrict__ ocol,
                          int* __restrict__ singular) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const int kb = rowptr[i], ke = rowptr[i + 1];
    int dp = -1;
    for (int k = kb; k < ke; k++)
        if (col[k] == i) dp = k;
    double d[9];
    if (dp < 0) {
        *singular = 1;
#pragma unroll
        for (int q = 0; q < 9; q++) d[q] = (q % 4 == 0) ? 1.0 : 0.0;
    } else {
        double a[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) a[3 * r + c] = val[(size_t)dp * 9 + 3 * r + c] * (S[3 * i + r] * S[3 * i + c]);
        if (!inv3(a, d)) *singular = 1;
    }
#pragma unroll
    for (int q = 0; q < 9; q++) dinv[(size_t)i * 9 + q] = d[q];
    orp[i] = kb - i;
    if (i == V - 1) orp[V] = ke - V;
    for (int k = kb; k < ke; k++) {
        if (k == dp) continue;
        const int j = col[k];
        double bq[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) bq[3 * r + c] = val[(size_t)k * 9 + 3 * r + c] * (S[3 * i + r] * S[3 * j + c]);
        const int ko = k - i - ((dp >= 0 && k > dp) ? 1 : 0);
        ocol[ko] = j;
        fold_block(d, bq, aoff + (size_t)ko * 9);
    }
}

// device address of the scratch array for the current device (looked up once per device)
int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return na_fail(SW2GPU_E_CUDA, "no current CUDA device");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return na_fail(SW2GPU_E_CUDA, cudaGetErrorString(e));
        g_scratch_dev[dev] = (double*)p;
    }
    *out = g_scratch_dev[dev];
    return SW2GPU_OK;
}

}  // namespace

extern "C" int sw2gpu_bcsr_solve_noalloc(int32_t nnodes, int32_t nnzb, const int32_t* row_ptr, const int32_t* col,
                                         const double* val, const double* rhs, double* x, double rtol, double atol,
                                         int32_t max_it, void* stream, int32_t* iterations) {
    if (nnodes <= 0 || nnzb <= 0 || !row_ptr || !col || !val || !rhs || !x || max_it <= 0)
        return na_fail(SW2GPU_E_ARG, "sw2gpu_bcsr_solve_noalloc: bad argument");
    if (nnodes > kMaxNodes || nnzb > kMaxBlocks) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "sw2gpu_bcsr_solve_noalloc: system of %d nodes / %d blocks exceeds the fixed scratch limit "
                 "of %d nodes / %d blocks",
                 nnodes, nnzb, kMaxNodes, kMaxBlocks);
        return na_fail(SW2GPU_E_ARG, buf);
    }
    double* sc = nullptr;
    int rc = scratch_for_current_device(&sc);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    KrylovCtl* ctl = reinterpret_cast<KrylovCtl*>(sc + kOffCtl);
    double* part = sc + kOffPart;
    double* S = sc + kOffS;
    double* bs = sc + kOffB;
    double* dinv = sc + kOffDinv;
    double* A = sc + kOffA;
    int* orp = reinterpret_cast<int*>(sc + kOffRp);
    int* ocol = reinterpret_cast<int*>(sc + kOffCol);
    double* v[kKrylovVectors];
    for (int k = 0; k < kKrylovVectors; k++) v[k] = sc + kOffVec + k * al(3ull * kMaxNodes);
    int* check = reinterpret_cast<int*>(reinterpret_cast<unsigned char*>(sc + kOffCtl) + kCheckByte);
    // the ends of the caller's row pointers, read back before any launch: they must describe
    // exactly nnzb blocks
    int32_t ends[2] = {-1, -1};
    cudaError_t e = cudaMemcpyAsync(&ends[0], row_ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ends[1], row_ptr + nnodes, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_fail(SW2GPU_E_CUDA, cudaGetErrorString(e));
    if (ends[0] != 0 || ends[1] != nnzb) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "sw2gpu_bcsr_solve_noalloc: row_ptr[0] = %d and row_ptr[%d] = %d do not describe nnzb = %d blocks",
                 ends[0], nnodes, ends[1], nnzb);
        return na_fail(SW2GPU_E_ARG, buf);
    }
    // the control words (barrier counter, error and result fields, structure-check word) must
    // start at zero; everything else is written before it is read
    if (cudaMemsetAsync(ctl, 0, kAlign * sizeof(double), st) != cudaSuccess)
        return na_fail(SW2GPU_E_CUDA, "cudaMemsetAsync of the control words failed");
    const int nb = (nnodes + 255) / 256;
    k_na_check<<<nb, 256, 0, st>>>(nnodes, nnzb, row_ptr, col, check);
    int bad = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, check, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_fail(SW2GPU_E_CUDA, cudaGetErrorString(e));
    if (bad) {
        char buf[240];
        snprintf(buf, sizeof buf, "sw2gpu_bcsr_solve_noalloc: bad block structure:%s%s%s",
                 (bad & kBadRowRange) ? " a row range outside [0, nnzb] or decreasing;" : "",
                 (bad & kBadColumn) ? " a column index outside [0, nnodes);" : "",
                 (bad & kBadDiagonal) ? " a row without exactly one diagonal block;" : "");
        return na_fail(SW2GPU_E_ARG, buf);
    }
    int* singular = reinterpret_cast<int*>(&ctl->pad);
    k_na_rowscale<<<nb, 256, 0, st>>>(nnodes, row_ptr, val, rhs, S, bs);
    k_na_fold<<<nb, 256, 0, st>>>(nnodes, row_ptr, col, val, S, dinv, A, orp, ocol, singular);
    if ((e = cudaGetLastError()) != cudaSuccess) return na_fail(SW2GPU_E_CUDA, cudaGetErrorString(e));
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bicgstab<double, double, 0, KrylovOne>,
                                                           kKrylovThreads, 0)) != cudaSuccess)
        return na_fail(SW2GPU_E_CUDA, cudaGetErrorString(e));
    const int grid = std::max(1, std::min({kMaxGrid, (nnodes + kKrylovThreads - 1) / kKrylovThreads,
                                           sms * std::max(per_sm, 1)}));
    // one instance, direct sweeps (no tile ring); the record is a kernel parameter
    static thread_local KrylovOne one;
    KrylovArgs& K = one.Q.K;
    K.V = nnodes;
    K.rowptr = orp;
    K.col = ocol;
    K.S = S;
    K.bs = bs;
    K.atol = atol;
    K.maxit = max_it;
    K.h = K.u = K.v = nullptr;
    K.sol = x;
    K.apply_inc = 0;
    K.part = part;
    K.ctl = ctl;
    K.vgrid = grid;
    K.fuse_update = krylov_fuse_update(nnodes);
    K.spin_limit = 0;   // the library's default bounds on the device waits
    K.copy_limit = 0;
    one.Q.A = A;
    one.Q.Dinv = dinv;
    for (int k = 0; k < kKrylovVectors; k++) one.Q.vec[k] = v[k];
    one.rtol = rtol;
    one.rtol_dev = nullptr;
    one.lay = StageLayout{0, 0, 0, 0};
    void* args[] = {(void*)&one};
    e = cudaLaunchCooperativeKernel((void*)k_bicgstab<double, double, 0, KrylovOne>, dim3(grid),
                                                dim3(kKrylovThreads), args, 0, st);
    if (e != cudaSuccess) return na_fail(SW2GPU_E_CUDA, cudaGetErrorString(e));
    KrylovCtl h;
    e = cudaMemcpyAsync(&h, ctl, sizeof(KrylovCtl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_fail(SW2GPU_E_CUDA, cudaGetErrorString(e));
    if (iterations) *iterations = h.iterations;
    if (h.err) return na_fail(SW2GPU_E_TIMEOUT, "Krylov grid barrier wait ran out");
    if (h.pad) return na_fail(SW2GPU_E_LINEAR, "a node row has a singular diagonal block");
    return h.converged ? SW2GPU_OK : na_fail(SW2GPU_E_LINEAR, "BiCGSTAB did not reach the tolerance");
}
