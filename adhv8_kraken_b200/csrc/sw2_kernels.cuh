// sw2_kernels.cuh -- assembly kernels of the SW2 Newton step (sm_100a).
//
// Assembly is atomic-free and deterministic: element kernels write their local
// contributions to per-element slots (coalesced), and gather kernels sum each node
// row / BCSR block over its contributing slots in the reference's element order
// (all 2D elements ascending, then the boundary edges ascending), which is the
// summation order of fe_sw2_resid / fe_global_matrix_assemble_sw2.
#pragma once
#include "sw2_krylov.cuh"   // inv3, fold_block
#include "sw2_mass.cuh"      // mass-balance terms
#include "sw2_physics.cuh"

namespace sw2 {

// Device view of one mesh instance (all arrays SoA, indices local to the instance).
struct DevMesh {
    int V, T, E, nnzb;
    const double *x, *y, *z;
    const int *en0, *en1, *en2, *emat;
    const double *djac, *gx0, *gy0, *gx1, *gy1, *gx2, *gy2;
    const unsigned char *efirst;      // bit i: element is the first 2D element holding its node i
    const unsigned char *dflag;       // [V] Dirichlet flags (bit0 PRS_DIR, bit1 VEL_DIR, bit2 VEL_PRS_DIR)
    const int *bn0, *bn1, *bkind, *bstr;
    const double *bdjac, *bnx, *bny;
    const MatParams *mats;
    const double *str_value;          // [nstrings] step value of each edge string's series
    const double *str_uv;             // [2 nstrings] NB OVH strings: step values of the vx, vy series
    const int *slot_ptr, *slot_idx;   // node -> residual slots in reference order
    const int *blk_ptr, *blk_src;     // BCSR block -> element-block slots in reference order
    const int *rowptr, *col, *blk_row, *dpos;
    const double *wsx, *wsy;          // [T] element wind surface stress (sw2gpu_set_wind), or null
    int qflag[3];                     // flags of global nodes 0..2 (fe_sw2_load.c:103 indexes by local id)
};

struct State {
    double *h, *u, *v;          // current
    const double *ho, *uo, *vo; // old
    const double *hoo, *uoo, *voo;
    const int *wd;
};

struct Norms {                  // get_residual_norms (src/fe/fe_newton.c:40-151)
    double rmax, l2sum, imax;
    int nan;
    int ngeneral;               // elements on the wet/dry (general) Jacobian list
};

// Everything the assembly kernels need about one instance (one mesh and its state).  A launch
// covers a list of instances -- a batch of independent solves of uneven size -- through a
// device table of these and a LaunchMap (instance ids[j] owns blocks boff[j]..boff[j+1]-1);
// a single solve is a batch of one.  Work indices inside a block are local to its instance,
// so every instance computes exactly what it computes alone.
struct __align__(16) Inst {
    DevMesh m;
    State s;
    PhysParams P;
    double *sc, *sx, *sy;       // residual slots (3T + 2E each)
    double *R, *sol, *jslots, *val, *S, *bs, *dinv;
    void* aoff;                 // folded off-diagonal blocks (MT of the Krylov launch)
    unsigned char *ewet, *mark;
    int *glist, *gcount;
    int* ngen;                  // general-list length of the last residual evaluation (the
                                // instance's own word: it outlives the batch slot of `norms`)
    Norms* npart;               // per-gather-block partials
    Norms* norms;               // result of the last residual evaluation
    unsigned* ncounter;
    int* singular;
    int ndir;                   // Dirichlet nodes and their step values
    const int *dir_node, *dir_mask;
    const double *dir_h, *dir_u, *dir_v;
    double* dacont;             // [3][T] elem_rhs_dacont_extra_terms of the last residual, or null
};

// Where a launch finds its instances.  SrcOne: a single instance, its descriptor a kernel
// parameter (fields read from the constant bank, the physics constants as direct operands);
// SrcPar (below): a group of instances, descriptors and block ranges as kernel parameters.
struct SrcOne {
    Inst I;
    __device__ __forceinline__ const Inst& get(int& lb, int& nb) const {
        lb = blockIdx.x;
        nb = gridDim.x;
        return I;
    }
    // block v of a persistent launch that walks nvirt blocks
    __device__ __forceinline__ const Inst& get_at(int v, int nvirt, int& lb, int& nb) const {
        lb = v;
        nb = nvirt;
        return I;
    }
};
// SrcPar: a group of up to kParInst instances whose descriptors are themselves kernel
// parameters (~22 KB; fields come from the constant cache like SrcOne's instead of a global
// table load in front of every gather); a batch is launched as ceil(n / kParInst) groups
constexpr int kParInst = 30;
struct SrcPar {
    int n;
    int boff[kParInst + 1];
    Inst I[kParInst];
    __device__ __forceinline__ const Inst& get(int& lb, int& nb) const { return get_at(blockIdx.x, 0, lb, nb); }
    // block b of the group's block ranges (a persistent launch walks b = blockIdx.x, + gridDim.x, ...)
    __device__ __forceinline__ const Inst& get_at(int b, int, int& lb, int& nb) const {
        int lo = 0, hi = n;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (boff[mid] <= b) lo = mid;
            else hi = mid;
        }
        lb = b - boff[lo];
        nb = boff[lo + 1] - boff[lo];
        return I[lo];
    }
};

// An element takes the fully wet Jacobian path when its flag is 0 and every vertex depth
// at all three levels is positive with a margin no finite-difference perturbation of h
// (|eps| <= max(1.5e-8, 1.5e-8 |h|)) can cross; every other element goes on the list.
constexpr double kWetMargin = 1e-6;

__device__ __forceinline__ void load_elem(const DevMesh& m, const State& s, int e, int rule_vel, ElemIn& in, int* n,
                                          int* df) {
    n[0] = m.en0[e];
    n[1] = m.en1[e];
    n[2] = m.en2[e];
    const unsigned first = rule_vel ? m.efirst[e] : 7u;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int k = n[i];
        in.x[i] = m.x[k];
        in.y[i] = m.y[k];
        in.z[i] = m.z[k];
        in.h[i] = s.h[k];
        in.ho[i] = s.ho[k];
        in.hoo[i] = s.hoo[k];
        // dry-node velocity zeroing is a side effect of fe_sw2_resid (:85-93): an element
        // sees the stored velocity of an old-dry node only if no earlier element touched it
        const bool zero = (in.ho[i] <= 0.) && !((first >> i) & 1u);
        in.u[i] = zero ? 0.0 : s.u[k];
        in.v[i] = zero ? 0.0 : s.v[k];
        in.uo[i] = s.uo[k];
        in.vo[i] = s.vo[k];
        in.uoo[i] = s.uoo[k];
        in.voo[i] = s.voo[k];
        df[i] = m.dflag[k];
    }
    in.djac = m.djac[e];
    in.wsx = m.wsx ? m.wsx[e] : 0.0;
    in.wsy = m.wsy ? m.wsy[e] : 0.0;
    in.gx[0] = m.gx0[e]; in.gy[0] = m.gy0[e];
    in.gx[1] = m.gx1[e]; in.gy[1] = m.gy1[e];
    in.gx[2] = m.gx2[e]; in.gy[2] = m.gy2[e];
}

// Residual contributions of every 2D element and boundary edge (fe_sw2_resid :51-191).
// slots: 3 SoA arrays (c, x, y) of length 3T + 2E.
__device__ __forceinline__ bool wet_depths(const double* h, const double* ho, const double* hoo) {
    bool wet = true;
#pragma unroll
    for (int i = 0; i < 3; i++) wet = wet && h[i] > kWetMargin && ho[i] > 0.0 && hoo[i] > 0.0;
    return wet;
}
__device__ __forceinline__ void classify_elem(int t, bool wet, unsigned char* ewet, int* glist, int* gcount) {
    ewet[t] = wet ? 1 : 0;
    if (!wet) glist[atomicAdd(gcount, 1)] = t;   // list order is free: each element is independent
}

// the same classification without a residual (sw2gpu_load called on its own)
template <class Src>
__global__ void k_classify(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const State s = I.s;
    unsigned char* ewet = I.ewet;
    int* glist = I.glist;
    int* gcount = I.gcount;
    const int t = lb * blockDim.x + threadIdx.x;
    if (t >= m.T) return;
    double h[3], ho[3], hoo[3];
    const int n[3] = {m.en0[t], m.en1[t], m.en2[t]};
#pragma unroll
    for (int i = 0; i < 3; i++) {
        h[i] = s.h[n[i]];
        ho[i] = s.ho[n[i]];
        hoo[i] = s.hoo[n[i]];
    }
    classify_elem(t, s.wd[t] == 0 && wet_depths(h, ho, hoo), ewet, glist, gcount);
}

// The element's record lives in shared memory (44 KB per CTA of 128 threads; 43 doubles per
// record, an odd stride in 8-byte words: no bank conflicts), which leaves the registers to the
// residual's arithmetic: three CTAs per SM instead of two.
static_assert(sizeof(ElemIn) % 8 == 0 && (sizeof(ElemIn) / 8) % 2 == 1, "odd record stride");
// DAC: also write the transport side output (instances whose `dacont` is set), vertex-major
// like the reference's elem_rhs_dacont_extra_terms[3][nelems2d]
template <class Src, bool DAC = false>
__global__ void __launch_bounds__(128, 3) k_resid_elem(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const State s = I.s;
    const PhysParams P = I.P;
    double* __restrict__ sc = I.sc;
    double* __restrict__ sx = I.sx;
    double* __restrict__ sy = I.sy;
    unsigned char* ewet = I.ewet;
    int* glist = I.glist;
    int* gcount = I.gcount;
    const int t = lb * blockDim.x + threadIdx.x;
    const int nslot = 3 * m.T + 2 * m.E;
    __shared__ ElemIn rec[128];
    if (t < m.T) {
        ElemIn& in = rec[threadIdx.x];
        int n[3], df[3];
        load_elem(m, s, t, 1, in, n, df);
        const int wd = s.wd[t];
        classify_elem(t, wd == 0 && wet_depths(in.h, in.ho, in.hoo), ewet, glist, gcount);
        double er[3][3], dac[3];
        sw2_elem_resid(in, in.h, in.u, in.v, wd, kPertNone, P, m.mats[m.emat[t]], df, er, DAC ? dac : nullptr);
        if (DAC && I.dacont) {
#pragma unroll
            for (int i = 0; i < 3; i++) I.dacont[(size_t)i * m.T + t] = dac[i];
        }
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const bool dry = in.ho[i] <= 0.;
            sc[3 * t + i] = er[i][0];
            sx[3 * t + i] = dry ? 0.0 : er[i][1];
            sy[3 * t + i] = dry ? 0.0 : er[i][2];
        }
    } else if (t < m.T + m.E) {
        const int j = t - m.T;
        EdgeIn in;
        const int b[2] = {m.bn0[j], m.bn1[j]};
        int df[2];
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int k = b[i];
            in.h[i] = s.h[k];
            const bool dry = s.ho[k] <= 0.;
            in.u[i] = dry ? 0.0 : s.u[k];
            in.v[i] = dry ? 0.0 : s.v[k];
            df[i] = m.dflag[k];
        }
        in.nx = m.bnx[j];
        in.ny = m.bny[j];
        in.djac = m.bdjac[j];
        in.z0 = m.z[b[0]];
        in.z1 = m.z[b[1]];
        const int kind = m.bkind[j], sid = m.bstr[j];
        in.bvx = kind == 4 ? m.str_uv[2 * sid] : 0.0;
        in.bvy = kind == 4 ? m.str_uv[2 * sid + 1] : 0.0;
        double er[2][3];
        sw2_edge_resid(in, kind, m.str_value[sid], kPertNone, P, df, er);
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const bool dry = s.ho[b[i]] <= 0.;
            const int q = 3 * m.T + 2 * j + i;
            sc[q] = er[i][0];
            sx[q] = dry ? 0.0 : er[i][1];
            sy[q] = dry ? 0.0 : er[i][2];
        }
    }
    (void)nslot;
}

// Last-block-done reduction helper for per-block partials (fixed order -> deterministic).
template <int NT>
__device__ __forceinline__ void block_reduce3(double& a, double& b, double& c, int& d) {
    __shared__ double sa[NT], sb[NT], s_c[NT];
    __shared__ int sd[NT];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    s_c[threadIdx.x] = c;
    sd[threadIdx.x] = d;
    __syncthreads();
#pragma unroll
    for (int w = NT / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sa[threadIdx.x] = fmax(sa[threadIdx.x], sa[threadIdx.x + w]);
            sb[threadIdx.x] += sb[threadIdx.x + w];
            s_c[threadIdx.x] = fmax(s_c[threadIdx.x], s_c[threadIdx.x + w]);
            sd[threadIdx.x] += sd[threadIdx.x + w];
        }
        __syncthreads();
    }
    a = sa[0];
    b = sb[0];
    c = s_c[0];
    d = sd[0];
    __syncthreads();
}

// Node gather: R = -(sum of slots in reference order) ([u, v, h] per node), the dry-node
// velocity zeroing, and get_residual_norms fused (max |R| and max |sol| over nodes with
// min(h, h_old) > 0, sum R^2 over all).  The last block to finish reduces the per-block
// partials in block order and writes *out (with the general-list length, after which the
// list counter returns to 0 for the next evaluation); `counter` returns to 0.
constexpr int kGatherThreads = 256;
template <class Src>
__global__ void __launch_bounds__(kGatherThreads) k_resid_gather(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const State s = I.s;
    const double* __restrict__ sc = I.sc;
    const double* __restrict__ sx = I.sx;
    const double* __restrict__ sy = I.sy;
    double* __restrict__ R = I.R;
    const double* __restrict__ sol = I.sol;
    Norms* partial = I.npart;
    unsigned* counter = I.ncounter;
    Norms* out = I.norms;
    int* gcount = I.gcount;
    const int n = lb * blockDim.x + threadIdx.x;
    double rmax = 0.0, l2 = 0.0, imax = 0.0;
    int nan = 0;
    if (n < m.V) {
        double ax = 0.0, ay = 0.0, ac = 0.0;
        for (int k = m.slot_ptr[n]; k < m.slot_ptr[n + 1]; k++) {
            const int q = m.slot_idx[k];
            ax += sx[q];
            ay += sy[q];
            ac += sc[q];
        }
        const double r0 = -ax, r1 = -ay, r2 = -ac;
        R[3 * n] = r0;
        R[3 * n + 1] = r1;
        R[3 * n + 2] = r2;
        const double ho = s.ho[n];
        if (ho <= 0.) {
            s.u[n] = 0.0;
            s.v[n] = 0.0;
        }
        const bool inc = fmin(s.h[n], ho) > 0;
        if (inc) {
            rmax = fmax(fmax(fabs(r0), fabs(r1)), fabs(r2));
            imax = fmax(fmax(fabs(sol[3 * n]), fabs(sol[3 * n + 1])), fabs(sol[3 * n + 2]));
        }
        l2 = r0 * r0 + r1 * r1 + r2 * r2;
        nan = (isnan(r0) || isnan(r1) || isnan(r2)) ? 1 : 0;
    }
    block_reduce3<kGatherThreads>(rmax, l2, imax, nan);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partial[lb] = Norms{rmax, l2, imax, nan, 0};
        __threadfence();
        last = (atomicAdd(counter, 1u) == (unsigned)nb - 1u);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double a = 0.0, b = 0.0, c = 0.0;
        int d = 0;
        for (int k = threadIdx.x; k < nb; k += blockDim.x) {
            a = fmax(a, __ldcg(&partial[k].rmax));
            b += __ldcg(&partial[k].l2sum);
            c = fmax(c, __ldcg(&partial[k].imax));
            d += __ldcg(&partial[k].nan);
        }
        block_reduce3<kGatherThreads>(a, b, c, d);
        if (threadIdx.x == 0) {
            const int ng = *(volatile int*)gcount;
            *out = Norms{a, b, c, d, ng};
            *I.ngen = ng;
            *gcount = 0;
            *counter = 0u;
        }
    }
}

// ---------------------------------------------------------------------------------
// FD Jacobian of the 2D elements (fe_sw2_load :85-142, perturb_sw2_head / perturb_sw2_vel).
// 32 elements x 9 perturbation columns (node b, variable u/v/h) at a time: warp w evaluates
// column w for the 32 elements (lane = element), so the pressure-term branch is warp-uniform.
// Element data are staged in shared memory once; each element's 9x9 matrix is an 81-double
// record (slot 9e + 3a + b) in global memory.
constexpr int kJacElems = 32;
constexpr int kJacThreads = kJacElems * 9;

// Lane l of a warp reads element l's record: an odd record stride in 8-byte words puts the
// 32 lanes' doubles in distinct bank pairs (an even stride such as 48 words would make every
// lane's read hit the same banks).
struct StagedElem {
    ElemIn in;
    int n[3], df[3], wd, mat;
};
static_assert(sizeof(StagedElem) % 8 == 0 && (sizeof(StagedElem) / 8) % 2 == 1, "odd record stride");
static_assert(sizeof(WetPre) % 8 == 0 && (sizeof(WetPre) / 8) % 2 == 1, "odd record stride");

__device__ __forceinline__ void stage_elem(const DevMesh& m, const State& s, int e, StagedElem& S) {
    load_elem(m, s, e, 0, S.in, S.n, S.df);
    S.wd = s.wd[e];
    S.mat = m.emat[e];
}

// One column (item = 3 b + var) of one element's 9x9 matrix into o[81] (or, when g is given,
// into the element's record g[81] in global memory, o holding only R(x + eps e_j)): R(x + eps e_j)
// and R(x - eps e_j), the central difference, and the Dirichlet zeroing of the element matrix.
// GENERAL = false: fully wet physics, with the parts the column leaves unperturbed read from
// `pre`; GENERAL = true: full wet/dry physics.
template <bool GENERAL>
__device__ __forceinline__ void jac_column(const DevMesh& m, const PhysParams& P, const StagedElem& S,
                                           const WetPre* pre, int item, double* o, double* g = nullptr) {
    const int b = item / 3, var = item % 3;  // var: 0 = u, 1 = v, 2 = h
    // only the current iterate (9 values) is private; everything else is read from the
    // staged element in shared memory
    double hc[3], uc[3], vc[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        hc[i] = S.in.h[i];
        uc[i] = S.in.u[i];
        vc[i] = S.in.v[i];
    }
    const MatParams M = m.mats[S.mat];
    // perturbed value, selected without runtime array indexing (keeps the arrays in registers)
    double cur = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (i == b) cur = (var == 0) ? uc[i] : (var == 1) ? vc[i] : hc[i];
    }
    const double eps = fd_eps(cur);
    const int pv = (var == 0) ? kPertU : (var == 1) ? kPertV : kPertH;
    // what this column leaves unperturbed
    const unsigned fix = (var == 0)   ? (kFixH | kFixV | ((7u & ~(1u << b)) << kFixNode))
                         : (var == 1) ? (kFixH | kFixU | ((7u & ~(1u << b)) << kFixNode))
                                      : (kFixU | kFixV | (7u << kFixNode));
    // Dirichlet zeroing of the element matrix (fe_assign_mom_db_dof3 / fe_assign_dacont_db_dof3):
    // D = momentum-Dirichlet nodes (old-dry or VEL/VEL_PRS string), P = continuity-Dirichlet.
    unsigned Dm = 0, Pm = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const int f = m.qflag[i];
        if (S.in.ho[i] <= 0.) Dm |= 1u << i;
        if (f & 1) Pm |= 1u << i;
        if (f & 2) Dm |= 1u << i;
        if (f & 4) { Dm |= 1u << i; Pm |= 1u << i; }
    }
    // the nine central differences of the column share one reciprocal of 2 eps (a product
    // instead of a quotient per entry: at most one rounding step away from (R+ - R-) / (2 eps),
    // far below the FD truncation error)
    const double ie2 = 1.0 / (2.0 * eps);
    // pass 0 stores R(x + eps e_j) in this thread's 9 output entries, pass 1 turns them
    // into the central difference; one residual body is instantiated, not two
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
        const double xv = pass == 0 ? cur + eps : cur - eps;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            if (i == b) {
                if (var == 0) uc[i] = xv;
                else if (var == 1) vc[i] = xv;
                else hc[i] = xv;
            }
        }
        double r[3][3];
        if (GENERAL) sw2_elem_resid(S.in, hc, uc, vc, S.wd, pv, P, M, S.df, r);
        else elem_resid_impl<true, true>(S.in, hc, uc, vc, S.wd, pv, P, M, S.df, r, pre, fix);
#pragma unroll
        for (int a = 0; a < 3; a++) {
#pragma unroll
            for (int eq = 0; eq < 3; eq++) {
                const int row = (eq == 0) ? 2 : eq - 1;  // block rows: x-mom, y-mom, continuity
                double& slot = o[(3 * a + b) * 9 + 3 * row + var];
                if (pass == 0) {
                    slot = r[a][eq];
                    continue;
                }
                double val = (slot - r[a][eq]) * ie2;
                const bool aD = (Dm >> a) & 1u, bD = (Dm >> b) & 1u, aP = (Pm >> a) & 1u, bP = (Pm >> b) & 1u;
                const bool zero = (aD && row < 2) || (bD && var < 2) || (aP && row == 2) || (bP && var == 2);
                const bool one = (a == b) && ((aD && ((var == 0 && row == 0) || (var == 1 && row == 1))) ||
                                              (aP && var == 2 && row == 2));
                if (one) val = 1.0;
                else if (zero) val = 0.0;
                if (g) g[(3 * a + b) * 9 + 3 * row + var] = val;
                else slot = val;
            }
        }
    }
}

// Fully wet elements: a persistent CTA of 9 column warps and one staging warp walks the
// launch's 32-element groups (virtual blocks v = blockIdx.x, + gridDim.x, ...).  The staging
// warp loads group i into buffer i % kJacBufs and forms its shared parts (WetPre) while the
// column warps evaluate earlier groups, so no column warp waits on element loads; buffers are
// handed over with named barriers (FULL: staged, EMPTY: read by every column warp), and a column
// warp may run ahead of the others by up to kJacBufs - 1 groups.  Elements not eligible for the wet
// physics are skipped; the general launch, which runs after this one on the same stream,
// writes their records.
constexpr int kJacWetThreads = kJacThreads + 32;
constexpr int kJacBufs = 2;
// named barriers of the wet-Jacobian CTA (0 is __syncthreads'), one FULL and one EMPTY per buffer
constexpr int kJacBarFull = 1, kJacBarEmpty = 1 + kJacBufs;
struct JacWetSmem {
    StagedElem se[kJacBufs][kJacElems];
    WetPre pre[kJacBufs][kJacElems];
    double out[kJacElems * 81];   // per column thread: its nine R(x + eps e_j) values
    int eid[kJacBufs][kJacElems];
};
constexpr size_t kJacWetSmem = sizeof(JacWetSmem);

// MINB: resident CTAs per SM the register budget is cut for (1: 168 registers, 2: 96 with
// spills); the autotuner picks per mesh, the arithmetic is the same
template <class Src, int MINB>
__global__ void __launch_bounds__(kJacWetThreads, MINB) k_jac_elem_wet(const __grid_constant__ Src src, int nvirt) {
    extern __shared__ __align__(16) unsigned char jac_smem[];
    JacWetSmem& sm = *reinterpret_cast<JacWetSmem*>(jac_smem);
    const int lane = threadIdx.x % kJacElems;
    const int item = threadIdx.x / kJacElems;
    const int stride = gridDim.x;
    if (item == 9) {
        for (int i = 0, v = blockIdx.x; v < nvirt; i++, v += stride) {
            const int j = i % kJacBufs;
            if (i >= kJacBufs) bar_sync_n(kJacBarEmpty + j, kJacWetThreads);
            int lb, nb;
            const Inst& I = src.get_at(v, nvirt, lb, nb);
            const DevMesh m = I.m;
            const int e0 = lb * kJacElems;
            int e = -1;
            if (e0 + lane < m.T && I.ewet[e0 + lane]) e = e0 + lane;
            sm.eid[j][lane] = e;
            if (e >= 0) {
                StagedElem& S = sm.se[j][lane];
                stage_elem(m, I.s, e, S);
                WetPre& p = sm.pre[j][lane];
                wet_levels(S.in, I.P, p.L);
                wet_depth(S.in, S.in.h, I.P, m.mats[S.mat], p.D);
                wet_pre_velocity(S.in, p);
            }
            __syncwarp();
            bar_arrive_n(kJacBarFull + j, kJacWetThreads);
        }
        return;
    }
    for (int i = 0, v = blockIdx.x; v < nvirt; i++, v += stride) {
        const int j = i % kJacBufs;
        bar_sync_n(kJacBarFull + j, kJacWetThreads);
        int lb, nb;
        const Inst& I = src.get_at(v, nvirt, lb, nb);
        // each column thread stores its nine finished entries itself (the nine columns of an
        // element meet in L2), so a column warp never waits for the others
        const int e = sm.eid[j][lane];
        if (e >= 0)
            jac_column<false>(I.m, I.P, sm.se[j][lane], &sm.pre[j][lane], item, sm.out + lane * 81,
                              I.jslots + (size_t)e * 81);
        __syncwarp();
        if (v + kJacBufs * stride < nvirt) bar_arrive_n(kJacBarEmpty + j, kJacWetThreads);
    }
}

// Elements of the general list (some vertex dry at some level, or a wet/dry-flagged
// element), full wet/dry physics; the list length is the one the last residual evaluation
// recorded.  One CTA per 32 listed elements.
template <class Src>
__global__ void __launch_bounds__(kJacThreads) k_jac_elem_general(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    __shared__ StagedElem se[kJacElems];
    __shared__ double out[kJacElems * 81];
    __shared__ int eid[kJacElems];
    const int count = *I.ngen;
    const int e0 = lb * kJacElems;
    const int lane = threadIdx.x % kJacElems;
    const int item = threadIdx.x / kJacElems;
    const int nel = min(kJacElems, count - e0);
    if (item == 0) {
        const int e = lane < nel ? I.glist[e0 + lane] : -1;
        eid[lane] = e;
        if (e >= 0) stage_elem(m, I.s, e, se[lane]);
    }
    __syncthreads();
    if (eid[lane] >= 0) jac_column<true>(m, I.P, se[lane], nullptr, item, out + lane * 81);
    __syncthreads();
    for (int k = threadIdx.x; k < nel * 81; k += blockDim.x) I.jslots[(size_t)eid[k / 81] * 81 + k % 81] = out[k];
}

// FD Jacobian of the boundary edges: one thread per (edge, node, variable); writes the
// four 3x3 blocks of edge j at slots 9T + 4j + 2a + b.
template <class Src>
__global__ void k_jac_edge(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const State s = I.s;
    const PhysParams P = I.P;
    double* __restrict__ jslots = I.jslots;
    const int t = lb * blockDim.x + threadIdx.x;
    if (t >= 6 * m.E) return;
    const int j = t / 6, b = (t % 6) / 3, var = t % 3;
    EdgeIn in;
    const int nd[2] = {m.bn0[j], m.bn1[j]};
    int df[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
        in.h[i] = s.h[nd[i]];
        in.u[i] = s.u[nd[i]];
        in.v[i] = s.v[nd[i]];
        df[i] = m.dflag[nd[i]];
    }
    in.nx = m.bnx[j];
    in.ny = m.bny[j];
    in.djac = m.bdjac[j];
    in.z0 = m.z[nd[0]];
    in.z1 = m.z[nd[1]];
    const int kind = m.bkind[j], sid = m.bstr[j];
    in.bvx = kind == 4 ? m.str_uv[2 * sid] : 0.0;
    in.bvy = kind == 4 ? m.str_uv[2 * sid + 1] : 0.0;
    const double value = m.str_value[sid];
    double cur = 0.0;
#pragma unroll
    for (int i = 0; i < 2; i++)
        if (i == b) cur = (var == 0) ? in.u[i] : (var == 1) ? in.v[i] : in.h[i];
    const double eps = fd_eps(cur);
    const int pv = (var == 0) ? kPertU : (var == 1) ? kPertV : kPertH;
    double rp[2][3], rm[2][3];
    EdgeIn ip = in, im = in;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        if (i != b) continue;
        if (var == 0) { ip.u[i] = cur + eps; im.u[i] = cur - eps; }
        else if (var == 1) { ip.v[i] = cur + eps; im.v[i] = cur - eps; }
        else { ip.h[i] = cur + eps; im.h[i] = cur - eps; }
    }
    sw2_edge_resid(ip, kind, value, pv, P, df, rp);
    sw2_edge_resid(im, kind, value, pv, P, df, rm);
    const double e2 = 2.0 * eps;
    unsigned Dm = 0, Pm = 0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int f = m.qflag[i];
        if (s.ho[nd[i]] <= 0.) Dm |= 1u << i;
        if (f & 1) Pm |= 1u << i;
        if (f & 2) Dm |= 1u << i;
        if (f & 4) { Dm |= 1u << i; Pm |= 1u << i; }
    }
    double* o = jslots + ((size_t)9 * m.T + 4 * j) * 9;
#pragma unroll
    for (int a = 0; a < 2; a++) {
#pragma unroll
        for (int eq = 0; eq < 3; eq++) {
            double val = (rp[a][eq] - rm[a][eq]) / e2;
            const int row = (eq == 0) ? 2 : eq - 1;
            const bool aD = (Dm >> a) & 1u, bD = (Dm >> b) & 1u, aP = (Pm >> a) & 1u, bP = (Pm >> b) & 1u;
            const bool zero = (aD && row < 2) || (bD && var < 2) || (aP && row == 2) || (bP && var == 2);
            const bool one = (a == b) && ((aD && ((var == 0 && row == 0) || (var == 1 && row == 1))) ||
                                          (aP && var == 2 && row == 2));
            if (one) val = 1.0;
            else if (zero) val = 0.0;
            o[(2 * a + b) * 9 + 3 * row + var] = val;
        }
    }
}

// BCSR values: thread k sums the nine entries of every element block contributing to BCSR
// block k, in reference order (fe_global_matrix_assemble_sw2 :166-224).  Four contributions
// (36 values) are loaded before they are added, so each warp keeps ~9 KB of loads in flight
// behind its one dependent index load; the sums go out through shared memory as contiguous
// 9-double records.
constexpr int kGatherBlocks = 128;
template <class Src>
__global__ void __launch_bounds__(kGatherBlocks) k_jac_gather(const __grid_constant__ Src src) {
    __shared__ double out[kGatherBlocks * 9];
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const double* __restrict__ jslots = I.jslots;
    double* __restrict__ val = I.val;
    const int k0 = lb * kGatherBlocks;
    const int k = k0 + threadIdx.x;
    if (k < m.nnzb) {
        double acc[9];
#pragma unroll
        for (int q = 0; q < 9; q++) acc[q] = 0.0;
        const int c0 = m.blk_ptr[k], c1 = m.blk_ptr[k + 1];
        for (int c = c0; c < c1; c += 4) {
            int sl[4];
            double v[4][9];
#pragma unroll
            for (int u = 0; u < 4; u++) sl[u] = (c + u < c1) ? __ldg(m.blk_src + c + u) : -1;
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int q = 0; q < 9; q++) v[u][q] = sl[u] >= 0 ? __ldg(jslots + (size_t)sl[u] * 9 + q) : 0.0;
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (c + u < c1)
#pragma unroll
                    for (int q = 0; q < 9; q++) acc[q] += v[u][q];
        }
#pragma unroll
        for (int q = 0; q < 9; q++) out[threadIdx.x * 9 + q] = acc[q];
    }
    __syncthreads();
    const int nk = min(kGatherBlocks, m.nnzb - k0);
    for (int i = threadIdx.x; i < nk * 9; i += kGatherBlocks) val[(size_t)k0 * 9 + i] = out[i];
}

// Tiny-diagonal fix of fe_sw2_load (:218-236), the Jacobi scale vector of spv_jacobi and the
// inverse of the scaled diagonal block (the block-Jacobi preconditioner, folded into the
// off-diagonal blocks by k_fold_offdiag) in one pass per node row
// (src/solver/spv_jacobi.c:222-285): S = 1/sqrt(max |row entry|), floored.  Also writes
// the scaled right-hand side b = S R.
template <class Src>
__global__ void k_rowscale(const __grid_constant__ Src src, int fix_only) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const State s = I.s;
    double* __restrict__ val = I.val;
    double* __restrict__ R = I.R;
    double* __restrict__ S = I.S;
    double* __restrict__ b = I.bs;
    const int n = lb * blockDim.x + threadIdx.x;
    if (n >= m.V) return;
    double* d = val + (size_t)m.dpos[n] * 9;
    if (fabs(d[0]) < kNotQuiteSmall) {
        d[0] = kNotQuiteSmall;
        if (fabs(R[3 * n]) < kNotQuiteSmall) R[3 * n] = -kNotQuiteSmall * s.u[n];
    }
    if (fabs(d[4]) < kNotQuiteSmall) {
        d[4] = kNotQuiteSmall;
        if (fabs(R[3 * n + 1]) < kNotQuiteSmall) R[3 * n + 1] = -kNotQuiteSmall * s.v[n];
    }
    if (fabs(d[8]) < kNotQuiteSmall) d[8] = kNotQuiteSmall;
    if (fix_only) return;
    double mx[3] = {0.0, 0.0, 0.0};
#pragma unroll 4
    for (int k = m.rowptr[n]; k < m.rowptr[n + 1]; k++) {
        const double* a = val + (size_t)k * 9;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) mx[r] = fmax(mx[r], fabs(a[3 * r + c]));
    }
    double sr[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const double sv = (mx[r] < kSmall) ? 1.0 / sqrt(kSmall) : 1.0 / sqrt(fabs(mx[r]));
        sr[r] = sv;
        S[3 * n + r] = sv;
        b[3 * n + r] = R[3 * n + r] * sv;
    }
    // D_n^-1 of the scaled diagonal block S_n A_nn S_n
    double a[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) a[3 * r + c] = d[3 * r + c] * (sr[r] * sr[c]);
    if (!inv3(a, I.dinv + (size_t)n * 9)) atomicExch(I.singular, 1);
}

// Block-Jacobi preconditioner folded into the matrix.  With A' = S A S (spv_jacobi scaling)
// and D_i the scaled diagonal block of row i, the Krylov operator M^-1 A' has identity
// diagonal blocks and off-diagonal blocks D_i^-1 A'_ij, so the sweeps stream only those
// (nnzb - V blocks, no inverses).  D_i^-1 comes from k_rowscale; the off-diagonal block k of
// row i goes to position k - i - (k > dpos_i) of the folded matrix,
// D_i^-1 (S_i A_ij S_j) formed in FP64 and stored as MT
template <class Src, typename MT>
__global__ void k_fold_offdiag(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const double* __restrict__ val = I.val;
    const double* __restrict__ S = I.S;
    const double* __restrict__ dinv = I.dinv;
    MT* __restrict__ aoff = (MT*)I.aoff;
    const int k = lb * blockDim.x + threadIdx.x;
    if (k >= m.nnzb) return;
    const int i = m.blk_row[k], j = m.col[k];
    const int dp = m.dpos[i];
    if (k == dp) return;
    double bq[9], d[9];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) bq[3 * r + c] = val[(size_t)k * 9 + 3 * r + c] * (S[3 * i + r] * S[3 * j + c]);
#pragma unroll
    for (int q = 0; q < 9; q++) d[q] = dinv[(size_t)i * 9 + q];
    MT* o = aoff + (size_t)(k - i - (k > dp ? 1 : 0)) * 9;
    fold_block(d, bq, o);
}

// line search halving (fe_newton.c:692-747): sol *= 0.5; state += sol (fe_sw2_inc)
template <class Src>
__global__ void k_half_inc(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    double* __restrict__ sol = I.sol;
    double* __restrict__ h = I.s.h;
    double* __restrict__ u = I.s.u;
    double* __restrict__ v = I.s.v;
    const int n = lb * blockDim.x + threadIdx.x;
    if (n >= I.m.V) return;
    const double a = sol[3 * n] * 0.5, b = sol[3 * n + 1] * 0.5, c = sol[3 * n + 2] * 0.5;
    sol[3 * n] = a;
    sol[3 * n + 1] = b;
    sol[3 * n + 2] = c;
    u[n] += a;
    v[n] += b;
    h[n] += c;
}

// fe_sw2_init (src/fe/sw2/fe_sw2_init.c:24-92), first part: current level <- old level,
// and the node marks of the wet/dry flag pass cleared
template <class Src>
__global__ void k_init_level(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const State s = I.s;
    const int n = lb * blockDim.x + threadIdx.x;
    if (n >= I.m.V) return;
    s.h[n] = s.ho[n];
    s.u[n] = s.uo[n];
    s.v[n] = s.vo[n];
    I.mark[n] = 0;
}

// fe_sw2_wdflag (src/fe/sw2/fe_sw2_wdflag.c:24-75), two passes
template <class Src>
__global__ void k_wd_mark(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const double* __restrict__ h = I.s.h;
    unsigned char* __restrict__ mark = I.mark;
    const int e = lb * blockDim.x + threadIdx.x;
    if (e >= m.T) return;
    const int a = m.en0[e], b = m.en1[e], c = m.en2[e];
    if (!(h[a] > 0.0 && h[b] > 0.0 && h[c] > 0.0)) {
        mark[a] = 1;
        mark[b] = 1;
        mark[c] = 1;
    }
}
template <class Src>
__global__ void k_wd_flag(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const DevMesh m = I.m;
    const double* __restrict__ h = I.s.h;
    const double* __restrict__ ho = I.s.ho;
    const unsigned char* __restrict__ mark = I.mark;
    int* __restrict__ wd = const_cast<int*>(I.s.wd);
    const int e = lb * blockDim.x + threadIdx.x;
    if (e >= m.T) return;
    const int a = m.en0[e], b = m.en1[e], c = m.en2[e];
    int f = (mark[a] | mark[b] | mark[c]) ? 1 : 0;
    if (h[a] < 0 && h[b] < 0 && h[c] < 0 && ho[a] < 0 && ho[b] < 0 && ho[c] < 0) f = 2;
    wd[e] = f;
}

// Dirichlet node values of fe_sw2_init (src/fe/sw2/fe_sw2_init.c:37-85)
template <class Src>
__global__ void k_dirichlet(const __grid_constant__ Src src) {
    int lb, nb;
    const Inst& I = src.get(lb, nb);
    const int t = lb * blockDim.x + threadIdx.x;
    if (t >= I.ndir) return;
    const int k = I.dir_node[t], f = I.dir_mask[t];
    if (f & 2) {
        I.s.u[k] = I.dir_u[t];
        I.s.v[k] = I.dir_v[t];
    }
    if (f & 1) I.s.h[k] = I.dir_h[t];
}

// ---------------------------------------------------------------------------------
// Wind surface stress per element (swind_elem2d_get_local_stress, src/structs/smeteor.c:241-306):
// the nodal wind values (what meteor_update puts in winds[node].stress) turned into a shear by
// the element material's flag -- 0: the value itself, 1: Wu's drag law (winds_proc_wu,
// src/meteor/winds_proc_wu.c:5-26, pow(x, 2.0) written as x * x, the same correctly rounded
// value) -- summed over the vertices in order and scaled by windatt^2 / (3 density) (`fac`,
// formed on the host with the reference's pow).
__device__ __forceinline__ void wind_wu(double g, double xs, double ys, double& sx, double& sy) {
    double wmag = sqrt(xs * xs + ys * ys + 1e-10), x = xs, y = ys;
    if (g > 10.) {
        wmag *= 0.3048;
        x *= 0.3048;
        y *= 0.3048;
    }
    const double cd = (0.8 + 0.065 * wmag) * .001;
    if (g > 10.) {
        sx = 1.225 * cd * x * wmag * 0.020885;
        sy = 1.225 * cd * y * wmag * 0.020885;
    } else {
        sx = 1.225 * cd * x * wmag;
        sy = 1.225 * cd * y * wmag;
    }
}
__global__ void k_elem_wind(const __grid_constant__ DevMesh m, double g, double density, const int* __restrict__ flag,
                            const double* __restrict__ fac, const double* __restrict__ nsx,
                            const double* __restrict__ nsy, double* __restrict__ wsx, double* __restrict__ wsy) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.T) return;
    const int mt = m.emat[e];
    const int n[3] = {m.en0[e], m.en1[e], m.en2[e]};
    double wx = 0., wy = 0.;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double sx = 0., sy = 0.;
        if (density > 0.0) {
            if (flag[mt] == 0) {
                sx = nsx[n[i]];
                sy = nsy[n[i]];
            } else {
                wind_wu(g, nsx[n[i]], nsy[n[i]], sx, sy);
            }
        }
        wx += sx;
        wy += sy;
    }
    wsx[e] = wx * fac[mt];
    wsy[e] = wy * fac[mt];
}

// Wave radiation stress of every element from the nodal radiation stresses Sxx, Sxy, Syy
// (swave_elem2d_get_local_stress, src/structs/smeteor.c:312-327, the CSTORM_WSID OFF branch):
// -sum_i (dphi_i/dx Sxx_i + dphi_i/dy Sxy_i) and -sum_i (dphi_i/dx Sxy_i + dphi_i/dy Syy_i), in
// vertex order; one thread per element, out = [x T][y T].
__global__ void k_elem_wave(const __grid_constant__ DevMesh m, const double* __restrict__ rxx,
                            const double* __restrict__ rxy, const double* __restrict__ ryy, double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.T) return;
    const int n[3] = {m.en0[e], m.en1[e], m.en2[e]};
    const double gx[3] = {m.gx0[e], m.gx1[e], m.gx2[e]}, gy[3] = {m.gy0[e], m.gy1[e], m.gy2[e]};
    double sx = 0., sy = 0.;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        sx -= (gx[i] * rxx[n[i]] + gy[i] * rxy[n[i]]);
        sy -= (gx[i] * rxy[n[i]] + gy[i] * ryy[n[i]]);
    }
    out[e] = sx;
    out[m.T + e] = sy;
}

// The element surface stress the residual reads (total_stress, fe_sw2_body_resid.c:674-694):
// wind + waves, either one 0 when it is off; arrays [x T][y T].
__global__ void k_surface_stress(int T, const double* __restrict__ wind, const double* __restrict__ wave,
                                 double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 2 * T) return;
    const double w = wind ? wind[k] : 0.0, r = wave ? wave[k] : 0.0;
    out[k] = w + r;
}

// ---------------------------------------------------------------------------------
// Adaption error indicator (ssw_2d_calculate_elem_error, src/structs/ssw_2d.c:424-500), one
// thread per element: the steady continuity residual at the vertices of the current level
// against the old one, ((h_i - ho_i) / dt + u_i dh/dx + v_i dh/dy + h_i (du/dx + dv/dy))^2,
// summed over the vertices, square root, times the area.  raw[e] keeps that value (the nodal
// average below adds it); err[e] = raw / refine_tol[material], 0.5 for wd_flag > 0 (partially
// wet elements are neither refined nor relaxed).  Every operation in the reference's order.
__global__ void k_elem_error(const __grid_constant__ DevMesh m, const double* __restrict__ h,
                             const double* __restrict__ ho, const double* __restrict__ u,
                             const double* __restrict__ v, const int* __restrict__ wd, double dt,
                             const double* __restrict__ refine_tol, double* __restrict__ raw,
                             double* __restrict__ err) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.T) return;
    const int n[3] = {m.en0[e], m.en1[e], m.en2[e]};
    const double gx[3] = {m.gx0[e], m.gx1[e], m.gx2[e]}, gy[3] = {m.gy0[e], m.gy1[e], m.gy2[e]};
    double hh[3], hp[3], uu[3], vv[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        hh[i] = h[n[i]];
        hp[i] = ho[n[i]];
        uu[i] = u[n[i]];
        vv[i] = v[n[i]];
    }
    double dhdx = 0., dhdy = 0., dudx = 0., dvdy = 0.;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        dhdx += gx[i] * hh[i];
        dhdy += gy[i] * hh[i];
        dudx += gx[i] * uu[i];
        dvdy += gy[i] * vv[i];
    }
    double c[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double t = (hh[i] - hp[i]) / dt;
        t += uu[i] * dhdx;
        t += vv[i] * dhdy;
        t += hh[i] * (dudx + dvdy);
        c[i] = t * t;
    }
    const double r = sqrt(c[0] + c[1] + c[2]) * m.djac[e];
    raw[e] = r;
    err[e] = wd[e] > 0 ? 0.5 : r / refine_tol[m.emat[e]];
}

// its nodal average (:471-496): the raw values of a node's elements summed in element order
// (the node's residual slots below 3T, which list its elements ascending) over their count
__global__ void k_node_error(const __grid_constant__ DevMesh m, const double* __restrict__ raw,
                             double* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.V) return;
    double s = 0.;
    int cnt = 0;
    for (int k = m.slot_ptr[n]; k < m.slot_ptr[n + 1]; k++) {
        const int q = m.slot_idx[k];
        if (q < 3 * m.T) {
            s += raw[q / 3];
            cnt++;
        }
    }
    out[n] = s / (double)cnt;
}

// ---------------------------------------------------------------------------------
// Mass-balance diagnostics (src/tools/tl_grid_mass.c): per-block partial sums of the terms of
// sw2_mass.cuh over a fixed grid, then one block adds the partials in block order, so a result
// is the same on every run and every GPU.
constexpr int kMassBlocks = 296;    // fixed, so the summation order is the same on every GPU
constexpr int kMassThreads = 256;

// fixed-order block sum of one value per thread (tree over the warp, then over the warps)
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    __syncthreads();
    return s;   // valid in thread 0
}

// Partial sums per block: part[b] = grid mass of depth h (density 1); with FLUX, instead
// part[2b] = source mass and part[2b+1] = boundary outflow of the step at state (h, u, v).
template <bool FLUX>
__global__ void __launch_bounds__(kMassThreads) k_mass_partial(const __grid_constant__ DevMesh m, const double* h,
                                                               const double* u, const double* v, double dt,
                                                               double density, double* part) {
    __shared__ double red[kMassThreads / 32];
    const int stride = kMassBlocks * kMassThreads;
    double a = 0.0, b = 0.0;
    for (int e = blockIdx.x * kMassThreads + threadIdx.x; e < m.T; e += stride) {
        const int n[3] = {m.en0[e], m.en1[e], m.en2[e]};
        double x[3], y[3], d[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            x[i] = m.x[n[i]];
            y[i] = m.y[n[i]];
            d[i] = h[n[i]];
        }
        if (!FLUX) {
            a += elem_mass(x, y, d, m.djac[e]);
        } else {
            const MatParams& M = m.mats[m.emat[e]];
            if (M.has_source) a += elem_source_mass(x, y, d, m.djac[e], M.water_src, dt, density);
        }
    }
    if (FLUX && m.E > 0) {
        const double djac0 = m.bdjac[0];
        for (int j = blockIdx.x * kMassThreads + threadIdx.x; j < m.E; j += stride) {
            const int n0 = m.bn0[j], n1 = m.bn1[j];
            const double nx = m.bnx[j], ny = m.bny[j];
            const double vn0 = u[n0] * nx + v[n0] * ny, vn1 = u[n1] * nx + v[n1] * ny;
            b += edge_outflow_term(djac0, density, dt, h[n0], h[n1], vn0, vn1);
        }
    }
    a = block_sum(a, red);
    if (FLUX) b = block_sum(b, red);
    if (threadIdx.x == 0) {
        if (FLUX) {
            part[2 * blockIdx.x] = a;
            part[2 * blockIdx.x + 1] = b;
        } else {
            part[blockIdx.x] = a;
        }
    }
}

// The partials in block order: out[0] = density x grid mass, or (FLUX) out[0] = sources minus
// boundary outflow of the step, the term tl_find_grid_mass_error_elem2d accumulates.
template <bool FLUX>
__global__ void __launch_bounds__(kMassThreads) k_mass_final(const double* part, double density, double* out) {
    __shared__ double red[kMassThreads / 32];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < kMassBlocks; i += kMassThreads) {
        if (FLUX) {
            a += part[2 * i];
            b += part[2 * i + 1];
        } else {
            a += part[i];
        }
    }
    a = block_sum(a, red);
    if (FLUX) b = block_sum(b, red);
    if (threadIdx.x == 0) out[0] = FLUX ? a - b : a * density;
}

}  // namespace sw2
