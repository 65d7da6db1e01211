// sw2gpu.cu -- host side of the B200 SW2 Newton step and the C ABI of include/sw2gpu.h.
//
// The host owns control flow only: mesh preprocessing at create time (geometry,
// BCSR pattern, reference-order contribution lists), the Newton loop of fe_newton
// (src/fe/fe_newton.c:214-912) with one 40-byte device->host read of the residual
// norms per residual evaluation, and the dt-retry contract of fe_main.  All
// element, node and Krylov work runs in the kernels of sw2_kernels.cuh /
// sw2_krylov.cuh on the context's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <queue>
#include <thread>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/sw2gpu.h"
#include "sw2_band.cuh"
#include "sw2_dilu.cuh"
#include "sw2_tables.h"
#include "sw2_kernels.cuh"
#include "sw2_krylov.cuh"
#include "sw2_series.h"
#include "sw2_shares.h"
#include "trn_kernels.cuh"
#include "newton_ctl.cuh"

using namespace sw2;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(e_ == cudaErrorMemoryAllocation ? SW2GPU_E_NOMEM : SW2GPU_E_CUDA,        \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

constexpr double kPi = 3.141592653589793238462643383279502884197169399375105820974944592308;
constexpr double kEarthRotat = 7.2722E-5;
constexpr double kUnsetFlt = -9999999.9;

// device bytes allocated by this thread go to *g_alloc_bytes while it is set (sw2gpu_create
// sets it to the context's total)
thread_local size_t* g_alloc_bytes = nullptr;

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    int alloc(size_t count) {
        n = count;
        if (count == 0) count = 1;
        // 16 spare bytes: bulk copies of a 16-byte-rounded range may reach past the last element
        cudaError_t e = cudaMalloc(&p, count * sizeof(T) + 16);
        if (e == cudaSuccess && g_alloc_bytes) *g_alloc_bytes += count * sizeof(T) + 16;
        return e == cudaSuccess ? 0 : -1;
    }
    ~DBuf() { if (p) cudaFree(p); }
};

}  // namespace

// lets other translation units of this library report through sw2gpu_last_error()
__attribute__((visibility("hidden"))) void sw2gpu_internal_set_error(const char* msg) { g_err = msg; }

struct Runner;

struct sw2gpu_ctx {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int V = 0, T = 0, E = 0, S = 0, M = 0, NS = 0, nnzb = 0;
    sw2gpu_params p{};
    double dt = 0.0;
    // host tables
    std::vector<int> str_bc, str_isigma, str_ivx, str_ivy, str_iu0;
    std::vector<MatParams> mats_h;
    std::vector<int> dir_node, dir_mask, dir_str;
    MeshTables tab;                    // pattern and gather lists (sw2_tables.h)
    std::vector<int> tri_h, edg_h;     // connectivity the tables were made from (sw2gpu_remesh)
    std::vector<int> node_str_h, edg_str_h;   // node and edge strings (transport boundary conditions)
    std::vector<int>& rowptr_h = tab.rp;
    std::vector<int>& col_h = tab.col;
    // device mesh
    DBuf<double> x, y, z, djac, gx0, gy0, gx1, gy1, gx2, gy2, bdjac, bnx, bny;
    DBuf<int> en0, en1, en2, emat, bn0, bn1, bkind, bstr;
    DBuf<unsigned char> efirst, dflag, mark;
    DBuf<MatParams> mats;
    DBuf<double> str_value, str_uv;
    DBuf<double> mass_part;     // mass-balance partials (2 per block) and three results
    // mass balance of every accepted step, reduced inside the step (sw2gpu_set_mass_tracking)
    bool mass_on = false;
    double mass_density = 0.0;
    double* mass_h = nullptr;   // pinned: grid mass and flux of the last accepted step
    bool mass_valid = false;
    double step_mass = 0.0, step_flux = 0.0;
    DBuf<double> dacont;        // [3][T] transport side output, allocated when first enabled
    DBuf<double> errind;        // adaption error indicator: raw [T], scaled [T], nodal [V], tolerances [M]
    // exact banded LU solve (SW2GPU_PREC_BAND): reverse Cuthill-McKee position of every node, the
    // band of the scaled system [3V][2 bw + 1] and its right-hand side / solution [3V]
    bool band = false;
    int band_bw = 0;
    DBuf<int> band_perm;
    DBuf<double> band_mem, band_y;
    // block D-ILU solve (SW2GPU_PREC_DILU): the coloured row order (colours padded to 32-row
    // tiles), the off-diagonal blocks in an ELL layout per colour, the operator and the solve's
    // own vectors
    bool dilu = false;
    int dl_ncol = 0, dl_rows = 0, dl_nlo = 0, dl_nup = 0, dl_cta = 0;
    int dl_cstart[kMaxColours + 1] = {}, dl_cend[kMaxColours + 1] = {};
    int dl_lbase[kMaxColours + 1] = {}, dl_ubase[kMaxColours + 1] = {}, dl_lkn[kMaxColours + 1] = {},
        dl_ukn[kMaxColours + 1] = {};
    DBuf<int> dl_lcol, dl_ucol, dl_lsrc, dl_usrc, dl_tslot, dl_old;
    DBuf<double> dl_blk64, dl_Dti, dl_Dd, dl_part;
    DBuf<float> dl_blk32;
    DBuf<double> dl_vec[kDiluVectors];
    DBuf<double> wind;          // wind: element stress x [T], y [T], nodal values x [V], y [V], factors [M]
    DBuf<int> wind_flag;        // [M] wind stress flag per material
    bool wind_on = false;
    DBuf<double> wave;          // waves: element stress x [T], y [T], nodal Sxx, Sxy, Syy [3][V]
    bool wave_on = false;
    DBuf<double> stress;        // element surface stress, wind + waves: x [T], y [T]
    bool dacont_on = false;
    // constituent transport (sw2gpu_set_transport): per constituent three levels rotated by index
    // like the flow's, its string table and MP DF coefficients; work arrays shared by all
    int ntrn = 0;
    std::vector<double> trn_refc, trn_dm_h;     // [ntrn], [ntrn * M]
    std::vector<int> trn_bc_h, trn_ser_h;       // [ntrn * S]
    std::vector<std::array<int, 3>> trn_lv;     // level rotation per constituent
    DBuf<double> tconc;                         // [ntrn][3][V]
    DBuf<int> tbc, tnode_str;                   // [ntrn * S], [V]
    DBuf<double> tdm, tsval;                    // [ntrn * M], [S]
    DBuf<unsigned char> tmask;                  // [V] bc_mask
    DBuf<double> trslot, tjslot, tR, tsol, taoff, tdinv, tkpart;
    DBuf<double> tkv[kTrnKVectors];
    DBuf<Norms> tnpart, tnorms;
    DBuf<unsigned> tncount;
    DBuf<KrylovCtl> tctl;
    Norms* tnorms_h = nullptr;                  // pinned: residual norms of the last evaluation
    KrylovCtl* tctl_h = nullptr;                // pinned: the last transport Krylov solve
    double* tsval_h = nullptr;                  // pinned [S]
    int trn_kgrid = 0;                          // CTAs of the transport Krylov solve
    double* tlevel(int k, int l) { return tconc.p + ((size_t)3 * k + trn_lv[k][l]) * V; }
    bool has_ovh = false;       // some edge string is NB OVH (its velocity series go up every step)
    DBuf<int> slot_ptr, slot_idx, blk_ptr, blk_src, rowptr, col, blk_row, dpos;
    DBuf<int> dir_node_d, dir_mask_d;
    DBuf<double> dir_h, dir_u, dir_v;
    // state: three levels, rotated by index
    DBuf<double> hs[3], us[3], vs[3];
    int lv[3] = {0, 1, 2};
    DBuf<int> wd;
    DBuf<unsigned char> ewet;    // element takes the fully wet Jacobian path
    DBuf<int> glist, gcount;     // elements on the general (wet/dry) Jacobian path
    DBuf<int> ngen;              // its length at the last residual evaluation (device copy)
    int ngeneral = 0;            // its length at the last residual evaluation
    // work
    DBuf<double> sc, sx, sy, R, sol, jslots, val, S_, bs;
    // Krylov operator: block-Jacobi inverse folded into the off-diagonal blocks
    // (orowptr / ocol: the BCSR pattern without its diagonal); FP64 or FP32 storage
    std::vector<int> orowptr_h;
    DBuf<int> orowptr, ocol;
    DBuf<double> aoff64, dinv64;
    DBuf<float> aoff32;
    DBuf<double> kv64[kKrylovVectors];
    DBuf<double> part;
    DBuf<Norms> npart;
    DBuf<unsigned> ncounter;
    int krylov_grid = 0;            // virtual CTAs of the Krylov solve (its partial structure)
    // Krylov iterations expected of the next solve, and those seen at each Newton iteration
    // of the last step (the first Newton iteration of a step needs the tightest solve) and of
    // the step before (its_snap holds its_at as the current step began, its_prev as the last one
    // began): they weight the instance's CTA share in a batch
    int pred_its = 20;
    size_t bytes = 0;               // device memory of the context
    int its_at[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int its_snap[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int its_prev[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    unsigned a_cap = 0, c_cap = 0;  // largest tile block / column-index ranges (staged sweeps)
    // autotuned launch variants (sw2gpu_autotune): they change speed, never results
    int tune_jac_minb = 2;          // wet-Jacobian CTAs per SM the register budget is cut for
    int tune_stages = 3;            // Krylov tile-ring depth (0: sweeps from global memory)
    // polls of a Krylov grid-barrier / tile-copy wait before it gives up (0: the library's
    // defaults); sw2gpu_set_wait_limits
    long long wait_barrier = 0, wait_copy = 0;
    DevMesh dm{};
    std::unique_ptr<Runner> self;   // runs this instance alone
    // CUDA graphs of a step's launch sequences (sw2gpu_set_graphs), one set per arrangement of
    // the three rotating state levels (index lv[0]); recaptured when dt or a variant changes
    struct StepGraph {
        cudaGraphExec_t start = nullptr, newton = nullptr;
        int kernels_start = 0, kernels_newton = 0;
        double dt = -1.0;
        int jac_minb = -1, stages = -1;
        // the whole step as one graph, its loops conditional nodes (graph mode 2): kernels of the
        // step start, of one Newton iteration, of one line-search halving, of the final test, of
        // the failure reset and of the tail (mass tracking)
        cudaGraphExec_t loop = nullptr;
        int k_start = 0, k_body = 0, k_ls = 0, k_final = 0, k_reset = 0, k_tail = 0;
        bool loop_mass = false;
    };
    bool use_graphs = false;
    bool loop_graphs = false;       // graph mode 2: the Newton loop's control on the device
    DBuf<NewtonCtl> nctl;           // its state
    NewtonCtl* nctl_h = nullptr;    // pinned: the state after the step
    StepGraph graphs[3];
    // pinned staging of the per-step tables; the event marks the end of their last upload
    double* stage_h = nullptr;
    cudaEvent_t stage_ev = nullptr;
    bool stage_pending = false;
    void drop_graphs() {
        for (auto& g : graphs) {
            if (g.start) cudaGraphExecDestroy(g.start);
            if (g.newton) cudaGraphExecDestroy(g.newton);
            if (g.loop) cudaGraphExecDestroy(g.loop);
            g = StepGraph();
        }
    }

    ~sw2gpu_ctx();
    double* H(int l) { return hs[lv[l]].p; }
    double* U(int l) { return us[lv[l]].p; }
    double* Vv(int l) { return vs[lv[l]].p; }
    State state() {
        State s;
        s.h = H(0); s.u = U(0); s.v = Vv(0);
        s.ho = H(1); s.uo = U(1); s.vo = Vv(1);
        s.hoo = H(2); s.uoo = U(2); s.voo = Vv(2);
        s.wd = wd.p;
        return s;
    }
    PhysParams phys() const {
        PhysParams P;
        P.g = p.gravity;
        P.dll = p.drying_lower_limit;
        P.dul = p.drying_upper_limit;
        P.alpha = p.tau_temporal;
        P.tau_pg = p.tau_pg;
        P.dt = dt;
        return P;
    }
};

namespace {

enum PhaseKind { kPhJac = 0, kPhKrylov = 1, kPhResid = 2 };

#ifndef SW2_MAX_STAGED_SMEM
#define SW2_MAX_STAGED_SMEM (96 * 1024)   // dynamic shared memory allowed for the tile ring
#endif
constexpr size_t kMaxStagedSmem = SW2_MAX_STAGED_SMEM;

// bytes per stage of the staged Krylov sweeps: the largest 16-byte-rounded block range and
// column-index range of any tile of kTileRows rows, for matrix elements of esz bytes
void stage_caps(const std::vector<int>& rp, int V, size_t esz, unsigned& a_cap, unsigned& c_cap) {
    size_t am = 16, cm = 16;
    for (int r0 = 0; r0 < V; r0 += kTileRows) {
        const size_t k0 = (size_t)rp[r0], k1 = (size_t)rp[std::min(r0 + kTileRows, V)];
        am = std::max(am, ((k1 * 9 * esz + 15) & ~size_t(15)) - ((k0 * 9 * esz) & ~size_t(15)));
        cm = std::max(cm, ((k1 * 4 + 15) & ~size_t(15)) - ((k0 * 4) & ~size_t(15)));
    }
    a_cap = (unsigned)am;
    c_cap = (unsigned)cm;
}

// largest band the direct solve accepts (bytes of the band of the scaled system)
constexpr size_t kBandMaxBytes = size_t(2) << 30;

// Krylov kernel with a tile ring of `stages` stages (0: sweeps read global memory)
template <typename MT, class KS>
void* krylov_kernel(int stages) {
    switch (stages) {
        case 2: return (void*)k_bicgstab<MT, double, 2, KS>;
        case 3: return (void*)k_bicgstab<MT, double, 3, KS>;
        default: return (void*)k_bicgstab<MT, double, 0, KS>;
    }
}

}  // namespace

// A batch of instances stepped together: device tables of the instances, per-instance
// results (norms, Krylov control words), the Krylov launch configuration and the phase
// timers.  Every kernel launch covers a subset of the instances through a LaunchMap.
struct Runner {
    cudaStream_t stream = nullptr;
    bool capturing = false;       // launches are being captured into a CUDA graph
    DBuf<double> eta_dev;         // Krylov tolerance of every instance in a graph-replayed Newton iteration
    double* eta_h = nullptr;      // its pinned host copy
    // CUDA graphs of a batch step (sw2gpu_batch_set_graphs): the step start and a Newton
    // iteration of all instances, per arrangement of the instances' time levels, dt and launch
    // variant (they are baked into the captured launches); a few are kept
    struct BatchGraph {
        std::vector<int> lv;
        std::vector<double> dt;
        int jac_minb = -1, stages = -1;
        cudaGraphExec_t start = nullptr, newton = nullptr;
        int kernels_start = 0, kernels_newton = 0;
    };
    bool use_graphs = false;
    std::vector<BatchGraph> bgraphs;
    void drop_batch_graphs() {
        for (auto& g : bgraphs) {
            if (g.start) cudaGraphExecDestroy(g.start);
            if (g.newton) cudaGraphExecDestroy(g.newton);
        }
        bgraphs.clear();
    }
    std::vector<sw2gpu_ctx*> ctx;
    bool mixed = false;
    DBuf<KrylovInst> ktab;
    std::vector<Inst> tab_h;       // descriptors (kernel parameters of every launch)
    KrylovInst* ktab_h = nullptr;  // pinned; uploaded to ktab for batch Krylov launches
    DBuf<DiluArgs> dtab;           // D-ILU descriptors (setup kernels and batch solves)
    DiluArgs* dtab_h = nullptr;    // pinned
    bool any_dilu = false;
    cudaEvent_t tab_ev = nullptr;  // end of the last ktab upload
    bool tab_pending = false;
    DBuf<Norms> norms;
    DBuf<KrylovCtl> ctl;
    DBuf<int> singular;
    Norms* norms_h = nullptr;     // pinned mirrors, one entry per instance
    KrylovCtl* ctl_h = nullptr;
    int stages = 0;               // Krylov tile-ring depth in use (0: sweeps from global memory)
    int jac_minb = 2;             // wet-Jacobian variant in use (register budget for 1 or 2 CTAs per SM)
    int jac_ctas[2] = {0, 0};     // persistent wet-Jacobian grid per variant (co-resident CTAs)
    bool jac_ready = false;       // jac_ctas set (kernel attributes applied)
    unsigned c_off = 0, r_off = 0, v_off = 0, stage_bytes = 0;
    size_t smem = 0;
    int capacity = 0;             // co-resident Krylov CTAs
    // Krylov rebalancing of host-driven batch launches: up to rb_rounds launches per solve; in
    // every launch but the last, once rb_frac of its CTAs have finished their instances, the
    // instances still running pause and the next launch shares all CTAs among them
    int rb_rounds = 4;
    double rb_frac = 0.5;
    DBuf<unsigned> kdone;         // finished-CTA counter of each round
    static constexpr int kMaxRounds = 8;
    int cap = 0;                  // instances the tables hold
    int launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    static constexpr int kMaxPhases = 512;
    std::vector<cudaEvent_t> pev;
    std::vector<int> pkind;
    int nphase = 0;
    ~Runner() {
        if (tab_ev) {
            cudaEventSynchronize(tab_ev);
            cudaEventDestroy(tab_ev);
        }
        drop_batch_graphs();
        if (ktab_h) cudaFreeHost(ktab_h);
        if (dtab_h) cudaFreeHost(dtab_h);
        if (eta_h) cudaFreeHost(eta_h);
        for (auto e : pev) cudaEventDestroy(e);
        if (norms_h) cudaFreeHost(norms_h);
        if (ctl_h) cudaFreeHost(ctl_h);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
};

sw2gpu_ctx::~sw2gpu_ctx() {
    drop_graphs();
    if (stage_ev) {
        cudaEventSynchronize(stage_ev);
        cudaEventDestroy(stage_ev);
    }
    if (stage_h) cudaFreeHost(stage_h);
    if (mass_h) cudaFreeHost(mass_h);
    if (tnorms_h) cudaFreeHost(tnorms_h);
    if (nctl_h) cudaFreeHost(nctl_h);
    if (tctl_h) cudaFreeHost(tctl_h);
    if (tsval_h) cudaFreeHost(tsval_h);
    self.reset();
    if (own_stream && stream) cudaStreamDestroy(stream);
}

struct sw2gpu_batch {
    std::unique_ptr<Runner> run;
    bool own_stream = false;
};

namespace {

// phase timer: brackets launches with an event pair when the pool has room
struct Phase {
    Runner* r;
    int slot;
    Phase(Runner* rr, int kind) : r(rr), slot(-1) {
        if (!r->capturing && r->nphase < Runner::kMaxPhases && !r->pev.empty()) {
            slot = r->nphase++;
            r->pkind[slot] = kind;
            cudaEventRecord(r->pev[2 * slot], r->stream);
        }
    }
    ~Phase() {
        if (slot >= 0) cudaEventRecord(r->pev[2 * slot + 1], r->stream);
    }
};

template <typename T>
int up(DBuf<T>& b, const std::vector<T>& v, cudaStream_t st) {
    if (b.alloc(v.size())) return fail(SW2GPU_E_NOMEM, "cudaMalloc of %zu bytes failed", v.size() * sizeof(T));
    if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return 0;
}
template <typename T>
int zalloc(DBuf<T>& b, size_t n, cudaStream_t st) {
    if (b.alloc(n)) return fail(SW2GPU_E_NOMEM, "cudaMalloc of %zu bytes failed", n * sizeof(T));
    CK(cudaMemsetAsync(b.p, 0, std::max<size_t>(n, 1) * sizeof(T), st));
    return 0;
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

// per-step tables: string values (edge series), material water sources, Dirichlet values
// Staging layout (doubles): S string values | M MatParams | 3 x ndir Dirichlet values |
// 2 x S NB OVH velocities.
size_t stage_doubles(const sw2gpu_ctx* c) {
    return (size_t)std::max(c->S, 1) + (sizeof(MatParams) * std::max(c->M, 1) + 7) / 8 + 3 * c->dir_node.size() +
           2 * (size_t)std::max(c->S, 1) + 1;
}

// per-step tables through the context's pinned staging buffer (no host sync; the buffer is
// rewritten only after its last upload completed)
int upload_step_tables(sw2gpu_ctx* c, const double* series, cudaStream_t st) {
    if (c->stage_pending) {
        CK(cudaEventSynchronize(c->stage_ev));
        c->stage_pending = false;
    }
    double* sv = c->stage_h;
    MatParams* mp = reinterpret_cast<MatParams*>(sv + std::max(c->S, 1));
    double* dv = sv + std::max(c->S, 1) + (sizeof(MatParams) * std::max(c->M, 1) + 7) / 8;
    for (int s = 0; s < c->S; s++) {
        int k = c->str_isigma[s];
        sv[s] = (k >= 0 && k < c->NS && series) ? series[k] : 0.0;
    }
    if (c->S) CK(cudaMemcpyAsync(c->str_value.p, sv, sizeof(double) * c->S, cudaMemcpyHostToDevice, st));
    bool any_src = false;
    for (int m = 0; m < c->M; m++) {
        if (c->mats_h[m].has_source) {
            int k = c->str_isigma[m];
            c->mats_h[m].water_src = (k >= 0 && k < c->NS && series) ? series[k] : 0.0;
            any_src = true;
        }
    }
    if (any_src) {
        memcpy(mp, c->mats_h.data(), sizeof(MatParams) * c->M);
        CK(cudaMemcpyAsync(c->mats.p, mp, sizeof(MatParams) * c->M, cudaMemcpyHostToDevice, st));
    }
    const int nd = (int)c->dir_node.size();
    if (nd) {
        double *h = dv, *u = dv + nd, *v = dv + 2 * nd;
        for (int i = 0; i < nd; i++) {
            int s = c->dir_str[i];
            auto get = [&](int k) { return (k >= 0 && k < c->NS && series) ? series[k] : 0.0; };
            u[i] = get(c->str_ivx[s]);
            v[i] = get(c->str_ivy[s]);
            h[i] = get(c->str_iu0[s]);
        }
        CK(cudaMemcpyAsync(c->dir_h.p, h, sizeof(double) * nd, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(c->dir_u.p, u, sizeof(double) * nd, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(c->dir_v.p, v, sizeof(double) * nd, cudaMemcpyHostToDevice, st));
    }
    if (c->has_ovh) {
        double* uv = dv + 3 * nd;
        auto get = [&](int k) { return (k >= 0 && k < c->NS && series) ? series[k] : 0.0; };
        for (int s = 0; s < c->S; s++) {
            const bool ovh = c->str_bc[s] == SW2GPU_BCT_OVH_NEU;
            uv[2 * s] = ovh ? get(c->str_ivx[s]) : 0.0;
            uv[2 * s + 1] = ovh ? get(c->str_ivy[s]) : 0.0;
        }
        CK(cudaMemcpyAsync(c->str_uv.p, uv, sizeof(double) * 2 * c->S, cudaMemcpyHostToDevice, st));
    }
    CK(cudaEventRecord(c->stage_ev, st));
    c->stage_pending = true;
    return 0;
}

// ---- runner ------------------------------------------------------------------------

// per-instance device arrays and pinned mirrors for up to `cap` instances, timing events
int runner_alloc(Runner& R, cudaStream_t stream, bool mixed, int cap) {
    R.stream = stream;
    R.mixed = mixed;
    R.cap = cap;
    if (R.ktab.alloc(cap) || R.dtab.alloc(cap) || R.norms.alloc(cap) || R.ctl.alloc(cap) || R.singular.alloc(cap) ||
        R.kdone.alloc(Runner::kMaxRounds))
        return fail(SW2GPU_E_NOMEM, "batch tables");
    CK(cudaMemsetAsync(R.norms.p, 0, sizeof(Norms) * cap, stream));
    CK(cudaMemsetAsync(R.ctl.p, 0, sizeof(KrylovCtl) * cap, stream));
    CK(cudaMallocHost(&R.norms_h, sizeof(Norms) * cap));
    CK(cudaMallocHost(&R.eta_h, sizeof(double) * cap));
    if (R.eta_dev.alloc(cap)) return fail(SW2GPU_E_NOMEM, "tolerance words");
    CK(cudaMallocHost(&R.ctl_h, sizeof(KrylovCtl) * cap));
    R.tab_h.resize(cap);
    CK(cudaMallocHost(&R.ktab_h, sizeof(KrylovInst) * cap));
    CK(cudaMallocHost(&R.dtab_h, sizeof(DiluArgs) * cap));
    CK(cudaEventCreateWithFlags(&R.tab_ev, cudaEventDisableTiming));
    CK(cudaEventCreate(&R.ev0));
    CK(cudaEventCreate(&R.ev1));
    R.pev.resize(2 * Runner::kMaxPhases);
    R.pkind.resize(Runner::kMaxPhases);
    for (auto& e : R.pev) CK(cudaEventCreate(&e));
    return 0;
}

// the instances of the runner (at most its capacity, one precision) and the launch variants
// for them: those tuned for the instance with the most blocks, the stage layout for the
// largest tile of any instance, the co-resident Krylov CTAs
int runner_set(Runner& R, const std::vector<sw2gpu_ctx*>& ctx) {
    if ((int)ctx.size() > R.cap) return fail(SW2GPU_E_ARG, "batch of %zu instances (at most %d)", ctx.size(), R.cap);
    for (auto* c : ctx)
        if ((c->p.precision == SW2GPU_MIXED) != R.mixed) return fail(SW2GPU_E_ARG, "a batch has one precision");
    R.ctx = ctx;
    unsigned a_cap = 16, c_cap = 16;
    const sw2gpu_ctx* big = nullptr;
    for (auto* c : ctx) {
        a_cap = std::max(a_cap, c->a_cap);
        c_cap = std::max(c_cap, c->c_cap);
        if (!big || c->nnzb > big->nnzb) big = c;
    }
    int want = big ? big->tune_stages : 3;
    R.jac_minb = big ? big->tune_jac_minb : 2;
    auto fitting_variant = [&R] {   // a wet-Jacobian variant that does not fit yields to the other
        if (R.jac_ready && !R.jac_ctas[R.jac_minb - 1] && R.jac_ctas[2 - R.jac_minb]) R.jac_minb = 3 - R.jac_minb;
    };
    fitting_variant();
    const unsigned c_off = a_cap, r_off = c_off + c_cap;
    const unsigned v_off = r_off + ((unsigned)(kTileRows + 1) * 4u + 15u) / 16u * 16u;
    const unsigned stage = (v_off + (unsigned)kMaxEpilogue * tile_vec_bytes<double>() + 127u) & ~127u;
    if (want > 0 && (size_t)want * stage > kMaxStagedSmem) want = (size_t)2 * stage <= kMaxStagedSmem ? 2 : 0;
    if (R.capacity > 0 && want == R.stages &&
        (!want || (a_cap <= R.c_off && c_cap <= R.r_off - R.c_off)))
        return 0;   // the current layout still holds every tile
    R.stages = want;
    R.c_off = R.r_off = R.v_off = R.stage_bytes = 0;
    if (R.stages) {
        R.c_off = c_off;
        R.r_off = r_off;
        R.v_off = v_off;
        R.stage_bytes = stage;
    }
    R.smem = (size_t)R.stages * R.stage_bytes;
    int dev = 0, sms = 0, per_sm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // the dynamic shared-memory cap is an attribute of the kernel, shared by every runner:
    // set to the largest tile ring any runner may use
    void* kone = R.mixed ? krylov_kernel<float, KrylovOne>(R.stages) : krylov_kernel<double, KrylovOne>(R.stages);
    void* ktab = R.mixed ? krylov_kernel<float, KrylovTab>(R.stages) : krylov_kernel<double, KrylovTab>(R.stages);
    if (R.stages) {
        CK(cudaFuncSetAttribute(kone, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxStagedSmem));
        CK(cudaFuncSetAttribute(ktab, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxStagedSmem));
    }
    int per_sm_tab = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kone, kKrylovThreads, R.smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_tab, ktab, kKrylovThreads, R.smem));
    per_sm = std::min(per_sm, per_sm_tab);
    R.capacity = sms * std::max(1, std::min(per_sm, 4));
    if (!R.jac_ready) {
        R.jac_ready = true;
        // wet-Jacobian kernels: double-buffered records above the 48 KB static limit, and a
        // persistent grid of the CTAs that fit at once
        const void* wet[2][2] = {{(const void*)k_jac_elem_wet<SrcOne, 1>, (const void*)k_jac_elem_wet<SrcPar, 1>},
                                 {(const void*)k_jac_elem_wet<SrcOne, 2>, (const void*)k_jac_elem_wet<SrcPar, 2>}};
        for (int v = 0; v < 2; v++) {
            int fit = 1 << 30;
            for (int k = 0; k < 2; k++) {
                int n = 0;
                CK(cudaFuncSetAttribute(wet[v][k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJacWetSmem));
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wet[v][k], kJacWetThreads, kJacWetSmem));
                fit = std::min(fit, n);
            }
            R.jac_ctas[v] = sms * fit;   // 0: the variant does not fit on this device
        }
    }
    fitting_variant();
    return 0;
}

int runner_init(Runner& R, const std::vector<sw2gpu_ctx*>& ctx, cudaStream_t stream) {
    if (ctx.empty() || (int)ctx.size() > kMaxBatch) return fail(SW2GPU_E_ARG, "batch of %zu instances (1..%d)", ctx.size(), kMaxBatch);
    int rc = runner_alloc(R, stream, ctx[0]->p.precision == SW2GPU_MIXED, (int)ctx.size());
    return rc ? rc : runner_set(R, ctx);
}

// device tables from the instances' current buffers and state levels
// the D-ILU descriptor of instance k (its state pointers follow the rotating levels)
void dilu_args(Runner& R, int k, int apply_inc) {
    sw2gpu_ctx* c = R.ctx[k];
    DiluArgs& D = R.dtab_h[k];
    D.V = c->V;
    D.N = c->dl_rows;
    D.ncol = c->dl_ncol;
    D.nlo = c->dl_nlo;
    D.nup = c->dl_nup;
    D.ncta = c->dl_cta;
    for (int i = 0; i <= kMaxColours; i++) {
        D.cstart[i] = c->dl_cstart[i];
        D.cend[i] = c->dl_cend[i];
        D.lbase[i] = c->dl_lbase[i];
        D.ubase[i] = c->dl_ubase[i];
        D.lkn[i] = c->dl_lkn[i];
        D.ukn[i] = c->dl_ukn[i];
    }
    D.lcol = c->dl_lcol.p;
    D.ucol = c->dl_ucol.p;
    D.lsrc = c->dl_lsrc.p;
    D.usrc = c->dl_usrc.p;
    D.tslot = c->dl_tslot.p;
    D.old = c->dl_old.p;
    D.blk = R.mixed ? (void*)c->dl_blk32.p : (void*)c->dl_blk64.p;
    D.Dti = c->dl_Dti.p;
    D.Dd = c->dl_Dd.p;
    D.blk_row = c->blk_row.p;
    D.bcol = c->col.p;
    D.dpos = c->dpos.p;
    D.val = c->val.p;
    D.S = c->S_.p;
    D.bs = c->bs.p;
    D.singular = R.singular.p + k;
    D.atol = c->p.lin_atol;
    D.maxit = c->p.max_lin_it;
    D.h = c->H(0);
    D.u = c->U(0);
    D.v = c->Vv(0);
    D.sol = c->sol.p;
    D.apply_inc = apply_inc;
    D.part = c->dl_part.p;
    D.ctl = R.ctl.p + k;
    D.spin_limit = c->wait_barrier;
    for (int i = 0; i < kDiluVectors; i++) D.vec[i] = c->dl_vec[i].p;
}

int runner_tables(Runner& R, int apply_inc) {
    const int K = (int)R.ctx.size();
    if (R.tab_pending) {   // the pinned Krylov table is rewritten only after its last upload
        CK(cudaEventSynchronize(R.tab_ev));
        R.tab_pending = false;
    }
    for (int k = 0; k < K; k++) {
        sw2gpu_ctx* c = R.ctx[k];
        Inst& I = R.tab_h[k];
        I.m = c->dm;
        I.s = c->state();
        I.P = c->phys();
        I.sc = c->sc.p; I.sx = c->sx.p; I.sy = c->sy.p;
        I.R = c->R.p; I.sol = c->sol.p; I.jslots = c->jslots.p; I.val = c->val.p;
        I.S = c->S_.p; I.bs = c->bs.p; I.dinv = c->dinv64.p;
        I.aoff = R.mixed ? (void*)c->aoff32.p : (void*)c->aoff64.p;
        I.ewet = c->ewet.p; I.mark = c->mark.p; I.glist = c->glist.p; I.gcount = c->gcount.p; I.ngen = c->ngen.p;
        I.npart = c->npart.p; I.norms = R.norms.p + k; I.ncounter = c->ncounter.p; I.singular = R.singular.p + k;
        I.ndir = (int)c->dir_node.size();
        I.dir_node = c->dir_node_d.p; I.dir_mask = c->dir_mask_d.p;
        I.dir_h = c->dir_h.p; I.dir_u = c->dir_u.p; I.dir_v = c->dir_v.p;
        I.dacont = c->dacont_on ? c->dacont.p : nullptr;
        KrylovInst& Q = R.ktab_h[k];
        KrylovArgs& A = Q.K;
        A.V = c->V;
        A.rowptr = c->orowptr.p;
        A.col = c->ocol.p;
        A.S = c->S_.p;
        A.bs = c->bs.p;
        A.atol = c->p.lin_atol;
        A.maxit = c->p.max_lin_it;
        A.h = c->H(0); A.u = c->U(0); A.v = c->Vv(0);
        A.sol = c->sol.p;
        A.apply_inc = apply_inc;
        A.part = c->part.p;
        A.ctl = R.ctl.p + k;
        A.vgrid = c->krylov_grid;
        A.fuse_update = krylov_fuse_update(c->V);   // alone; a batch launch decides for its group
        A.spin_limit = c->wait_barrier;
        A.copy_limit = c->wait_copy;
        Q.A = I.aoff;
        Q.Dinv = c->dinv64.p;
        for (int v = 0; v < kKrylovVectors; v++) Q.vec[v] = c->kv64[v].p;
        if (c->dilu) dilu_args(R, k, apply_inc);
    }
    R.any_dilu = false;
    for (auto* c : R.ctx) R.any_dilu |= c->dilu;
    // the descriptors travel as kernel parameters; batch Krylov launches and the D-ILU setup
    // kernels read a table
    if (K > 1) CK(cudaMemcpyAsync(R.ktab.p, R.ktab_h, sizeof(KrylovInst) * K, cudaMemcpyHostToDevice, R.stream));
    if (R.any_dilu) CK(cudaMemcpyAsync(R.dtab.p, R.dtab_h, sizeof(DiluArgs) * K, cudaMemcpyHostToDevice, R.stream));
    if (K > 1 || R.any_dilu) {
        CK(cudaEventRecord(R.tab_ev, R.stream));
        R.tab_pending = true;
    }
    return 0;
}

// map of a subset: instance k gets blocks(k) blocks (none: left out); returns the block total
template <class F>
int make_map(LaunchMap& mp, const std::vector<int>& subset, F blocks) {
    int off = 0;
    mp.n = 0;
    for (int k : subset) {
        const int nb = blocks(k);
        if (nb <= 0) continue;
        mp.boff[mp.n] = off;
        mp.ids[mp.n] = k;
        off += nb;
        mp.n++;
    }
    mp.boff[mp.n] = off;
    return off;
}

// one launch over the subset: instance k gets blocks(k) blocks of `threads` threads, and
// go(src, blocks, threads) launches the kernel with its instance source -- the descriptor
// itself when one instance is mapped, else groups of descriptors with their block ranges
template <class F, class G>
int launch_map(Runner& R, const std::vector<int>& subset, int threads, F blocks, G go) {
    static thread_local LaunchMap mp;   // ~2 KB: not on every caller's stack
    static thread_local SrcPar par;     // ~22 KB
    const int nb = make_map(mp, subset, blocks);
    if (nb == 0) return 0;
    if (mp.n == 1) {
        SrcOne one;
        one.I = R.tab_h[mp.ids[0]];
        go(one, nb, threads);
        R.launches++;
    } else {
        // groups of kParInst instances, descriptors as kernel parameters
        for (int j0 = 0; j0 < mp.n; j0 += kParInst) {
            const int j1 = std::min(mp.n, j0 + kParInst);
            par.n = j1 - j0;
            for (int j = j0; j < j1; j++) {
                par.boff[j - j0] = mp.boff[j] - mp.boff[j0];
                par.I[j - j0] = R.tab_h[mp.ids[j]];
            }
            par.boff[j1 - j0] = mp.boff[j1] - mp.boff[j0];
            go(par, par.boff[j1 - j0], threads);
            R.launches++;
        }
    }
    CK(cudaGetLastError());
    return 0;
}
#define SW2_GO(kernel, ...) [&](const auto& src, int nb_, int th_) { kernel<<<nb_, th_, 0, R.stream>>>(src, ##__VA_ARGS__); }
#define SW2_GO_T(kernel, T, ...) \
    [&](const auto& src, int nb_, int th_) { kernel<std::decay_t<decltype(src)>, T><<<nb_, th_, 0, R.stream>>>(src, ##__VA_ARGS__); }

int launch_init(Runner& R, const std::vector<int>& sub) {     // fe_sw2_init
    int rc = 0;
    auto C = [&](int k) { return R.ctx[k]; };
    if ((rc = launch_map(R, sub, 256, [&](int k) { return nblk(C(k)->V, 256); }, SW2_GO(k_init_level<std::decay_t<decltype(src)>>)))) return rc;
    if ((rc = launch_map(R, sub, 128, [&](int k) { return nblk((int)C(k)->dir_node.size(), 128); }, SW2_GO(k_dirichlet<std::decay_t<decltype(src)>>))))
        return rc;
    if ((rc = launch_map(R, sub, 256, [&](int k) { return nblk(C(k)->T, 256); }, SW2_GO(k_wd_mark<std::decay_t<decltype(src)>>)))) return rc;
    return launch_map(R, sub, 256, [&](int k) { return nblk(C(k)->T, 256); }, SW2_GO(k_wd_flag<std::decay_t<decltype(src)>>));
}

// residual at the current state: element slots, reference-order gather, norms (async)
int launch_resid(Runner& R, const std::vector<int>& sub) {
    Phase ph(&R, kPhResid);
    bool dac = false;   // some instance keeps the transport side output
    for (int k : sub) dac |= R.ctx[k]->dacont_on;
    auto blocks = [&](int k) { return nblk(R.ctx[k]->T + R.ctx[k]->E, 128); };
    int rc = dac ? launch_map(R, sub, 128, blocks,
                              [&](const auto& src, int nb_, int th_) {
                                  k_resid_elem<std::decay_t<decltype(src)>, true><<<nb_, th_, 0, R.stream>>>(src);
                              })
                 : launch_map(R, sub, 128, blocks, SW2_GO(k_resid_elem<std::decay_t<decltype(src)>>));
    if (rc) return rc;
    return launch_map(R, sub, kGatherThreads, [&](int k) { return nblk(R.ctx[k]->V, kGatherThreads); },
                      SW2_GO(k_resid_gather<std::decay_t<decltype(src)>>));
}

// norms (and Krylov control words) of every instance; the one host sync of an evaluation.
// `evaluated`: the instances whose residual was just computed (their slots hold fresh norms;
// the others' slots may hold an earlier occupant's)
int enqueue_results(Runner& R) {
    const int K = (int)R.ctx.size();
    CK(cudaMemcpyAsync(R.norms_h, R.norms.p, sizeof(Norms) * K, cudaMemcpyDeviceToHost, R.stream));
    CK(cudaMemcpyAsync(R.ctl_h, R.ctl.p, sizeof(KrylovCtl) * K, cudaMemcpyDeviceToHost, R.stream));
    return 0;
}
int finish_results(Runner& R, const std::vector<int>& evaluated) {
    CK(cudaStreamSynchronize(R.stream));
    for (int k : evaluated) R.ctx[k]->ngeneral = R.norms_h[k].ngeneral;
    return 0;
}
int read_results(Runner& R, const std::vector<int>& evaluated) {
    int rc = enqueue_results(R);
    return rc ? rc : finish_results(R, evaluated);
}

int launch_jacobian(Runner& R, const std::vector<int>& sub) {
    Phase ph(&R, kPhJac);
    auto C = [&](int k) { return R.ctx[k]; };
    // the general list and the wet flags come from the residual evaluated at this same state
    auto wet_blocks = [&](int k) { return nblk(C(k)->T, kJacElems); };
    auto wet = [&](auto minb) {   // persistent: the grid walks the launch's nb_ element groups
        constexpr int MB = decltype(minb)::value;
        return launch_map(R, sub, kJacWetThreads, wet_blocks, [&](const auto& src, int nb_, int th_) {
            k_jac_elem_wet<std::decay_t<decltype(src)>, MB>
                <<<std::min(nb_, R.jac_ctas[MB - 1]), th_, kJacWetSmem, R.stream>>>(src, nb_);
        });
    };
    if (!R.jac_ctas[R.jac_minb - 1])
        return fail(SW2GPU_E_CUDA, "wet-Jacobian variant %d does not fit on this device", R.jac_minb);
    int rc = R.jac_minb == 1 ? wet(std::integral_constant<int, 1>{}) : wet(std::integral_constant<int, 2>{});
    if (rc) return rc;
    // a captured launch covers the largest list (the kernel reads the list's length itself)
    if ((rc = launch_map(R, sub, kJacThreads,
                         [&](int k) { return nblk(R.capturing ? C(k)->T : C(k)->ngeneral, kJacElems); },
                         SW2_GO(k_jac_elem_general<std::decay_t<decltype(src)>>))))
        return rc;
    if ((rc = launch_map(R, sub, 128, [&](int k) { return nblk(6LL * C(k)->E, 128); }, SW2_GO(k_jac_edge<std::decay_t<decltype(src)>>)))) return rc;
    return launch_map(R, sub, kGatherBlocks, [&](int k) { return nblk(C(k)->nnzb, kGatherBlocks); },
                      SW2_GO(k_jac_gather<std::decay_t<decltype(src)>>));
}

// Krylov CTAs per instance: shares of the co-resident capacity by expected work (blocks x
// iterations of the instance's last solve), at least one, at most its virtual CTAs, so that
// the instances of a launch finish together
std::vector<int> krylov_shares(Runner& R, const std::vector<int>& sub, const std::vector<int>* done = nullptr) {
    // the min-max allocation of sw2_shares.h over the instances' predicted work (done[k]:
    // iterations a resumed solve has behind it)
    const int n = (int)sub.size();
    std::vector<double> W(n);
    std::vector<int> G(n);
    for (int j = 0; j < n; j++) {
        const sw2gpu_ctx* c = R.ctx[sub[j]];
        W[j] = krylov_work(c->nnzb, c->pred_its, done ? (*done)[sub[j]] : 0);
        G[j] = c->krylov_grid;
    }
    return krylov_shares_minmax(W, G, R.capacity);
}

// scaling, preconditioner folding and the persistent BiCGSTAB of the subset, each instance
// with its own relative tolerance eta[k]
// The exact banded LU solve of instance k (SW2GPU_PREC_BAND), after k_rowscale: the scaled system
// into the band, its factors, the two triangular solves and the increment, on the runner's stream.
int launch_band(Runner& R, int k) {
    sw2gpu_ctx* c = R.ctx[k];
    BandArgs B;
    B.V = c->V;
    B.n = 3 * c->V;
    B.bw = c->band_bw;
    B.width = 2 * c->band_bw + 1;
    B.perm = c->band_perm.p;
    B.rowptr = c->rowptr.p;
    B.col = c->col.p;
    B.val = c->val.p;
    B.S = c->S_.p;
    B.bs = c->bs.p;
    B.band = c->band_mem.p;
    B.y = c->band_y.p;
    CK(cudaMemsetAsync(B.band, 0, sizeof(double) * (size_t)B.n * B.width, R.stream));
    k_band_fill<<<nblk(c->nnzb, 256), 256, 0, R.stream>>>(B, c->blk_row.p, c->nnzb);
    k_band_rhs<<<nblk(c->V, 256), 256, 0, R.stream>>>(B);
    k_band_factor<<<1, kBandThreads, 0, R.stream>>>(B);
    k_band_solve<<<1, kBandThreads, 0, R.stream>>>(B);
    k_band_apply<<<nblk(c->V, 256), 256, 0, R.stream>>>(B, c->H(0), c->U(0), c->Vv(0), c->sol.p,
                                                          R.ktab_h[k].K.apply_inc, R.ctl.p + k);
    CK(cudaGetLastError());
    R.launches += 5;
    return 0;
}

// co-resident CTAs of the D-ILU solve kernel on this device (every instantiation)
int dilu_capacity() {
    static int cap = 0;
    if (cap) return cap;
    int dev = 0, sms = 0, fit = 1 << 30;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    const void* ks[4] = {(const void*)k_dilu_bicgstab<double, DiluOne>, (const void*)k_dilu_bicgstab<double, DiluTab>,
                         (const void*)k_dilu_bicgstab<float, DiluOne>, (const void*)k_dilu_bicgstab<float, DiluTab>};
    for (const void* k : ks) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kDiluThreads, 0) != cudaSuccess) return 0;
        fit = std::min(fit, n);
    }
    cap = sms * std::max(fit, 0);
    return cap;
}

// The block D-ILU setup and solve of the instances `dl` (after k_rowscale): the scaled blocks
// into the coloured order, the modified diagonal blocks colour by colour, then one cooperative
// solve per group of instances whose CTAs fit on the device at once.
int launch_dilu(Runner& R, const std::vector<int>& dl, const std::vector<double>& eta) {
    if (dl.empty()) return 0;
    auto C = [&](int k) { return R.ctx[k]; };
    static thread_local DiluMap dmap;   // ~2 KB: not on every caller's stack
    dmap.tab = R.dtab.p;
    int nb = make_map(dmap.mp, dl, [&](int k) { return nblk(C(k)->dl_nlo + C(k)->dl_nup + C(k)->dl_rows, 256); });
    if (nb) {
        if (R.mixed) k_dilu_scatter<float><<<nb, 256, 0, R.stream>>>(dmap);
        else k_dilu_scatter<double><<<nb, 256, 0, R.stream>>>(dmap);
        R.launches++;
    }
    int maxc = 0;
    for (int k : dl) maxc = std::max(maxc, C(k)->dl_ncol);
    for (int c = 0; c < maxc; c++) {
        nb = make_map(dmap.mp, dl, [&](int k) {
            const sw2gpu_ctx* x = C(k);
            return c < x->dl_ncol ? nblk(x->dl_cend[c] - x->dl_cstart[c], 256) : 0;
        });
        if (!nb) continue;
        if (R.mixed) k_dilu_diag<float><<<nb, 256, 0, R.stream>>>(dmap, c);
        else k_dilu_diag<double><<<nb, 256, 0, R.stream>>>(dmap, c);
        R.launches++;
    }
    CK(cudaGetLastError());
    const int cap = dilu_capacity();
    if (cap <= 0) return fail(SW2GPU_E_CUDA, "the D-ILU solve kernel does not fit on this device");
    size_t j0 = 0;
    while (j0 < dl.size()) {
        std::vector<int> grp;
        int total = 0;
        for (size_t j = j0; j < dl.size() && (int)grp.size() < kMaxBatch; j++) {
            const int q = C(dl[j])->dl_cta;
            if (!grp.empty() && total + q > cap) break;
            grp.push_back(dl[j]);
            total += q;
        }
        j0 += grp.size();
        if (grp.size() == 1) {
            DiluOne one;
            one.K = R.dtab_h[grp[0]];
            one.rtol = eta[grp[0]];
            one.rtol_dev = R.capturing ? R.eta_dev.p + grp[0] : nullptr;
            void* args[] = {(void*)&one};
            void* kern = R.mixed ? (void*)k_dilu_bicgstab<float, DiluOne> : (void*)k_dilu_bicgstab<double, DiluOne>;
            CK(cudaLaunchCooperativeKernel(kern, dim3(total), dim3(kDiluThreads), args, 0, R.stream));
        } else {
            static thread_local DiluTab t;   // ~4 KB
            t.tab = R.dtab.p;
            t.rtol_dev = R.capturing ? R.eta_dev.p : nullptr;
            make_map(t.mp, grp, [&](int k) { return C(k)->dl_cta; });
            for (size_t j = 0; j < grp.size(); j++) t.rtol[j] = eta[grp[j]];
            void* args[] = {(void*)&t};
            void* kern = R.mixed ? (void*)k_dilu_bicgstab<float, DiluTab> : (void*)k_dilu_bicgstab<double, DiluTab>;
            CK(cudaLaunchCooperativeKernel(kern, dim3(total), dim3(kDiluThreads), args, 0, R.stream));
        }
        R.launches++;
    }
    return 0;
}

int launch_linear(Runner& R, const std::vector<int>& all, const std::vector<double>& eta) {
    auto C = [&](int k) { return R.ctx[k]; };
    std::vector<int> sub, band, dl;   // block-Jacobi Krylov instances, direct banded solves, D-ILU solves
    for (int k : all) (C(k)->band ? band : C(k)->dilu ? dl : sub).push_back(k);
    CK(cudaMemsetAsync(R.singular.p, 0, sizeof(int) * R.ctx.size(), R.stream));
    int rc = launch_map(R, all, 256, [&](int k) { return nblk(C(k)->V, 256); }, SW2_GO(k_rowscale<std::decay_t<decltype(src)>>, 0));
    if (rc) return rc;
    if (R.mixed)
        rc = launch_map(R, sub, 256, [&](int k) { return nblk(C(k)->nnzb, 256); }, SW2_GO_T(k_fold_offdiag, float));
    else
        rc = launch_map(R, sub, 256, [&](int k) { return nblk(C(k)->nnzb, 256); }, SW2_GO_T(k_fold_offdiag, double));
    if (rc) return rc;
    CK(cudaMemsetAsync(R.ctl.p, 0, sizeof(KrylovCtl) * R.ctx.size(), R.stream));
    Phase ph(&R, kPhKrylov);
    for (int k : band)
        if ((rc = launch_band(R, k))) return rc;
    if ((rc = launch_dilu(R, dl, eta))) return rc;
    // instances that cannot all be co-resident go in successive launches
    size_t j0 = 0;
    const StageLayout lay{R.c_off, R.r_off, R.v_off, R.stage_bytes};
    while (j0 < sub.size()) {
        std::vector<int> grp;
        for (size_t j = j0; j < sub.size() && (int)grp.size() < R.capacity; j++) grp.push_back(sub[j]);
        j0 += grp.size();
        if (grp.size() == 1) {
            const std::vector<int> P = krylov_shares(R, grp);
            KrylovOne one;
            one.Q = R.ktab_h[grp[0]];
            one.rtol = eta[grp[0]];
            one.rtol_dev = R.capturing ? R.eta_dev.p + grp[0] : nullptr;
            one.lay = lay;
            void* args[] = {(void*)&one};
            void* kern = R.mixed ? krylov_kernel<float, KrylovOne>(R.stages) : krylov_kernel<double, KrylovOne>(R.stages);
            CK(cudaLaunchCooperativeKernel(kern, dim3(P[0]), dim3(kKrylovThreads), args, R.smem, R.stream));
            R.launches++;
            continue;
        }
        // rebalancing rounds (host-driven launches only: the host reads which instances paused)
        const int rounds = R.capturing ? 1 : std::max(1, std::min(R.rb_rounds, (int)Runner::kMaxRounds));
        if (rounds > 1) CK(cudaMemsetAsync(R.kdone.p, 0, sizeof(unsigned) * rounds, R.stream));
        std::vector<int> done(R.ctx.size(), 0);   // iterations a paused solve has behind it
        for (int round = 0; round < rounds; round++) {
            const bool last = round + 1 == rounds;
            const std::vector<int> P = krylov_shares(R, grp, round ? &done : nullptr);
            int total = 0;
            for (int q : P) total += q;
            static thread_local KrylovTab t;   // ~4 KB: not on the stack of every caller
            int off = 0;
            t.tab = R.ktab.p;
            t.rtol_dev = R.capturing ? R.eta_dev.p : nullptr;
            t.mp.n = (int)grp.size();
            for (size_t j = 0; j < grp.size(); j++) {
                t.mp.boff[j] = off;
                t.mp.ids[j] = grp[j];
                t.rtol[j] = eta[grp[j]];
                off += P[j];
            }
            t.mp.boff[grp.size()] = off;
            t.lay = lay;
            long long nodes = 0;
            for (int k : grp) nodes += C(k)->V;
            t.fuse = krylov_fuse_update(nodes);
            t.done_ctas = last ? nullptr : R.kdone.p + round;
            t.pause_after = (unsigned)std::ceil(R.rb_frac * total);
            t.resume = round > 0 ? 1 : 0;
            if (round > 0) {
                k_krylov_rearm<<<nblk((int)grp.size(), 128), 128, 0, R.stream>>>(R.ctl.p, t.mp);
                R.launches++;
            }
            void* args[] = {(void*)&t};
            void* kern = R.mixed ? krylov_kernel<float, KrylovTab>(R.stages) : krylov_kernel<double, KrylovTab>(R.stages);
            CK(cudaLaunchCooperativeKernel(kern, dim3(total), dim3(kKrylovThreads), args, R.smem, R.stream));
            R.launches++;
            if (last) break;
            CK(cudaMemcpyAsync(R.ctl_h, R.ctl.p, sizeof(KrylovCtl) * R.ctx.size(), cudaMemcpyDeviceToHost, R.stream));
            CK(cudaStreamSynchronize(R.stream));
            std::vector<int> next;
            for (int k : grp)
                if (R.ctl_h[k].paused && !R.ctl_h[k].err) {
                    next.push_back(k);
                    done[k] = R.ctl_h[k].s_it;
                }
            if (next.empty()) break;
            grp.swap(next);
        }
    }
    return 0;
}

int launch_half_inc(Runner& R, const std::vector<int>& sub) {
    return launch_map(R, sub, 256, [&](int k) { return nblk(R.ctx[k]->V, 256); }, SW2_GO(k_half_inc<std::decay_t<decltype(src)>>));
}

// Newton state of one instance inside a time step (fe_newton.c:214-912)
struct NState {
    double rmax = 0, l2 = 0, imax = 0, old_l2 = 0, eta = 0;
    int it = 0, lin = 0, cuts = 0, cuts_total = 0;
    bool ok = true, nan = false, done = false;
};

// Inexact Newton: the linear residual of iteration k only needs to be small next to the
// Newton tolerance, so the Krylov test is relative with
//   eta_k = max(lin_rtol, kEtaNtl * tol_nonlin / max|R_k|)      (capped at 1e-5).
// Early iterations (large R) solve to near round-off like the reference's exact LU; late
// ones (R close to tol_nonlin) stop early.  A solve that reaches max_lin_it but reduced its
// residual by kAcceptRel is accepted: its error is already far below what the next residual
// evaluation can see.
constexpr double kEtaNtl = 1e-4, kAcceptRel = 1e-8;

// the state after the residual at the start of a step (norms read)
void newton_begin(Runner& R, int k, NState& ns) {
    const Norms& nm = R.norms_h[k];
    ns = NState();
    ns.rmax = nm.rmax;
    ns.l2 = std::sqrt(nm.l2sum / (3.0 * R.ctx[k]->V));
    ns.imax = nm.imax;
    if (nm.nan) {
        ns.nan = true;
        ns.ok = false;
        ns.done = true;
    }
}

// one Newton iteration (Jacobian, Krylov, update, residual, line search, convergence test) of
// every instance of `act`, each in one launch per phase; sets ns[k].done when k's step ends
// Krylov tolerances of the instances' next solves (and their predicted iteration counts)
std::vector<double> newton_eta(Runner& R, const std::vector<int>& act, const std::vector<NState>& ns) {
    std::vector<double> eta(R.ctx.size(), 0.0);
    for (int k : act) {
        sw2gpu_ctx* c = R.ctx[k];
        const sw2gpu_params& p = c->p;
        eta[k] = std::min(1e-5, std::max(p.lin_rtol, kEtaNtl * p.tol_nonlin / std::max(ns[k].rmax, 1e-300)));
        // the larger count of the last two steps at this Newton iteration: a launch lasts as
        // long as its most underestimated instance, and one atypical solve (a line-search cut,
        // an extra iteration) would otherwise set the next prediction far too low
        const int i = std::min(ns[k].it, 7);
        const int seen = std::max(c->its_at[i], c->its_prev[i]);
        if (seen > 0) c->pred_its = seen;
    }
    return eta;
}

// the launches of one Newton iteration (Jacobian, Krylov with its update, residual, result copies)
int newton_launch(Runner& R, const std::vector<int>& act, const std::vector<double>& eta) {
    int rc = launch_jacobian(R, act);
    if (!rc) rc = launch_linear(R, act, eta);
    if (!rc) rc = launch_resid(R, act);
    if (!rc) rc = enqueue_results(R);
    return rc;
}

int newton_finish(Runner& R, const std::vector<int>& act, std::vector<NState>& ns);

int newton_iteration(Runner& R, const std::vector<int>& act, std::vector<NState>& ns) {
    const std::vector<double> eta = newton_eta(R, act, ns);
    for (int k : act) ns[k].old_l2 = ns[k].l2;
    int rc = newton_launch(R, act, eta);
    return rc ? rc : newton_finish(R, act, ns);
}

// results of a Newton iteration: line search, convergence test
int newton_finish(Runner& R, const std::vector<int>& act, std::vector<NState>& ns) {
    int rc = finish_results(R, act);
    if (rc) return rc;
    std::vector<int> ls;
    for (int k : act) {
        NState& n = ns[k];
        const sw2gpu_params& p = R.ctx[k]->p;
        const KrylovCtl& q = R.ctl_h[k];
        if (q.err) return fail(SW2GPU_E_TIMEOUT, "instance %d: Krylov barrier or tile-copy wait ran out", k);
        n.lin += q.iterations;
        R.ctx[k]->its_at[std::min(n.it, 7)] = std::max(q.iterations, 1);
        R.ctx[k]->pred_its = std::max(q.iterations, 1);
        // the plain path fails the step when BiCGSTAB hits max_lin_it without a useful
        // reduction (solv_bcgstab.c:280-292); on the mixed path the FP32 inner solve is a
        // correction refined by the FP64 Newton loop, so its last iterate is accepted (the
        // reference's force_lin_it behaviour)
        if (!q.converged && p.precision != SW2GPU_MIXED && !(q.rnorm <= kAcceptRel * q.bnorm)) n.ok = false;
        const Norms& nm = R.norms_h[k];
        n.rmax = nm.rmax;
        n.l2 = std::sqrt(nm.l2sum / (3.0 * R.ctx[k]->V));
        n.imax = nm.imax;
        if (nm.nan || std::isnan(n.l2) || std::isinf(n.l2)) {
            n.ok = false;
            n.nan = true;
        }
        n.cuts = 0;
        if (n.rmax > p.tol_nonlin && n.l2 > n.old_l2 && n.cuts < p.max_linesearch_cuts) ls.push_back(k);
    }
    // line search (fe_newton.c:692-747): halve the increment while the l2 norm grew
    while (!ls.empty()) {
        if ((rc = launch_half_inc(R, ls))) return rc;
        if ((rc = launch_resid(R, ls))) return rc;
        if ((rc = read_results(R, ls))) return rc;
        std::vector<int> next;
        for (int k : ls) {
            NState& n = ns[k];
            const sw2gpu_params& p = R.ctx[k]->p;
            const Norms& nm = R.norms_h[k];
            n.rmax = nm.rmax;
            n.l2 = std::sqrt(nm.l2sum / (3.0 * R.ctx[k]->V));
            n.imax = nm.imax;
            n.cuts++;
            if (n.rmax > p.tol_nonlin && n.l2 > n.old_l2 && n.cuts < p.max_linesearch_cuts) next.push_back(k);
        }
        ls.swap(next);
    }
    for (int k : act) {
        NState& n = ns[k];
        const sw2gpu_params& p = R.ctx[k]->p;
        n.cuts_total += n.cuts;
        n.it++;
        const bool keep = n.ok && n.it < p.max_nonlin_it && n.rmax < 1.0E+20 && (n.rmax > p.tol_nonlin && n.imax > p.inc_nonlin);
        if (!keep) n.done = true;
    }
    return 0;
}

// status of a finished step (0 = YES)
int newton_status(const NState& n, const sw2gpu_params& p) {
    if (!n.ok || (n.rmax > p.tol_nonlin && n.imax > p.inc_nonlin) || n.rmax >= 1.0E+20)
        return n.nan ? SW2GPU_E_NAN : (!n.ok ? SW2GPU_E_LINEAR : SW2GPU_E_NEWTON);
    return SW2GPU_OK;
}

// start of a step for instance k: dt, level rotation (fe_sw2: older <- old <- current, no
// copies) and the step tables
int step_begin(Runner& R, int k, double dt, const double* series) {
    sw2gpu_ctx* c = R.ctx[k];
    c->dt = dt;
    for (int i = 0; i < 8; i++) {
        c->its_prev[i] = c->its_snap[i];
        c->its_snap[i] = c->its_at[i];
    }
    const int o2 = c->lv[2];
    c->lv[2] = c->lv[1];
    c->lv[1] = c->lv[0];
    c->lv[0] = o2;
    return upload_step_tables(c, series, R.stream);
}

void phase_times(Runner& R, double ph[3]) {
    ph[0] = ph[1] = ph[2] = 0.0;
    for (int q = 0; q < R.nphase; q++) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, R.pev[2 * q], R.pev[2 * q + 1]) == cudaSuccess) ph[R.pkind[q]] += t;
    }
}

// the grid mass and the mass flux of instance c's accepted step, reduced on its stream `st`
// into the context's pinned mirror (the values are read after the step's final sync)
int enqueue_step_mass(sw2gpu_ctx* c, cudaStream_t st) {
    double* part = c->mass_part.p;
    double* res = part + 2 * kMassBlocks + 1;   // [0] grid mass, [1] flux
    k_mass_partial<false><<<kMassBlocks, kMassThreads, 0, st>>>(c->dm, c->H(0), nullptr, nullptr, 0.0, c->mass_density,
                                                                part);
    k_mass_final<false><<<1, kMassThreads, 0, st>>>(part, c->mass_density, res);
    k_mass_partial<true><<<kMassBlocks, kMassThreads, 0, st>>>(c->dm, c->H(0), c->U(0), c->Vv(0), c->dt,
                                                               c->mass_density, part);
    k_mass_final<true><<<1, kMassThreads, 0, st>>>(part, c->mass_density, res + 1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->mass_h, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    return 0;
}

// after a Krylov wait ran out: the instances back at their old level, the error text kept
void reset_after_timeout(Runner& R, const std::vector<int>& sub) {
    const std::string msg = g_err;
    if (launch_init(R, sub) == 0) cudaStreamSynchronize(R.stream);
    g_err = msg;
}

// One time step of every instance (fe_sw2 level shift + fe_newton), the instances in
// lockstep: each Newton phase is one launch over the instances still iterating, and each
// instance follows exactly the decisions it takes alone.
int ensure_batch_graphs(Runner& R, const std::vector<int>& all, Runner::BatchGraph** out);

int runner_step(Runner& R, const double* dt, const double* const* series, sw2gpu_stats* stats, int* status) {
    const int K = (int)R.ctx.size();
    for (int k = 0; k < K; k++)
        if (!(dt[k] > 0.0)) return fail(SW2GPU_E_ARG, "instance %d: bad dt", k);
    R.launches = 0;
    R.nphase = 0;
    CK(cudaEventRecord(R.ev0, R.stream));
    int rc = 0;
    for (int k = 0; k < K; k++)
        if ((rc = step_begin(R, k, dt[k], series ? series[k] : nullptr))) return rc;
    if ((rc = runner_tables(R, 1))) return rc;
    std::vector<int> all(K);
    for (int k = 0; k < K; k++) all[k] = k;
    // a batch replaying from CUDA graphs: the step start and every Newton iteration in which all
    // instances iterate are graph launches; iterations of a subset launch directly
    Runner::BatchGraph* G = nullptr;
    if (R.use_graphs && K > 1 && (rc = ensure_batch_graphs(R, all, &G))) return rc;
    if (G) {
        CK(cudaGraphLaunch(G->start, R.stream));
        R.launches += G->kernels_start;
        if ((rc = finish_results(R, all))) return rc;
    } else {
        if ((rc = launch_init(R, all))) return rc;
        if ((rc = launch_resid(R, all))) return rc;
        if ((rc = read_results(R, all))) return rc;
    }
    std::vector<NState> ns(K);
    for (int k = 0; k < K; k++) newton_begin(R, k, ns[k]);
    for (;;) {
        std::vector<int> act;
        for (int k = 0; k < K; k++)
            if (!ns[k].done) act.push_back(k);
        if (act.empty()) break;
        if (G && (int)act.size() == K) {
            const std::vector<double> eta = newton_eta(R, act, ns);
            for (int k = 0; k < K; k++) {
                R.eta_h[k] = eta[k];
                ns[k].old_l2 = ns[k].l2;
            }
            CK(cudaMemcpyAsync(R.eta_dev.p, R.eta_h, sizeof(double) * K, cudaMemcpyHostToDevice, R.stream));
            CK(cudaGraphLaunch(G->newton, R.stream));
            R.launches += G->kernels_newton;
            rc = newton_finish(R, act, ns);
        } else {
            rc = newton_iteration(R, act, ns);
        }
        if (rc) {
            // a device wait that ran out ends the step like a failed one: every instance is
            // back at its old level (fe_sw2_init) and the caller may step again
            if (rc == SW2GPU_E_TIMEOUT) reset_after_timeout(R, all);
            return rc;
        }
    }
    std::vector<int> failed;
    for (int k = 0; k < K; k++) {
        status[k] = newton_status(ns[k], R.ctx[k]->p);
        if (status[k] != SW2GPU_OK) failed.push_back(k);
    }
    if (!failed.empty() && (rc = launch_init(R, failed))) return rc;   // reset to the old level
    // mass balance of the accepted steps, in the same stream order (no extra host round trip)
    for (int k = 0; k < K; k++) {
        sw2gpu_ctx* c = R.ctx[k];
        c->mass_valid = false;
        if (c->mass_on && status[k] == SW2GPU_OK) {
            if ((rc = enqueue_step_mass(c, R.stream))) return rc;
            R.launches += 4;
        }
    }
    CK(cudaEventRecord(R.ev1, R.stream));
    CK(cudaEventSynchronize(R.ev1));
    for (int k = 0; k < K; k++) {
        sw2gpu_ctx* c = R.ctx[k];
        if (c->mass_on && status[k] == SW2GPU_OK) {
            c->step_mass = c->mass_h[0];
            c->step_flux = c->mass_h[1];
            c->mass_valid = true;
        }
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, R.ev0, R.ev1);
    double ph[3];
    phase_times(R, ph);
    if (stats) {
        for (int k = 0; k < K; k++) {
            sw2gpu_stats& st = stats[k];
            const NState& n = ns[k];
            memset(&st, 0, sizeof(st));
            st.status = status[k];
            st.newton_its = n.it;
            st.linear_its = n.lin;
            st.linesearch_cuts = n.cuts_total;
            st.resid_max = n.rmax;
            st.resid_l2 = n.l2;
            st.inc_max = n.imax;
            st.device_ms = ms;
            st.kernel_launches = R.launches;
            st.jac_ms = ph[kPhJac];
            st.krylov_ms = ph[kPhKrylov];
            st.resid_ms = ph[kPhResid];
            st.other_ms = ms - ph[0] - ph[1] - ph[2];
        }
    }
    return 0;
}


// captures body()'s launches on R.stream into an executable graph; `kernels` = launches made
template <class F>
int capture_graph(Runner& R, cudaGraphExec_t* out, int* kernels, F body) {
    cudaGraph_t g = nullptr;
    const int l0 = R.launches;
    CK(cudaStreamBeginCapture(R.stream, cudaStreamCaptureModeThreadLocal));
    R.capturing = true;
    const int rc = body();
    R.capturing = false;
    const cudaError_t e = cudaStreamEndCapture(R.stream, &g);
    *kernels = R.launches - l0;
    R.launches = l0;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(SW2GPU_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return fail(SW2GPU_E_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ei));
    return 0;
}

// the batch graphs of the instances' current level arrangement, dt and launch variant
// (captured when new; the three most recent are kept)
int ensure_batch_graphs(Runner& R, const std::vector<int>& all, Runner::BatchGraph** out) {
    std::vector<int> lv;
    std::vector<double> dts;
    for (auto* c : R.ctx) {
        lv.push_back(c->lv[0]);
        dts.push_back(c->dt);
    }
    for (auto& g : R.bgraphs)
        if (g.lv == lv && g.dt == dts && g.jac_minb == R.jac_minb && g.stages == R.stages) {
            *out = &g;
            return 0;
        }
    if (R.bgraphs.size() >= 3) {
        if (R.bgraphs.front().start) cudaGraphExecDestroy(R.bgraphs.front().start);
        if (R.bgraphs.front().newton) cudaGraphExecDestroy(R.bgraphs.front().newton);
        R.bgraphs.erase(R.bgraphs.begin());
    }
    Runner::BatchGraph g;
    g.lv = lv;
    g.dt = dts;
    g.jac_minb = R.jac_minb;
    g.stages = R.stages;
    int rc = capture_graph(R, &g.start, &g.kernels_start, [&] {
        int r = launch_init(R, all);
        if (!r) r = launch_resid(R, all);
        if (!r) r = enqueue_results(R);
        return r;
    });
    if (!rc) rc = capture_graph(R, &g.newton, &g.kernels_newton, [&] {
        // every Krylov launch reads its instance's tolerance from eta_dev
        return newton_launch(R, all, std::vector<double>(all.size(), 0.0));
    });
    if (rc) {
        if (g.start) cudaGraphExecDestroy(g.start);
        if (g.newton) cudaGraphExecDestroy(g.newton);
        return rc;
    }
    R.bgraphs.push_back(g);
    *out = &R.bgraphs.back();
    return 0;
}

// the graphs of the current level arrangement, (re)captured if dt or a variant changed since;
// the descriptors (state pointers of this arrangement, dt) are baked into their launches
int ensure_graphs(sw2gpu_ctx* c) {
    Runner& R = *c->self;
    sw2gpu_ctx::StepGraph& G = c->graphs[c->lv[0]];
    if (G.start && G.newton && G.dt == c->dt && G.jac_minb == R.jac_minb && G.stages == R.stages) return 0;
    if (G.start) cudaGraphExecDestroy(G.start);
    if (G.newton) cudaGraphExecDestroy(G.newton);
    G = sw2gpu_ctx::StepGraph();
    const std::vector<int> one(1, 0);
    int rc = capture_graph(R, &G.start, &G.kernels_start, [&] {
        int r = launch_init(R, one);
        if (!r) r = launch_resid(R, one);
        if (!r) r = enqueue_results(R);
        return r;
    });
    if (!rc) rc = capture_graph(R, &G.newton, &G.kernels_newton, [&] {
        return newton_launch(R, one, std::vector<double>(1, c->p.lin_rtol));   // tolerance read from eta_dev
    });
    if (rc) {
        if (G.start) cudaGraphExecDestroy(G.start);
        G = sw2gpu_ctx::StepGraph();
        return rc;
    }
    G.dt = c->dt;
    G.jac_minb = R.jac_minb;
    G.stages = R.stages;
    return 0;
}

// One time step of a single instance replayed from CUDA graphs: the step start and each
// Newton iteration are one graph launch each (the iteration's Krylov tolerance goes to the
// device first); line-search halvings and the failure reset are direct launches.  Same
// kernels, same arithmetic as runner_step.
int graph_step(sw2gpu_ctx* c, double dt, const double* series, sw2gpu_stats* stats, int* status) {
    Runner& R = *c->self;
    const std::vector<int> one(1, 0);
    R.launches = 0;
    R.nphase = 0;
    CK(cudaEventRecord(R.ev0, R.stream));
    int rc = step_begin(R, 0, dt, series);
    if (!rc) rc = runner_tables(R, 1);
    if (!rc) rc = ensure_graphs(c);
    if (rc) return rc;
    const sw2gpu_ctx::StepGraph& G = c->graphs[c->lv[0]];
    CK(cudaGraphLaunch(G.start, R.stream));
    R.launches += G.kernels_start;
    if ((rc = finish_results(R, one))) return rc;
    std::vector<NState> ns(1);
    newton_begin(R, 0, ns[0]);
    while (!ns[0].done) {
        const std::vector<double> eta = newton_eta(R, one, ns);
        *R.eta_h = eta[0];
        CK(cudaMemcpyAsync(R.eta_dev.p, R.eta_h, sizeof(double), cudaMemcpyHostToDevice, R.stream));
        ns[0].old_l2 = ns[0].l2;
        CK(cudaGraphLaunch(G.newton, R.stream));
        R.launches += G.kernels_newton;
        if ((rc = newton_finish(R, one, ns))) {
            if (rc == SW2GPU_E_TIMEOUT) reset_after_timeout(R, one);
            return rc;
        }
    }
    status[0] = newton_status(ns[0], c->p);
    if (status[0] != SW2GPU_OK && (rc = launch_init(R, one))) return rc;   // reset to the old level
    c->mass_valid = false;
    const bool mass = c->mass_on && status[0] == SW2GPU_OK;
    if (mass) {
        if ((rc = enqueue_step_mass(c, R.stream))) return rc;
        R.launches += 4;
    }
    CK(cudaEventRecord(R.ev1, R.stream));
    CK(cudaEventSynchronize(R.ev1));
    if (mass) {
        c->step_mass = c->mass_h[0];
        c->step_flux = c->mass_h[1];
        c->mass_valid = true;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, R.ev0, R.ev1);
    if (stats) {
        const NState& n = ns[0];
        memset(stats, 0, sizeof(*stats));
        stats->status = status[0];
        stats->newton_its = n.it;
        stats->linear_its = n.lin;
        stats->linesearch_cuts = n.cuts_total;
        stats->resid_max = n.rmax;
        stats->resid_l2 = n.l2;
        stats->inc_max = n.imax;
        stats->device_ms = ms;
        stats->kernel_launches = R.launches;
        stats->other_ms = ms;   // phases are not timed inside graphs
    }
    return 0;
}

// ---------------------------------------------------------------------------------------------
// graph mode 2: the whole step as one graph, the Newton loop and the line search as conditional
// WHILE nodes whose conditions the control kernels of newton_ctl.cuh set, the failure reset as an
// IF node; the host launches it and reads one status word

// nodes of `g` with no outgoing edge
int graph_sinks(cudaGraph_t g, std::vector<cudaGraphNode_t>& out) {
    size_t nn = 0, ne = 0;
    CK(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) CK(cudaGraphGetNodes(g, nodes.data(), &nn));
    CK(cudaGraphGetEdges(g, nullptr, nullptr, &ne));
    std::vector<cudaGraphNode_t> from(ne), to(ne);
    if (ne) CK(cudaGraphGetEdges(g, from.data(), to.data(), &ne));
    out.clear();
    for (cudaGraphNode_t n : nodes)
        if (std::find(from.begin(), from.end(), n) == from.end()) out.push_back(n);
    return 0;
}

// launches of `body` captured into `g` after `deps`; `sinks` receives the graph's new sinks
template <class F>
int capture_into(Runner& R, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, int* kernels,
                 std::vector<cudaGraphNode_t>& sinks, F body) {
    const int l0 = R.launches;
    CK(cudaStreamBeginCaptureToGraph(R.stream, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                     cudaStreamCaptureModeThreadLocal));
    R.capturing = true;
    const int rc = body();
    R.capturing = false;
    cudaGraph_t same = nullptr;
    const cudaError_t e = cudaStreamEndCapture(R.stream, &same);
    *kernels = R.launches - l0;
    R.launches = l0;
    if (rc) return rc;
    if (e != cudaSuccess) return fail(SW2GPU_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    return graph_sinks(g, sinks);
}

int add_conditional(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, cudaGraphConditionalHandle h,
                    cudaGraphConditionalNodeType type, cudaGraphNode_t* node, cudaGraph_t* body) {
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = type;
    np.conditional.size = 1;
    CK(cudaGraphAddNode(node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &np));
    *body = np.conditional.phGraph_out[0];
    return 0;
}

NewtonParams newton_params(const sw2gpu_ctx* c) {
    NewtonParams P;
    P.tol_nonlin = c->p.tol_nonlin;
    P.inc_nonlin = c->p.inc_nonlin;
    P.lin_rtol = c->p.lin_rtol;
    P.eta_ntl = kEtaNtl;
    P.accept_rel = kAcceptRel;
    P.max_nonlin_it = c->p.max_nonlin_it;
    P.max_ls_cuts = c->p.max_linesearch_cuts;
    P.mixed = c->p.precision == SW2GPU_MIXED ? 1 : 0;
    P.V = c->V;
    return P;
}

int ensure_loop_graph(sw2gpu_ctx* c) {
    Runner& R = *c->self;
    sw2gpu_ctx::StepGraph& G = c->graphs[c->lv[0]];
    if (G.loop && G.dt == c->dt && G.jac_minb == R.jac_minb && G.stages == R.stages && G.loop_mass == c->mass_on)
        return 0;
    if (G.loop) cudaGraphExecDestroy(G.loop);
    G.loop = nullptr;
    if (!c->nctl.p) {
        g_alloc_bytes = &c->bytes;
        const int r = zalloc(c->nctl, 1, R.stream);
        g_alloc_bytes = nullptr;
        if (r) return r;
        CK(cudaMallocHost(&c->nctl_h, sizeof(NewtonCtl)));
    }
    const std::vector<int> one(1, 0);
    const NewtonParams P = newton_params(c);
    NewtonCtl* S = c->nctl.p;
    const Norms* NM = R.norms.p;
    const KrylovCtl* KC = R.ctl.p;
    double* ETA = R.eta_dev.p;
    cudaGraph_t T = nullptr;
    CK(cudaGraphCreate(&T, 0));
    struct Own {
        cudaGraph_t g;
        ~Own() { if (g) cudaGraphDestroy(g); }
    } own{T};
    cudaGraphConditionalHandle hN, hF, hL;
    CK(cudaGraphConditionalHandleCreate(&hN, T, 0, cudaGraphCondAssignDefault));
    CK(cudaGraphConditionalHandleCreate(&hF, T, 0, cudaGraphCondAssignDefault));
    std::vector<cudaGraphNode_t> sinks, none;
    int rc;
    // step start: fe_sw2_init, the first residual, the control state
    if ((rc = capture_into(R, T, none, &G.k_start, sinks, [&] {
             int r = launch_init(R, one);
             if (!r) r = launch_resid(R, one);
             if (!r) {
                 k_ctl_begin<<<1, 1, 0, R.stream>>>(S, P, NM, hN);
                 R.launches++;
             }
             return r;
         })))
        return rc;
    // the Newton loop
    cudaGraphNode_t wn;
    cudaGraph_t BN;
    if ((rc = add_conditional(T, sinks, hN, cudaGraphCondTypeWhile, &wn, &BN))) return rc;
    CK(cudaGraphConditionalHandleCreate(&hL, BN, 0, cudaGraphCondAssignDefault));
    int k1 = 0, k2 = 0;
    if ((rc = capture_into(R, BN, none, &k1, sinks, [&] {
             k_ctl_eta<<<1, 1, 0, R.stream>>>(S, P, ETA);
             R.launches++;
             int r = launch_jacobian(R, one);
             if (!r) r = launch_linear(R, one, std::vector<double>(1, c->p.lin_rtol));   // reads eta_dev
             if (!r) r = launch_resid(R, one);
             if (!r) {
                 k_ctl_after<<<1, 1, 0, R.stream>>>(S, P, NM, KC, hL);
                 R.launches++;
             }
             return r;
         })))
        return rc;
    cudaGraphNode_t wl;
    cudaGraph_t BL;
    if ((rc = add_conditional(BN, sinks, hL, cudaGraphCondTypeWhile, &wl, &BL))) return rc;
    std::vector<cudaGraphNode_t> lsinks;
    if ((rc = capture_into(R, BL, none, &G.k_ls, lsinks, [&] {
             int r = launch_half_inc(R, one);
             if (!r) r = launch_resid(R, one);
             if (!r) {
                 k_ctl_ls<<<1, 1, 0, R.stream>>>(S, P, NM, hL);
                 R.launches++;
             }
             return r;
         })))
        return rc;
    if ((rc = capture_into(R, BN, std::vector<cudaGraphNode_t>{wl}, &k2, sinks, [&] {
             k_ctl_end<<<1, 1, 0, R.stream>>>(S, P, hN);
             R.launches++;
             return 0;
         })))
        return rc;
    G.k_body = k1 + k2;
    // the status, the reset of a failed step, the tail
    if ((rc = capture_into(R, T, std::vector<cudaGraphNode_t>{wn}, &G.k_final, sinks, [&] {
             k_ctl_final<<<1, 1, 0, R.stream>>>(S, P, SW2GPU_E_NAN, SW2GPU_E_LINEAR, SW2GPU_E_NEWTON, SW2GPU_E_TIMEOUT,
                                                hF);
             R.launches++;
             return 0;
         })))
        return rc;
    cudaGraphNode_t fi;
    cudaGraph_t BF;
    if ((rc = add_conditional(T, sinks, hF, cudaGraphCondTypeIf, &fi, &BF))) return rc;
    if ((rc = capture_into(R, BF, none, &G.k_reset, lsinks, [&] { return launch_init(R, one); }))) return rc;
    if ((rc = capture_into(R, T, std::vector<cudaGraphNode_t>{fi}, &G.k_tail, sinks, [&] {
             int r = 0;
             if (c->mass_on) {   // reduced whatever the status; the host keeps it for an accepted step
                 r = enqueue_step_mass(c, R.stream);
                 R.launches += 4;
             }
             if (!r && cudaMemcpyAsync(c->nctl_h, S, sizeof(NewtonCtl), cudaMemcpyDeviceToHost, R.stream) != cudaSuccess)
                 r = fail(SW2GPU_E_CUDA, "capturing the status copy failed");
             if (!r) r = enqueue_results(R);
             return r;
         })))
        return rc;
    const cudaError_t ei = cudaGraphInstantiate(&G.loop, T, 0);
    if (ei != cudaSuccess) {
        G.loop = nullptr;
        return fail(SW2GPU_E_CUDA, "step graph instantiation failed: %s", cudaGetErrorString(ei));
    }
    G.dt = c->dt;
    G.jac_minb = R.jac_minb;
    G.stages = R.stages;
    G.loop_mass = c->mass_on;
    return 0;
}

// One time step of a single instance as one graph launch (graph mode 2): the Newton loop's
// decisions are taken on the device; same kernels, same arithmetic as direct stepping.
int loop_step(sw2gpu_ctx* c, double dt, const double* series, sw2gpu_stats* stats, int* status) {
    Runner& R = *c->self;
    R.launches = 0;
    R.nphase = 0;
    CK(cudaEventRecord(R.ev0, R.stream));
    int rc = step_begin(R, 0, dt, series);
    if (!rc) rc = runner_tables(R, 1);
    if (!rc) rc = ensure_loop_graph(c);
    if (rc) return rc;
    const sw2gpu_ctx::StepGraph& G = c->graphs[c->lv[0]];
    CK(cudaGraphLaunch(G.loop, R.stream));
    CK(cudaEventRecord(R.ev1, R.stream));
    CK(cudaEventSynchronize(R.ev1));
    const NewtonCtl n = *c->nctl_h;
    c->ngeneral = R.norms_h[0].ngeneral;
    for (int i = 0; i < std::min(n.it, 8); i++) c->its_at[i] = n.its_at[i];
    if (n.it > 0) c->pred_its = n.its_at[std::min(n.it - 1, 7)];
    R.launches = G.k_start + n.it * G.k_body + (n.timeout ? G.k_body : 0) + n.cuts_total * G.k_ls + G.k_final +
                 (n.status ? G.k_reset : 0) + G.k_tail;
    status[0] = n.status;
    c->mass_valid = false;
    if (c->mass_on && n.status == SW2GPU_OK) {
        c->step_mass = c->mass_h[0];
        c->step_flux = c->mass_h[1];
        c->mass_valid = true;
    }
    if (n.status == SW2GPU_E_TIMEOUT) return fail(SW2GPU_E_TIMEOUT, "Krylov barrier or tile-copy wait ran out");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, R.ev0, R.ev1);
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->status = n.status;
        stats->newton_its = n.it;
        stats->linear_its = n.lin;
        stats->linesearch_cuts = n.cuts_total;
        stats->resid_max = n.rmax;
        stats->resid_l2 = n.l2;
        stats->inc_max = n.imax;
        stats->device_ms = ms;
        stats->kernel_launches = R.launches;
        stats->other_ms = ms;   // phases are not timed inside graphs
    }
    return 0;
}

}  // namespace

extern "C" {

int sw2gpu_abi_version(void) { return SW2GPU_ABI_VERSION; }
const char* sw2gpu_last_error(void) { return g_err.c_str(); }

// The D-ILU order and structure of a context (SW2GPU_PREC_DILU) from the BCSR pattern rp/col:
// greedy colouring of the node graph (nodes in smallest-last order, each taking the lowest
// colour none of its neighbours has), new rows colour by colour in natural order, each new
// row's off-diagonal blocks sorted by new column (lower blocks first), the position of every
// lower block's transpose, and the solve's CTAs: enough warps for the largest colour's 32-row
// tiles, at most the co-resident grid.
int build_dilu(sw2gpu_ctx* c, const std::vector<int>& rp, const std::vector<int>& col, cudaStream_t st) {
    const int V = c->V;
    std::vector<int> colour;
    const int ncol = smallest_last_colouring(rp, col, V, kMaxColours, colour);
    if (ncol < 0) return fail(SW2GPU_E_ARG, "the node graph needs more than %d colours for the D-ILU order", kMaxColours);
    // new rows: colour q occupies pst[q] .. pst[q+1]-1, padded to whole 32-row tiles, its
    // cnt[q] real rows first (natural order); padding rows have old = -1
    std::vector<int> cnt(ncol, 0), pst(ncol + 1, 0);
    for (int n = 0; n < V; n++) cnt[colour[n]]++;
    for (int q = 0; q < ncol; q++) pst[q + 1] = pst[q] + (cnt[q] + 31) / 32 * 32;
    const int N = pst[ncol];
    std::vector<int> old(N, -1), nw(V);
    {
        std::vector<int> f(pst.begin(), pst.end() - 1);
        for (int n = 0; n < V; n++) {
            const int q = f[colour[n]]++;
            old[q] = n;
            nw[n] = q;
        }
    }
    // each real row's off-diagonal blocks (new column, natural block) sorted by new column;
    // lower = lower colours, upper = higher colours
    std::vector<int> lcnt(N, 0), ucnt(N, 0);
    std::vector<std::pair<int, int>> row;
    auto row_of = [&](int n) {
        const int i = old[n];
        row.clear();
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (col[k] != i) row.push_back({nw[col[k]], k});
        std::sort(row.begin(), row.end());
        return (int)(std::lower_bound(row.begin(), row.end(), std::make_pair(n, -1)) - row.begin());
    };
    for (int n = 0; n < N; n++)
        if (old[n] >= 0) {
            lcnt[n] = row_of(n);
            ucnt[n] = (int)row.size() - lcnt[n];
        }
    // ELL layout per colour: colour q's rows take lkn[q] lower and ukn[q] upper slots each (its
    // longest row's counts, at most kDiluMaxSlots); the k-th lower slot of row n is
    // lbase[q] + k L_q + (n - pst[q]), L_q = pst[q+1] - pst[q] (upper: ubase, ukn)
    std::vector<int> lkn(ncol, 0), ukn(ncol, 0), lbase(ncol + 1, 0), ubase(ncol + 1, 0);
    for (int q = 0; q < ncol; q++) {
        for (int n = pst[q]; n < pst[q + 1]; n++) {
            lkn[q] = std::max(lkn[q], lcnt[n]);
            ukn[q] = std::max(ukn[q], ucnt[n]);
        }
        if (lkn[q] > kDiluMaxSlots || ukn[q] > kDiluMaxSlots)
            return fail(SW2GPU_E_ARG, "a node has more than %d neighbours of lower or higher colour (D-ILU order)",
                        kDiluMaxSlots);
        lbase[q + 1] = lbase[q] + lkn[q] * (pst[q + 1] - pst[q]);
        ubase[q + 1] = ubase[q] + ukn[q] * (pst[q + 1] - pst[q]);
    }
    std::vector<int> colour_of(N);
    for (int q = 0; q < ncol; q++)
        for (int n = pst[q]; n < pst[q + 1]; n++) colour_of[n] = q;
    auto lslot = [&](int n, int k) { const int q = colour_of[n]; return lbase[q] + k * (pst[q + 1] - pst[q]) + n - pst[q]; };
    auto uslot = [&](int n, int k) { const int q = colour_of[n]; return ubase[q] + k * (pst[q + 1] - pst[q]) + n - pst[q]; };
    const int nlo = lbase[ncol], nup = ubase[ncol];
    std::vector<int> lcol(nlo, -1), lsrc(nlo, -1), ucol(nup, -1), usrc(nup, -1), tslot(nlo, -1);
    for (int n = 0; n < N; n++) {
        if (old[n] < 0) continue;
        const int nl = row_of(n);
        for (int k = 0; k < (int)row.size(); k++) {
            const int s2 = k < nl ? lslot(n, k) : uslot(n, k - nl);
            (k < nl ? lcol : ucol)[s2] = row[k].first;
            (k < nl ? lsrc : usrc)[s2] = row[k].second;
        }
    }
    // the transpose of every lower block (n, j): the slot of n among j's upper blocks
    for (int n = 0; n < N; n++)
        for (int k = 0; k < lcnt[n]; k++) {
            const int s2 = lslot(n, k), jj = lcol[s2];
            int found = -1;
            for (int k2 = 0; k2 < ucnt[jj]; k2++)
                if (ucol[uslot(jj, k2)] == n) found = uslot(jj, k2);
            if (found < 0) return fail(SW2GPU_E_ARG, "the block pattern is not symmetric (D-ILU order)");
            tslot[s2] = found;
        }
    int mt = 1;
    for (int q = 0; q < ncol; q++) mt = std::max(mt, (pst[q + 1] - pst[q]) / 32);
    const int cap = dilu_capacity();
    if (cap <= 0) return fail(SW2GPU_E_CUDA, "the D-ILU solve kernel does not fit on this device");
    c->dilu = true;
    c->dl_ncol = ncol;
    c->dl_rows = N;
    c->dl_nlo = nlo;
    c->dl_nup = nup;
    c->dl_cta = std::max(1, std::min(cap, (mt + kDiluWarps - 1) / kDiluWarps));
    for (int q = 0; q <= kMaxColours; q++) {
        c->dl_cstart[q] = pst[std::min(q, ncol)];
        c->dl_cend[q] = q < ncol ? pst[q] + cnt[q] : N;
        c->dl_lbase[q] = q < ncol ? lbase[q] : nlo;
        c->dl_ubase[q] = q < ncol ? ubase[q] : nup;
        c->dl_lkn[q] = q < ncol ? lkn[q] : 0;
        c->dl_ukn[q] = q < ncol ? ukn[q] : 0;
    }
    int rc = 0;
    rc |= up(c->dl_lcol, lcol, st); rc |= up(c->dl_ucol, ucol, st);
    rc |= up(c->dl_lsrc, lsrc, st); rc |= up(c->dl_usrc, usrc, st);
    rc |= up(c->dl_tslot, tslot, st); rc |= up(c->dl_old, old, st);
    const size_t nval = 9ull * std::max(nlo + nup, 1);
    if (c->p.precision == SW2GPU_MIXED) rc |= zalloc(c->dl_blk32, nval, st);
    else rc |= zalloc(c->dl_blk64, nval, st);
    rc |= zalloc(c->dl_Dti, 9ull * N, st); rc |= zalloc(c->dl_Dd, 9ull * N, st);
    rc |= zalloc(c->dl_part, 8ull * c->dl_cta, st);
    for (auto& b : c->dl_vec) rc |= zalloc(b, 3ull * N, st);
    return rc;
}

// create with the mesh tables made by the caller (sw2gpu_remesh) or here (pre == nullptr)
int create_impl(const sw2gpu_mesh* m, const sw2gpu_params* prm, void* stream, MeshTables* pre, sw2gpu_ctx** out);

int sw2gpu_create(const sw2gpu_mesh* m, const sw2gpu_params* prm, void* stream, sw2gpu_ctx** out) {
    return create_impl(m, prm, stream, nullptr, out);
}

int create_impl(const sw2gpu_mesh* m, const sw2gpu_params* prm, void* stream, MeshTables* pre, sw2gpu_ctx** out) {
    if (!m || !prm || !out) return fail(SW2GPU_E_ARG, "null argument");
    *out = nullptr;
    if (m->nnodes <= 0 || m->nelems2d < 0 || m->nelems1d < 0) return fail(SW2GPU_E_ARG, "bad mesh sizes");
    if (prm->precision != SW2GPU_FP64 && prm->precision != SW2GPU_MIXED) return fail(SW2GPU_E_ARG, "bad precision");
    if (prm->precond != SW2GPU_PREC_BJACOBI && prm->precond != SW2GPU_PREC_BAND && prm->precond != SW2GPU_PREC_DILU)
        return fail(SW2GPU_E_ARG, "preconditioner %d not built (SW2GPU_PREC_BJACOBI, _BAND or _DILU)", prm->precond);
    if (prm->precond == SW2GPU_PREC_BAND && prm->precision != SW2GPU_FP64)
        return fail(SW2GPU_E_ARG, "the banded LU solve is FP64 only");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    auto* c = new sw2gpu_ctx();
    std::unique_ptr<sw2gpu_ctx> guard(c);
    struct Count {   // counts this context's device allocations
        explicit Count(size_t* b) { g_alloc_bytes = b; }
        ~Count() { g_alloc_bytes = nullptr; }
    } count(&c->bytes);
    c->p = *prm;
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    cudaStream_t st = c->stream;
    const int V = c->V = m->nnodes, T = c->T = m->nelems2d, E = c->E = m->nelems1d;
    c->S = m->nstrings;
    c->M = m->nmats;
    c->NS = m->nseries;
    const int* tri = m->elem2d_nodes;
    const int* edg = m->elem1d_nodes;
    for (int e = 0; e < T; e++)
        for (int i = 0; i < 3; i++)
            if (tri[3 * e + i] < 0 || tri[3 * e + i] >= V) return fail(SW2GPU_E_ARG, "element %d: node out of range", e);
    for (int e = 0; e < T; e++)
        if (m->elem2d_mat[e] < 0 || m->elem2d_mat[e] >= c->M || m->elem2d_mat[e] >= c->S)
            return fail(SW2GPU_E_ARG, "element %d: bad material", e);
    c->str_bc.assign(m->str_bc_flag, m->str_bc_flag + c->S);
    c->str_isigma.assign(m->str_isigma, m->str_isigma + c->S);
    c->str_ivx.assign(m->str_ivx, m->str_ivx + c->S);
    c->str_ivy.assign(m->str_ivy, m->str_ivy + c->S);
    c->str_iu0.assign(m->str_iu0, m->str_iu0 + c->S);

    // geometry (element_djac_nrml_gradPhi.c:193-273); kept in SoA arrays
    std::vector<double> djac(T), g[6];
    for (auto& a : g) a.resize(T);
    for (int e = 0; e < T; e++) {
        const int a = tri[3 * e], b = tri[3 * e + 1], cc = tri[3 * e + 2];
        const double s1x = m->x[b] - m->x[a], s1y = m->y[b] - m->y[a], s2x = m->x[cc] - m->x[a], s2y = m->y[cc] - m->y[a];
        const double cr = s1x * s2y - s2x * s1y;
        g[0][e] = (s1y - s2y) / cr;
        g[1][e] = (s2x - s1x) / cr;
        g[2][e] = s2y / cr;
        g[3][e] = -s2x / cr;
        g[4][e] = -s1y / cr;
        g[5][e] = s1x / cr;
        djac[e] = cr * 0.5;
        if (djac[e] < 1e-6) return fail(SW2GPU_E_ARG, "element %d is not counter-clockwise (djac %g)", e, djac[e]);
    }
    // boundary edges: length, outward normal (elem1d_outward_nrml.c), kind
    std::vector<double> bdj(E), bnx(E), bny(E);
    std::vector<int> bkind(E), bstr(E), bn0(E), bn1(E);
    for (int j = 0; j < E; j++) {
        const int a = edg[2 * j], b = edg[2 * j + 1], pe = m->elem1d_parent[j], s = m->elem1d_string[j];
        if (a < 0 || a >= V || b < 0 || b >= V || pe < 0 || pe >= T || s < 0 || s >= c->S)
            return fail(SW2GPU_E_ARG, "edge %d: bad node, parent or string", j);
        const double dx = m->x[b] - m->x[a], dy = m->y[b] - m->y[a], L = std::sqrt(dx * dx + dy * dy);
        double nx = dy / L, ny = -dx / L;
        const double cx = kOne3 * (m->x[tri[3 * pe]] + m->x[tri[3 * pe + 1]] + m->x[tri[3 * pe + 2]]);
        const double cy = kOne3 * (m->y[tri[3 * pe]] + m->y[tri[3 * pe + 1]] + m->y[tri[3 * pe + 2]]);
        if ((cx - m->x[a]) * nx + (cy - m->y[a]) * ny > 0.) { nx = -nx; ny = -ny; }
        bdj[j] = std::sqrt((m->x[a] - m->x[b]) * (m->x[a] - m->x[b]) + (m->y[a] - m->y[b]) * (m->y[a] - m->y[b]));
        bnx[j] = nx;
        bny[j] = ny;
        bn0[j] = a;
        bn1[j] = b;
        bstr[j] = s;
        const int f = c->str_bc[s];
        bkind[j] = f == SW2GPU_BCT_VEL_NEU ? 1 : f == SW2GPU_BCT_PRS_NEU ? 2 : f == SW2GPU_BCT_OUTFLOW ? 3
                 : f == SW2GPU_BCT_OVH_NEU ? 4 : 0;
        if (bkind[j] == 4) c->has_ovh = true;
        if (!bkind[j]) return fail(SW2GPU_E_ARG, "edge %d: boundary condition %d not supported", j, f);
    }
    // Dirichlet flags per node
    std::vector<unsigned char> dflag(V, 0);
    for (int n = 0; n < V; n++) {
        const int s = m->node_string[n];
        if (s >= c->S) return fail(SW2GPU_E_ARG, "node %d: bad string %d", n, s);
        if (s > SW2GPU_NORMAL) {
            const int f = c->str_bc[s];
            if (f == SW2GPU_BCT_LID_DFT || f == SW2GPU_BCT_LID_ELV || f == SW2GPU_BCT_LID_DEP)
                return fail(SW2GPU_E_ARG, "node %d: lid boundary condition %d (string %d) not supported", n, f, s);
            dflag[n] = f == SW2GPU_BCT_PRS_DIR ? 1 : f == SW2GPU_BCT_VEL_DIR ? 2 : f == SW2GPU_BCT_VEL_PRS_DIR ? 4 : 0;
            if (dflag[n]) {
                c->dir_node.push_back(n);
                c->dir_mask.push_back(f == SW2GPU_BCT_PRS_DIR ? 1 : f == SW2GPU_BCT_VEL_DIR ? 2 : 3);
                c->dir_str.push_back(s);
            }
        }
    }
    // first 2D element of every node (the dry-velocity side effect of fe_sw2_resid)
    std::vector<int> first(V, -1);
    std::vector<unsigned char> efirst(T, 0);
    for (int e = 0; e < T; e++)
        for (int i = 0; i < 3; i++) {
            const int n = tri[3 * e + i];
            if (first[n] < 0) first[n] = e;
            if (first[n] == e) efirst[e] |= (unsigned char)(1u << i);
        }
    // materials
    c->mats_h.resize(std::max(c->M, 1));
    for (int k = 0; k < c->M; k++) {
        MatParams& mp = c->mats_h[k];
        memset(&mp, 0, sizeof mp);
        mp.ks = (k < c->S) ? m->str_rough_height[k] : kUnsetFlt;
        mp.eev_mode = m->mat_eev_mode[k];
        mp.eev_coef = m->mat_eev_coef[k];
        const double xx = m->mat_ev[3 * k] + prm->viscosity, yy = m->mat_ev[3 * k + 1] + prm->viscosity;
        mp.ev_st = std::fabs(xx - yy);
        mp.ev_tr = std::min(xx, yy);
        mp.cor_speed = std::sin((kPi / 180.) * m->mat_coriolis[k]) * 2. * kEarthRotat;
        mp.has_source = (k < c->S && c->str_bc[k] == SW2GPU_BCT_WATER_SOURCE) ? 1 : 0;
    }
    // BCSR pattern and reference-order gather lists (sw2_tables.h)
    c->tri_h.assign(tri, tri + 3ull * T);
    c->edg_h.assign(edg, edg + 2ull * E);
    c->node_str_h.assign(m->node_string, m->node_string + V);
    c->edg_str_h.assign(m->elem1d_string, m->elem1d_string + E);
    if (pre) {
        c->tab = std::move(*pre);
    } else {
        const int tr = build_tables(V, T, E, tri, edg, c->tab);
        if (tr > 0) return fail(SW2GPU_E_ARG, "node %d belongs to no element", tr - 1);
    }
    if (c->tab.V != V || c->tab.T != T || c->tab.E != E) return fail(SW2GPU_E_ARG, "mesh tables of another mesh");
    const std::vector<int>& rp = c->tab.rp;
    const std::vector<int>& col = c->tab.col;
    const std::vector<int>& blk_row = c->tab.blk_row;
    const std::vector<int>& dpos = c->tab.dpos;
    const std::vector<int>& blk_ptr = c->tab.blk_ptr;
    const std::vector<int>& blk_src = c->tab.blk_src;
    const std::vector<int>& slot_ptr = c->tab.slot_ptr;
    const std::vector<int>& slot_idx = c->tab.slot_idx;
    const int nnzb = c->nnzb = (int)col.size();
    const size_t nsrc = 9ull * T + 4ull * E;
    const size_t nslot = 3ull * T + 2ull * E;
    // upload
    std::vector<double> xv(m->x, m->x + V), yv(m->y, m->y + V), zv(m->z, m->z + V);
    std::vector<int> e0(T), e1(T), e2(T), em(m->elem2d_mat, m->elem2d_mat + T);
    for (int e = 0; e < T; e++) { e0[e] = tri[3 * e]; e1[e] = tri[3 * e + 1]; e2[e] = tri[3 * e + 2]; }
    int rc = 0;
    rc |= up(c->x, xv, st); rc |= up(c->y, yv, st); rc |= up(c->z, zv, st);
    rc |= up(c->djac, djac, st);
    rc |= up(c->gx0, g[0], st); rc |= up(c->gy0, g[1], st); rc |= up(c->gx1, g[2], st);
    rc |= up(c->gy1, g[3], st); rc |= up(c->gx2, g[4], st); rc |= up(c->gy2, g[5], st);
    rc |= up(c->en0, e0, st); rc |= up(c->en1, e1, st); rc |= up(c->en2, e2, st); rc |= up(c->emat, em, st);
    rc |= up(c->efirst, efirst, st); rc |= up(c->dflag, dflag, st);
    rc |= up(c->bn0, bn0, st); rc |= up(c->bn1, bn1, st); rc |= up(c->bkind, bkind, st); rc |= up(c->bstr, bstr, st);
    rc |= up(c->bdjac, bdj, st); rc |= up(c->bnx, bnx, st); rc |= up(c->bny, bny, st);
    rc |= up(c->mats, c->mats_h, st);
    rc |= zalloc(c->str_value, std::max(c->S, 1), st);
    rc |= zalloc(c->str_uv, 2 * std::max(c->S, 1), st);
    rc |= zalloc(c->mass_part, 2 * kMassBlocks + 3, st);
    rc |= up(c->slot_ptr, slot_ptr, st); rc |= up(c->slot_idx, slot_idx, st);
    rc |= up(c->blk_ptr, blk_ptr, st); rc |= up(c->blk_src, blk_src, st);
    rc |= up(c->rowptr, rp, st); rc |= up(c->col, col, st); rc |= up(c->blk_row, blk_row, st); rc |= up(c->dpos, dpos, st);
    rc |= up(c->dir_node_d, c->dir_node, st); rc |= up(c->dir_mask_d, c->dir_mask, st);
    rc |= zalloc(c->dir_h, c->dir_node.size(), st); rc |= zalloc(c->dir_u, c->dir_node.size(), st);
    rc |= zalloc(c->dir_v, c->dir_node.size(), st);
    for (int l = 0; l < 3; l++) { rc |= zalloc(c->hs[l], V, st); rc |= zalloc(c->us[l], V, st); rc |= zalloc(c->vs[l], V, st); }
    rc |= zalloc(c->wd, std::max(T, 1), st);
    rc |= zalloc(c->ewet, std::max(T, 1), st);
    rc |= zalloc(c->glist, std::max(T, 1), st);
    rc |= zalloc(c->gcount, 1, st);
    rc |= zalloc(c->ngen, 1, st);
    rc |= zalloc(c->mark, V, st);
    rc |= zalloc(c->sc, nslot, st); rc |= zalloc(c->sx, nslot, st); rc |= zalloc(c->sy, nslot, st);
    rc |= zalloc(c->R, 3ull * V, st); rc |= zalloc(c->sol, 3ull * V, st);
    rc |= zalloc(c->jslots, nsrc * 9, st);
    rc |= zalloc(c->val, 9ull * nnzb, st);
    rc |= zalloc(c->S_, 3ull * V, st); rc |= zalloc(c->bs, 3ull * V, st);
    rc |= zalloc(c->dinv64, 9ull * V, st);
    const bool bjacobi = prm->precond == SW2GPU_PREC_BJACOBI;   // the folded operator and its vectors
    if (bjacobi && prm->precision == SW2GPU_MIXED)
        rc |= zalloc(c->aoff32, 9ull * (nnzb - V), st);
    else if (bjacobi)
        rc |= zalloc(c->aoff64, 9ull * (nnzb - V), st);
    {
        // the pattern without its diagonal (one diagonal block per row, checked above)
        std::vector<int>& orp = c->orowptr_h;
        orp.assign(V + 1, 0);
        std::vector<int> ocol;
        ocol.reserve(nnzb - V);
        for (int n = 0; n < V; n++) {
            for (int k = rp[n]; k < rp[n + 1]; k++)
                if (col[k] != n) ocol.push_back(col[k]);
            orp[n + 1] = (int)ocol.size();
        }
        rc |= up(c->orowptr, orp, st);
        rc |= up(c->ocol, ocol, st);
    }
    if (prm->precond == SW2GPU_PREC_BAND) {
        std::vector<int> perm;
        const int bwn = rcm_order(rp, col, V, perm);
        c->band = true;
        c->band_bw = 3 * bwn + 2;
        const size_t nb = (size_t)3 * V * (2 * (size_t)c->band_bw + 1) * sizeof(double);
        if (nb > kBandMaxBytes)
            return fail(SW2GPU_E_ARG, "the band of this system (%zu MB, half-width %d) exceeds the direct solve's %zu MB",
                        nb >> 20, c->band_bw, kBandMaxBytes >> 20);
        rc |= up(c->band_perm, perm, st);
        rc |= zalloc(c->band_mem, 3ull * V * (2ull * c->band_bw + 1), st);
        rc |= zalloc(c->band_y, 3ull * V, st);
    }
    if (prm->precond == SW2GPU_PREC_DILU && !rc) {
        const int r2 = build_dilu(c, rp, col, st);
        if (r2) return r2;
    }
    if (bjacobi)
        for (auto& b : c->kv64) rc |= zalloc(b, 3ull * V, st);
    rc |= zalloc(c->ncounter, 1, st);
    const int gblocks = nblk(V, kGatherThreads);
    rc |= zalloc(c->npart, gblocks, st);
    if (rc) return rc;
    // Krylov: the largest tile ranges (for the staged sweeps' stage layout) and the virtual
    // grid, which is the co-resident grid this instance gets alone (it fixes the order of
    // every Krylov reduction, so the instance's results do not depend on its batch)
    {
        const bool mixed = prm->precision == SW2GPU_MIXED;
        const unsigned esz = mixed ? sizeof(float) : sizeof(double);
        stage_caps(c->orowptr_h, V, esz, c->a_cap, c->c_cap);
    }
    CK(cudaMallocHost(&c->stage_h, sizeof(double) * stage_doubles(c)));
    CK(cudaEventCreateWithFlags(&c->stage_ev, cudaEventDisableTiming));
    std::vector<sw2gpu_ctx*> me(1, c);
    c->self.reset(new Runner());
    if ((rc = runner_init(*c->self, me, st))) return rc;
    // one virtual CTA per tile of kTileRows rows, at most kVirtualPerSM per SM: small meshes get
    // many CTAs when batched (a Krylov launch lasts as long as its slowest instance).  Fixed by
    // the device, not by the tuned occupancy: it sets the order of every Krylov reduction
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int ntiles = nblk(V, kTileRows);
    c->krylov_grid = std::max(1, std::min(ntiles, kVirtualPerSM * sms));
    if (zalloc(c->part, 8ull * c->krylov_grid, st)) return SW2GPU_E_NOMEM;
    DevMesh& d = c->dm;
    d.V = V; d.T = T; d.E = E; d.nnzb = nnzb;
    d.x = c->x.p; d.y = c->y.p; d.z = c->z.p;
    d.en0 = c->en0.p; d.en1 = c->en1.p; d.en2 = c->en2.p; d.emat = c->emat.p;
    d.djac = c->djac.p; d.gx0 = c->gx0.p; d.gy0 = c->gy0.p; d.gx1 = c->gx1.p; d.gy1 = c->gy1.p; d.gx2 = c->gx2.p;
    d.gy2 = c->gy2.p;
    d.efirst = c->efirst.p; d.dflag = c->dflag.p;
    d.bn0 = c->bn0.p; d.bn1 = c->bn1.p; d.bkind = c->bkind.p; d.bstr = c->bstr.p;
    d.bdjac = c->bdjac.p; d.bnx = c->bnx.p; d.bny = c->bny.p;
    d.mats = c->mats.p; d.str_value = c->str_value.p; d.str_uv = c->str_uv.p;
    d.slot_ptr = c->slot_ptr.p; d.slot_idx = c->slot_idx.p; d.blk_ptr = c->blk_ptr.p; d.blk_src = c->blk_src.p;
    d.rowptr = c->rowptr.p; d.col = c->col.p; d.blk_row = c->blk_row.p; d.dpos = c->dpos.p;
    for (int i = 0; i < 3; i++) d.qflag[i] = (i < V) ? dflag[i] : 0;
    CK(cudaStreamSynchronize(st));
    *out = guard.release();
    return SW2GPU_OK;
}

int64_t sw2gpu_device_bytes(const sw2gpu_ctx* c) { return c ? (int64_t)c->bytes : 0; }

int sw2gpu_destroy(sw2gpu_ctx* c) {
    if (!c) return SW2GPU_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    delete c;
    return SW2GPU_OK;
}

int sw2gpu_remesh(sw2gpu_ctx* old, const sw2gpu_mesh* m, sw2gpu_ctx** out) {
    if (!old || !m || !out) return fail(SW2GPU_E_ARG, "null argument");
    *out = nullptr;
    const int V = m->nnodes, T = m->nelems2d, E = m->nelems1d;
    if (V <= 0 || T < 0 || E < 0) return fail(SW2GPU_E_ARG, "bad mesh sizes");
    for (size_t q = 0; q < 3ull * T; q++)
        if (m->elem2d_nodes[q] < 0 || m->elem2d_nodes[q] >= V) return fail(SW2GPU_E_ARG, "element %zu: node out of range", q / 3);
    for (size_t q = 0; q < 2ull * E; q++)
        if (m->elem1d_nodes[q] < 0 || m->elem1d_nodes[q] >= V) return fail(SW2GPU_E_ARG, "edge %zu: node out of range", q / 2);
    // the tables: only the pattern rows the adaption touched are rebuilt (from scratch when the
    // mesh lost nodes)
    MeshTables t;
    int tr = update_tables(old->tab, old->tri_h.data(), old->edg_h.data(), V, T, E, m->elem2d_nodes, m->elem1d_nodes, t);
    if (tr < 0) tr = build_tables(V, T, E, m->elem2d_nodes, m->elem1d_nodes, t);
    if (tr > 0) return fail(SW2GPU_E_ARG, "node %d belongs to no element", tr - 1);
    sw2gpu_params prm = old->p;
    sw2gpu_ctx* c = nullptr;
    int rc = create_impl(m, &prm, (void*)old->stream, &t, &c);
    if (rc) return rc;
    // the new context takes over the stream and the settings
    c->own_stream = old->own_stream;
    old->own_stream = false;
    c->dt = old->dt;
    c->wait_barrier = old->wait_barrier;
    c->wait_copy = old->wait_copy;
    c->tune_jac_minb = old->tune_jac_minb;
    c->tune_stages = old->tune_stages;
    if (!rc && old->dacont_on) rc = sw2gpu_set_dacont(c, 1);
    if (!rc && old->mass_on) rc = sw2gpu_set_mass_tracking(c, 1, old->mass_density);
    if (!rc && (old->use_graphs || old->loop_graphs)) rc = sw2gpu_set_graphs(c, old->loop_graphs ? 2 : 1);
    if (!rc && old->ntrn) {
        if (c->S != old->S || c->M != old->M) {
            rc = fail(SW2GPU_E_ARG, "remesh: the constituents need the same strings and materials");
        } else {
            sw2gpu_transport spec{old->ntrn, old->trn_refc.data(), old->trn_dm_h.data(), old->trn_bc_h.data(),
                                  old->trn_ser_h.data()};
            rc = sw2gpu_set_transport(c, &spec);
        }
        // the concentration levels of the nodes both meshes have
        for (int k = 0; !rc && k < old->ntrn; k++) {
            c->trn_lv[k] = old->trn_lv[k];
            for (int l = 0; !rc && l < 3; l++)
                if (cudaMemcpyAsync(c->tconc.p + ((size_t)3 * k + l) * c->V, old->tconc.p + ((size_t)3 * k + l) * old->V,
                                    sizeof(double) * std::min(V, old->V), cudaMemcpyDeviceToDevice,
                                    c->stream) != cudaSuccess)
                    rc = fail(SW2GPU_E_CUDA, "copying the concentrations: %s", cudaGetErrorString(cudaGetLastError()));
        }
    }
    // the three time levels of the nodes both meshes have (node numbers are kept); new nodes start at 0
    const size_t nb = sizeof(double) * std::min(V, old->V);
    for (int l = 0; !rc && l < 3; l++) {
        if (cudaMemcpyAsync(c->H(l), old->H(l), nb, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess ||
            cudaMemcpyAsync(c->U(l), old->U(l), nb, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess ||
            cudaMemcpyAsync(c->Vv(l), old->Vv(l), nb, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
            rc = fail(SW2GPU_E_CUDA, "copying the time levels: %s", cudaGetErrorString(cudaGetLastError()));
    }
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = fail(SW2GPU_E_CUDA, "remesh: stream error");
    if (rc) {   // the old context keeps its stream and stays usable
        old->own_stream = c->own_stream;
        c->own_stream = false;
        delete c;
        return rc;
    }
    sw2gpu_destroy(old);
    *out = c;
    return SW2GPU_OK;
}

int sw2gpu_set_state(sw2gpu_ctx* c, int level, const double* h, const double* u, const double* v) {
    if (!c || level < 0 || level > 2) return fail(SW2GPU_E_ARG, "bad context or level");
    const size_t nb = sizeof(double) * c->V;
    if (h) CK(cudaMemcpyAsync(c->H(level), h, nb, cudaMemcpyHostToDevice, c->stream));
    if (u) CK(cudaMemcpyAsync(c->U(level), u, nb, cudaMemcpyHostToDevice, c->stream));
    if (v) CK(cudaMemcpyAsync(c->Vv(level), v, nb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_get_state(sw2gpu_ctx* c, int level, double* h, double* u, double* v) {
    if (!c || level < 0 || level > 2) return fail(SW2GPU_E_ARG, "bad context or level");
    const size_t nb = sizeof(double) * c->V;
    if (h) CK(cudaMemcpyAsync(h, c->H(level), nb, cudaMemcpyDeviceToHost, c->stream));
    if (u) CK(cudaMemcpyAsync(u, c->U(level), nb, cudaMemcpyDeviceToHost, c->stream));
    if (v) CK(cudaMemcpyAsync(v, c->Vv(level), nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_snapshot(sw2gpu_ctx* c, int level, double* d_h, double* d_u, double* d_v) {
    if (!c || level < 0 || level > 2) return fail(SW2GPU_E_ARG, "bad context or level");
    const size_t nb = sizeof(double) * c->V;
    if (d_h) CK(cudaMemcpyAsync(d_h, c->H(level), nb, cudaMemcpyDeviceToDevice, c->stream));
    if (d_u) CK(cudaMemcpyAsync(d_u, c->U(level), nb, cudaMemcpyDeviceToDevice, c->stream));
    if (d_v) CK(cudaMemcpyAsync(d_v, c->Vv(level), nb, cudaMemcpyDeviceToDevice, c->stream));
    return SW2GPU_OK;
}

int sw2gpu_get_wd_flag(sw2gpu_ctx* c, int32_t* wd) {
    if (!c || !wd) return fail(SW2GPU_E_ARG, "null argument");
    if (c->T) CK(cudaMemcpyAsync(wd, c->wd.p, sizeof(int) * c->T, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_set_wd_flag(sw2gpu_ctx* c, const int32_t* wd) {
    if (!c || !wd) return fail(SW2GPU_E_ARG, "null argument");
    if (c->T) CK(cudaMemcpyAsync(c->wd.p, wd, sizeof(int) * c->T, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

// Mass-balance diagnostics (src/tools/tl_grid_mass.c): one fixed-grid partial pass and one
// block adding the partials in order
static int mass_reduce(sw2gpu_ctx* c, bool flux, const double* h, double density, double* out) {
    double* part = c->mass_part.p;
    double* res = part + 2 * kMassBlocks;
    if (flux) {
        k_mass_partial<true><<<kMassBlocks, kMassThreads, 0, c->stream>>>(c->dm, h, c->U(0), c->Vv(0), c->dt, density,
                                                                          part);
        CK(cudaGetLastError());
        k_mass_final<true><<<1, kMassThreads, 0, c->stream>>>(part, density, res);
    } else {
        k_mass_partial<false><<<kMassBlocks, kMassThreads, 0, c->stream>>>(c->dm, h, nullptr, nullptr, 0.0, density,
                                                                           part);
        CK(cudaGetLastError());
        k_mass_final<false><<<1, kMassThreads, 0, c->stream>>>(part, density, res);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_grid_mass(sw2gpu_ctx* c, int level, double density, double* mass) {
    if (!c || !mass || level < 0 || level > 2) return fail(SW2GPU_E_ARG, "bad context, level or output");
    return mass_reduce(c, false, c->H(level), density, mass);
}

int sw2gpu_mass_flux(sw2gpu_ctx* c, double density, double* flux) {
    if (!c || !flux) return fail(SW2GPU_E_ARG, "bad context or output");
    if (!(c->dt > 0.0)) return fail(SW2GPU_E_ARG, "no step taken yet (dt unset)");
    return mass_reduce(c, true, c->H(0), density, flux);
}

// The element surface stress (wind + waves) the residual kernels read, after either part changed;
// captured step graphs hold the mesh descriptor, so they are dropped when the stress turns on or off.
int update_surface_stress(sw2gpu_ctx* c) {
    const bool on = c->wind_on || c->wave_on, was = c->dm.wsx != nullptr;
    const int T = c->T;
    if (on) {
        if (!c->stress.p) {
            g_alloc_bytes = &c->bytes;
            const int rc = zalloc(c->stress, 2 * (size_t)T, c->stream);
            g_alloc_bytes = nullptr;
            if (rc) return rc;
        }
        if (T) {
            k_surface_stress<<<nblk(2 * T, 256), 256, 0, c->stream>>>(T, c->wind_on ? c->wind.p : nullptr,
                                                                     c->wave_on ? c->wave.p : nullptr, c->stress.p);
            CK(cudaGetLastError());
        }
        c->dm.wsx = c->stress.p;
        c->dm.wsy = c->stress.p + T;
    } else {
        c->dm.wsx = c->dm.wsy = nullptr;
    }
    if (on != was) c->drop_graphs();
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_set_wind(sw2gpu_ctx* c, const int32_t* mat_flag, const double* mat_windatt, const double* stress_x,
                    const double* stress_y) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    if (!stress_x || !stress_y) {   // off
        c->wind_on = false;
        return update_surface_stress(c);
    }
    if (!mat_flag || !mat_windatt) return fail(SW2GPU_E_ARG, "null material wind tables");
    const int T = c->T, V = c->V, M = std::max(c->M, 1);
    std::vector<double> fac(M, 0.0);
    std::vector<int> flag(M, 0);
    for (int k = 0; k < c->M; k++) {
        if (mat_flag[k] != 0 && mat_flag[k] != 1)
            return fail(SW2GPU_E_ARG, "material %d: wind stress flag %d not supported (0 or 1)", k, mat_flag[k]);
        flag[k] = mat_flag[k];
        fac[k] = std::pow(mat_windatt[k], 2.0) / (3 * c->p.density);   // smeteor.c:302-303
    }
    if (!c->wind.p) {
        g_alloc_bytes = &c->bytes;
        int rc = zalloc(c->wind, 2 * (size_t)T + 2 * (size_t)V + M, c->stream);
        if (!rc) rc = zalloc(c->wind_flag, M, c->stream);
        g_alloc_bytes = nullptr;
        if (rc) return rc;
    }
    double* wsx = c->wind.p;
    double* wsy = wsx + T;
    double* nsx = wsy + T;
    double* nsy = nsx + V;
    double* fd = nsy + V;
    CK(cudaMemcpyAsync(nsx, stress_x, sizeof(double) * V, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(nsy, stress_y, sizeof(double) * V, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(fd, fac.data(), sizeof(double) * M, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->wind_flag.p, flag.data(), sizeof(int) * M, cudaMemcpyHostToDevice, c->stream));
    if (T) {
        k_elem_wind<<<nblk(T, 256), 256, 0, c->stream>>>(c->dm, c->p.gravity, c->p.density, c->wind_flag.p, fd, nsx, nsy,
                                                         wsx, wsy);
        CK(cudaGetLastError());
    }
    c->wind_on = true;
    return update_surface_stress(c);   // synchronizes: the host tables above are released on return
}

int sw2gpu_set_waves(sw2gpu_ctx* c, const double* rads_xx, const double* rads_xy, const double* rads_yy) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    if (!rads_xx || !rads_xy || !rads_yy) {   // off
        c->wave_on = false;
        return update_surface_stress(c);
    }
    const int T = c->T, V = c->V;
    if (!c->wave.p) {
        g_alloc_bytes = &c->bytes;
        const int rc = zalloc(c->wave, 2 * (size_t)T + 3 * (size_t)V, c->stream);
        g_alloc_bytes = nullptr;
        if (rc) return rc;
    }
    double* rads = c->wave.p + 2 * (size_t)T;
    CK(cudaMemcpyAsync(rads, rads_xx, sizeof(double) * V, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(rads + V, rads_xy, sizeof(double) * V, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(rads + 2 * (size_t)V, rads_yy, sizeof(double) * V, cudaMemcpyHostToDevice, c->stream));
    if (T) {
        k_elem_wave<<<nblk(T, 256), 256, 0, c->stream>>>(c->dm, rads, rads + V, rads + 2 * (size_t)V, c->wave.p);
        CK(cudaGetLastError());
    }
    c->wave_on = true;
    return update_surface_stress(c);
}

int sw2gpu_elem_error(sw2gpu_ctx* c, const double* refine_tol, double* elem_error, double* node_error) {
    if (!c || !refine_tol || !elem_error) return fail(SW2GPU_E_ARG, "null argument");
    if (!(c->dt > 0.0)) return fail(SW2GPU_E_ARG, "no step taken yet (dt unset)");
    const int T = c->T, V = c->V, M = std::max(c->M, 1);
    if (!c->errind.p) {
        g_alloc_bytes = &c->bytes;
        const int rc = zalloc(c->errind, 2 * (size_t)T + V + M, c->stream);
        g_alloc_bytes = nullptr;
        if (rc) return rc;
    }
    double* raw = c->errind.p;
    double* err = raw + T;
    double* nod = err + T;
    double* tol = nod + V;
    if (c->M) CK(cudaMemcpyAsync(tol, refine_tol, sizeof(double) * c->M, cudaMemcpyHostToDevice, c->stream));
    if (T) {
        k_elem_error<<<nblk(T, 256), 256, 0, c->stream>>>(c->dm, c->H(0), c->H(1), c->U(0), c->Vv(0), c->wd.p, c->dt,
                                                          tol, raw, err);
        CK(cudaGetLastError());
    }
    k_node_error<<<nblk(V, 256), 256, 0, c->stream>>>(c->dm, raw, nod);
    CK(cudaGetLastError());
    if (T) CK(cudaMemcpyAsync(elem_error, err, sizeof(double) * T, cudaMemcpyDeviceToHost, c->stream));
    if (node_error) CK(cudaMemcpyAsync(node_error, nod, sizeof(double) * V, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_set_mass_tracking(sw2gpu_ctx* c, int32_t enable, double density) {
    if (!c || (enable && !(density > 0.0))) return fail(SW2GPU_E_ARG, "bad context or density");
    if (enable && !c->mass_h) CK(cudaMallocHost(&c->mass_h, 2 * sizeof(double)));
    c->mass_on = enable != 0;
    c->mass_density = density;
    c->mass_valid = false;
    return SW2GPU_OK;
}

int sw2gpu_step_mass(sw2gpu_ctx* c, double* mass, double* flux) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    if (!c->mass_valid) return fail(SW2GPU_E_ARG, "no accepted step with mass tracking on since it was enabled");
    if (mass) *mass = c->step_mass;
    if (flux) *flux = c->step_flux;
    return SW2GPU_OK;
}

int sw2gpu_set_dacont(sw2gpu_ctx* c, int32_t enable) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    if (enable && !c->dacont.p) {
        g_alloc_bytes = &c->bytes;
        const int rc = zalloc(c->dacont, 3 * (size_t)c->T, c->stream);
        g_alloc_bytes = nullptr;
        if (rc) return rc;
        CK(cudaStreamSynchronize(c->stream));
    }
    c->dacont_on = enable != 0;
    c->drop_graphs();   // the residual launches change
    return SW2GPU_OK;
}

int sw2gpu_get_dacont(sw2gpu_ctx* c, double* out) {
    if (!c || !out) return fail(SW2GPU_E_ARG, "null argument");
    if (!c->dacont_on) return fail(SW2GPU_E_ARG, "transport side output not enabled (sw2gpu_set_dacont)");
    if (c->T) CK(cudaMemcpyAsync(out, c->dacont.p, sizeof(double) * 3 * c->T, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

// ---------------------------------------------------------------------------------------------
// constituent transport (fe_transport, src/fe/transport/fe_transport.c:31-113)

int sw2gpu_set_transport(sw2gpu_ctx* c, const sw2gpu_transport* t) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    if (!t || t->ntransport == 0) {
        c->ntrn = 0;
        return SW2GPU_OK;
    }
    const int n = t->ntransport, S = c->S, M = c->M, V = c->V, T = c->T, E = c->E;
    if (n < 0 || !t->ref_conc || (M && !t->diffusion) || (S && (!t->str_bc_flag || !t->str_series)))
        return fail(SW2GPU_E_ARG, "bad transport description");
    for (int k = 0; k < n; k++) {
        if (!(t->ref_conc[k] != 0.0) || !std::isfinite(t->ref_conc[k]))
            return fail(SW2GPU_E_ARG, "constituent %d: reference concentration must be finite and nonzero", k);
        for (int s = 0; s < S; s++) {
            const int f = t->str_bc_flag[k * S + s], q = t->str_series[k * S + s];
            if (f != 0 && f != SW2GPU_BCT_DIR && f != SW2GPU_BCT_NEU)
                return fail(SW2GPU_E_ARG, "constituent %d, string %d: bc flag %d not supported", k, s, f);
            if (f != 0 && (q < 0 || q >= c->NS))
                return fail(SW2GPU_E_ARG, "constituent %d, string %d: series %d out of range", k, s, q);
        }
        for (int j = 0; j < E; j++)
            if (t->str_bc_flag[k * S + c->edg_str_h[j]] == SW2GPU_BCT_DIR)
                return fail(SW2GPU_E_ARG, "constituent %d: DB TRN on edge string %d", k, c->edg_str_h[j]);
    }
    c->trn_refc.assign(t->ref_conc, t->ref_conc + n);
    c->trn_dm_h.assign((size_t)n * M, 0.0);
    if (M) std::copy(t->diffusion, t->diffusion + (size_t)n * M, c->trn_dm_h.begin());
    c->trn_bc_h.assign((size_t)n * S, 0);
    c->trn_ser_h.assign((size_t)n * S, -1);
    if (S) {
        std::copy(t->str_bc_flag, t->str_bc_flag + (size_t)n * S, c->trn_bc_h.begin());
        std::copy(t->str_series, t->str_series + (size_t)n * S, c->trn_ser_h.begin());
    }
    c->trn_lv.assign(n, std::array<int, 3>{0, 1, 2});
    cudaStream_t st = c->stream;
    g_alloc_bytes = &c->bytes;
    int rc = 0;
    if (c->ntrn != n || !c->tconc.p) rc |= zalloc(c->tconc, (size_t)3 * n * V, st);
    rc |= up(c->tbc, c->trn_bc_h, st);
    rc |= up(c->tdm, c->trn_dm_h, st);
    if (!c->tnode_str.p) {
        std::vector<int> ns(V, -1);
        for (int i = 0; i < V; i++) ns[i] = c->node_str_h[i] > SW2GPU_NORMAL ? c->node_str_h[i] : -1;
        rc |= up(c->tnode_str, ns, st);
        rc |= zalloc(c->tsval, std::max(S, 1), st);
        rc |= zalloc(c->tmask, V, st);
        rc |= zalloc(c->trslot, 3ull * T + 2ull * E, st);
        rc |= zalloc(c->tjslot, 9ull * T + 4ull * E, st);
        rc |= zalloc(c->tR, V, st);
        rc |= zalloc(c->tsol, V, st);
        rc |= zalloc(c->taoff, (size_t)(c->nnzb - V), st);
        rc |= zalloc(c->tdinv, V, st);
        for (auto& b : c->tkv) rc |= zalloc(b, V, st);
        rc |= zalloc(c->tnpart, nblk(V, kGatherThreads), st);
        rc |= zalloc(c->tnorms, 1, st);
        rc |= zalloc(c->tncount, 1, st);
        rc |= zalloc(c->tctl, 1, st);
        int dev = 0, sms = 0, per_sm = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trn_bicgstab<kTrnKThreads>, kTrnKThreads, 0));
        // at most the co-resident CTAs (a cooperative launch), at least 512 rows each
        c->trn_kgrid = std::max(1, std::min(sms * std::max(per_sm, 1), V / 512));
        if (per_sm < 1) return fail(SW2GPU_E_CUDA, "the transport Krylov kernel does not fit on an SM");
        rc |= zalloc(c->tkpart, 12ull * c->trn_kgrid, st);
        if (!c->tnorms_h) CK(cudaMallocHost(&c->tnorms_h, sizeof(Norms)));
        if (!c->tctl_h) CK(cudaMallocHost(&c->tctl_h, sizeof(KrylovCtl)));
        if (!c->tsval_h) CK(cudaMallocHost(&c->tsval_h, sizeof(double) * std::max(S, 1)));
    }
    g_alloc_bytes = nullptr;
    if (rc) return rc;
    c->ntrn = n;
    if (!c->dacont_on && (rc = sw2gpu_set_dacont(c, 1))) return rc;   // the transport residual reads it
    CK(cudaStreamSynchronize(st));
    return SW2GPU_OK;
}

int sw2gpu_set_conc(sw2gpu_ctx* c, int32_t itrn, int32_t level, const double* conc) {
    if (!c || !conc || itrn < 0 || itrn >= c->ntrn || level < 0 || level > 2)
        return fail(SW2GPU_E_ARG, "bad context, constituent or level");
    CK(cudaMemcpyAsync(c->tlevel(itrn, level), conc, sizeof(double) * c->V, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_get_conc(sw2gpu_ctx* c, int32_t itrn, int32_t level, double* conc) {
    if (!c || !conc || itrn < 0 || itrn >= c->ntrn || level < 0 || level > 2)
        return fail(SW2GPU_E_ARG, "bad context, constituent or level");
    CK(cudaMemcpyAsync(conc, c->tlevel(itrn, level), sizeof(double) * c->V, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

namespace {

TrnArgs trn_args(sw2gpu_ctx* c, int k) {
    TrnArgs A{};
    A.m = c->dm;
    A.h = c->H(0);
    A.u = c->U(0);
    A.v = c->Vv(0);
    A.ho = c->H(1);
    A.hoo = c->H(2);
    A.wd = c->wd.p;
    A.dac = c->dacont.p;
    A.c = c->tlevel(k, 0);
    A.co = c->tlevel(k, 1);
    A.coo = c->tlevel(k, 2);
    A.node_str = c->tnode_str.p;
    A.tbc = c->tbc.p + (size_t)k * c->S;
    A.tsval = c->tsval.p;
    A.tdm = c->tdm.p + (size_t)k * c->M;
    A.refc = c->trn_refc[k];
    A.mask = c->tmask.p;
    A.rslot = c->trslot.p;
    A.jslot = c->tjslot.p;
    A.R = c->tR.p;
    A.sol = c->tsol.p;
    A.aoff = c->taoff.p;
    A.dinv = c->tdinv.p;
    A.val = nullptr;
    A.npart = c->tnpart.p;
    A.norms = c->tnorms.p;
    A.ncounter = c->tncount.p;
    A.P = TrnParams{c->p.gravity, c->p.drying_lower_limit, c->p.tau_temporal, c->p.tau_pg, c->dt};
    return A;
}

// step values of constituent k's string series over property[0] (DB TRN: fe_transport_init.c:93-100;
// NB TRN: fe_2d_transport_boundary_resid.c:194, :240)
int trn_upload_series(sw2gpu_ctx* c, int k, const double* series) {
    const double c_inv = 1. / c->trn_refc[k];
    for (int s = 0; s < c->S; s++) {
        const int f = c->trn_bc_h[(size_t)k * c->S + s], q = c->trn_ser_h[(size_t)k * c->S + s];
        c->tsval_h[s] = (f != 0 && q >= 0 && series) ? series[q] * c_inv : 0.0;
    }
    if (c->S) CK(cudaMemcpyAsync(c->tsval.p, c->tsval_h, sizeof(double) * c->S, cudaMemcpyHostToDevice, c->stream));
    return 0;
}

int trn_init(sw2gpu_ctx* c, const TrnArgs& A) {
    k_trn_init<<<nblk(c->V, kTrnThreads), kTrnThreads, 0, c->stream>>>(A);
    CK(cudaGetLastError());
    return 0;
}

// residual and its norms (fe_transport_resid + get_residual_norms); waits for them
int trn_resid(sw2gpu_ctx* c, const TrnArgs& A, Norms& out, int& launches) {
    k_trn_elem<false><<<nblk(c->T + c->E, kTrnThreads), kTrnThreads, 0, c->stream>>>(A);
    k_trn_resid_gather<<<nblk(c->V, kGatherThreads), kGatherThreads, 0, c->stream>>>(A);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->tnorms_h, c->tnorms.p, sizeof(Norms), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out = *c->tnorms_h;
    launches += 2;
    return 0;
}

// FD Jacobian and the folded operator (fe_transport_load)
int trn_load(sw2gpu_ctx* c, const TrnArgs& A, int& launches) {
    k_trn_elem<true><<<nblk(c->T + c->E, kTrnThreads), kTrnThreads, 0, c->stream>>>(A);
    k_trn_jac_gather<<<nblk(c->V, kTrnThreads), kTrnThreads, 0, c->stream>>>(A);
    CK(cudaGetLastError());
    launches += 2;
    return 0;
}

// the Krylov solve of the folded system into tsol; its outcome lands in tctl_h at the next sync
int trn_krylov(sw2gpu_ctx* c, int& launches) {
    TrnKrylovArgs K{};
    K.V = c->V;
    K.orowptr = c->orowptr.p;
    K.ocol = c->ocol.p;
    K.aoff = c->taoff.p;
    K.dinv = c->tdinv.p;
    K.R = c->tR.p;
    K.x = c->tsol.p;
    for (int q = 0; q < kTrnKVectors; q++) K.vec[q] = c->tkv[q].p;
    K.part = c->tkpart.p;
    K.ctl = c->tctl.p;
    // the reference solves each transport system exactly (its profile LU preconditioner makes
    // BiCGSTAB converge in one iteration) and its Newton rule then stops after one iteration
    // whenever the residual falls below tol_nonlin; a relative 1e-12 keeps the device's answer
    // at the exact solve's
    K.rtol = std::min(c->p.lin_rtol, kTrnKrylovRtol);
    K.atol = c->p.lin_atol;
    K.max_it = c->p.max_lin_it;
    K.spin_limit = c->wait_barrier;
    CK(cudaMemsetAsync(c->tctl.p, 0, sizeof(KrylovCtl), c->stream));
    void* args[] = {&K};
    CK(cudaLaunchCooperativeKernel((void*)k_trn_bicgstab<kTrnKThreads>, dim3(c->trn_kgrid), dim3(kTrnKThreads), args, 0,
                                   c->stream));
    CK(cudaMemcpyAsync(c->tctl_h, c->tctl.p, sizeof(KrylovCtl), cudaMemcpyDeviceToHost, c->stream));
    launches += 1;
    return 0;
}

int trn_inc(sw2gpu_ctx* c, int k, int mode, int& launches) {
    k_trn_inc<<<nblk(c->V, kTrnThreads), kTrnThreads, 0, c->stream>>>(c->tlevel(k, 0), c->tsol.p, c->V, mode);
    CK(cudaGetLastError());
    launches += 1;
    return 0;
}

// fe_transport for constituent k (fe_transport.c:58-74): level shift, fe_transport_init, then
// fe_newton with the transport functions, whose linear-problem test keeps iterating while the
// residual max norm exceeds tol_nonlin (fe_newton.c:817-823, :855-856)
int trn_step_one(sw2gpu_ctx* c, int k, const double* series, sw2gpu_stats* st) {
    const sw2gpu_params& P = c->p;
    auto& lv = c->trn_lv[k];
    const int o2 = lv[2];
    lv[2] = lv[1];
    lv[1] = lv[0];
    lv[0] = o2;
    int rc, launches = 0;
    // phase timers: event pairs around the Jacobian (0), Krylov (1) and residual (2) launches
    std::vector<cudaEvent_t> evs;
    std::vector<int> kinds;
    auto ev = [&]() -> cudaEvent_t {   // pushed even when creation failed: pairs stay in step
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) e = nullptr;
        evs.push_back(e);
        return e;
    };
    auto phase_begin = [&](int kind) {
        kinds.push_back(kind);
        cudaEvent_t e = ev();
        if (e) cudaEventRecord(e, c->stream);
    };
    auto phase_end = [&]() {
        cudaEvent_t e = ev();
        if (e) cudaEventRecord(e, c->stream);
    };
    struct Release {
        std::vector<cudaEvent_t>& v;
        ~Release() {
            for (cudaEvent_t e : v)
                if (e) cudaEventDestroy(e);
        }
    } release{evs};
    cudaEvent_t e0 = ev(), e1 = nullptr;
    if (!e0) return fail(SW2GPU_E_CUDA, "cudaEventCreate failed");
    CK(cudaEventRecord(e0, c->stream));
    if ((rc = trn_upload_series(c, k, series))) return rc;
    const TrnArgs A = trn_args(c, k);
    CK(cudaMemsetAsync(c->tsol.p, 0, sizeof(double) * c->V, c->stream));
    if ((rc = trn_init(c, A))) return rc;
    launches++;
    Norms nr{};
    phase_begin(2);
    auto resid = [&](Norms& out) {   // the residual phase ends before its host wait
        k_trn_elem<false><<<nblk(c->T + c->E, kTrnThreads), kTrnThreads, 0, c->stream>>>(A);
        k_trn_resid_gather<<<nblk(c->V, kGatherThreads), kGatherThreads, 0, c->stream>>>(A);
        phase_end();
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(c->tnorms_h, c->tnorms.p, sizeof(Norms), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        out = *c->tnorms_h;
        launches += 2;
        return 0;
    };
    if ((rc = resid(nr))) return rc;
    const bool lin_test = P.tol_nonlin > kSmall;
    int it = 0, lin_total = 0, cuts_total = 0, status = SW2GPU_OK;
    bool solv_ok = true, nan_flag = false, timeout = false;
    double rl2 = sqrt(nr.l2sum / c->V);
    for (;;) {
        phase_begin(0);
        if ((rc = trn_load(c, A, launches))) return rc;
        phase_end();
        phase_begin(1);
        if ((rc = trn_krylov(c, launches))) return rc;
        phase_end();
        if ((rc = trn_inc(c, k, 0, launches))) return rc;
        const double old_l2 = rl2;
        phase_begin(2);
        if ((rc = resid(nr))) return rc;   // also brings the Krylov outcome
        const KrylovCtl kc = *c->tctl_h;
        if (kc.err) {
            timeout = true;
            break;
        }
        lin_total += kc.iterations;
        if (!kc.converged) solv_ok = false;
        rl2 = sqrt(nr.l2sum / c->V);
        if (std::isnan(rl2) || std::isinf(rl2)) {
            solv_ok = false;
            nan_flag = true;
        }
        int cuts = 0;
        while (nr.rmax > P.tol_nonlin && rl2 > old_l2 && cuts < P.max_linesearch_cuts) {
            if ((rc = trn_inc(c, k, 1, launches))) return rc;
            phase_begin(2);
            if ((rc = resid(nr))) return rc;
            rl2 = sqrt(nr.l2sum / c->V);
            cuts++;
        }
        cuts_total += cuts;
        it++;
        const bool keep = solv_ok && it < P.max_nonlin_it && nr.rmax < 1.0E+20 && (lin_test && nr.rmax > P.tol_nonlin);
        if (!keep) break;
    }
    if (timeout) status = SW2GPU_E_TIMEOUT;
    else if (!solv_ok || (lin_test && nr.rmax > P.tol_nonlin) || nr.rmax >= 1.0E+20)
        status = nan_flag ? SW2GPU_E_NAN : (!solv_ok ? SW2GPU_E_LINEAR : SW2GPU_E_NEWTON);
    if (status != SW2GPU_OK) {   // reset to the old level (fe_newton.c:883)
        if ((rc = trn_init(c, A))) return rc;
        launches++;
    }
    e1 = ev();
    if (!e1) return fail(SW2GPU_E_CUDA, "cudaEventCreate failed");
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    double ph[3] = {0.0, 0.0, 0.0};
    for (size_t q = 0; q < kinds.size(); q++) {   // pairs follow e0 in the event list
        float t = 0.f;
        if (2 + 2 * q < evs.size() && evs[1 + 2 * q] && evs[2 + 2 * q] &&
            cudaEventElapsedTime(&t, evs[1 + 2 * q], evs[2 + 2 * q]) == cudaSuccess)
            ph[kinds[q]] += t;
    }
    if (st) {
        memset(st, 0, sizeof(*st));
        st->status = status;
        st->newton_its = it;
        st->linear_its = lin_total;
        st->linesearch_cuts = cuts_total;
        st->resid_max = nr.rmax;
        st->resid_l2 = rl2;
        st->inc_max = nr.imax;
        st->device_ms = ms;
        st->kernel_launches = launches;
        st->jac_ms = ph[0];
        st->krylov_ms = ph[1];
        st->resid_ms = ph[2];
        st->other_ms = ms - ph[0] - ph[1] - ph[2];
    }
    return status;
}

}  // namespace

int sw2gpu_transport_step(sw2gpu_ctx* c, const double* series, sw2gpu_stats* stats) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    if (!c->ntrn) return fail(SW2GPU_E_ARG, "no constituents (sw2gpu_set_transport)");
    if (!(c->dt > 0.0)) return fail(SW2GPU_E_ARG, "no flow step yet (dt unset)");
    for (int k = 0; k < c->ntrn; k++) {
        const int rc = trn_step_one(c, k, series, stats ? stats + k : nullptr);
        if (rc) {
            if (rc == SW2GPU_E_NEWTON || rc == SW2GPU_E_LINEAR || rc == SW2GPU_E_NAN || rc == SW2GPU_E_TIMEOUT)
                return fail(rc, "transport of constituent %d did not converge (status %d)", k, rc);
            return rc;
        }
    }
    return SW2GPU_OK;
}

int sw2gpu_transport_init(sw2gpu_ctx* c, int32_t itrn, const double* series) {
    if (!c || itrn < 0 || itrn >= c->ntrn) return fail(SW2GPU_E_ARG, "bad context or constituent");
    int rc;
    if ((rc = trn_upload_series(c, itrn, series))) return rc;
    if ((rc = trn_init(c, trn_args(c, itrn)))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_transport_load(sw2gpu_ctx* c, int32_t itrn, double* resid, double* val) {
    if (!c || itrn < 0 || itrn >= c->ntrn) return fail(SW2GPU_E_ARG, "bad context or constituent");
    DBuf<double> full;
    if (val && full.alloc(c->nnzb)) return fail(SW2GPU_E_NOMEM, "cudaMalloc failed");
    TrnArgs A = trn_args(c, itrn);
    Norms nr{};
    int launches = 0, rc;
    if ((rc = trn_resid(c, A, nr, launches))) return rc;
    A.val = val ? full.p : nullptr;
    if ((rc = trn_load(c, A, launches))) return rc;
    if (resid) CK(cudaMemcpyAsync(resid, c->tR.p, sizeof(double) * c->V, cudaMemcpyDeviceToHost, c->stream));
    if (val) CK(cudaMemcpyAsync(val, full.p, sizeof(double) * c->nnzb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_transport_elem_error(sw2gpu_ctx* c, const double* refine_tol, double* elem_error, double* node_error) {
    if (!c || !refine_tol || !elem_error) return fail(SW2GPU_E_ARG, "null argument");
    if (!c->ntrn) return fail(SW2GPU_E_ARG, "no constituents (sw2gpu_set_transport)");
    if (!(c->dt > 0.0)) return fail(SW2GPU_E_ARG, "no step yet (dt unset)");
    for (int q = 0; q < c->ntrn * c->M; q++)
        if (!(refine_tol[q] > 0.0)) return fail(SW2GPU_E_ARG, "refine tolerance %d must be positive", q);
    const int T = c->T, V = c->V, M = c->M;
    DBuf<double> elem, raw, tol, nodal;
    if (elem.alloc(T) || raw.alloc(T) || tol.alloc(std::max(M, 1)) || nodal.alloc(V))
        return fail(SW2GPU_E_NOMEM, "cudaMalloc failed");
    cudaStream_t st = c->stream;
    CK(cudaMemcpyAsync(elem.p, elem_error, sizeof(double) * T, cudaMemcpyHostToDevice, st));
    for (int k = 0; k < c->ntrn; k++) {
        CK(cudaMemcpyAsync(tol.p, refine_tol + (size_t)k * M, sizeof(double) * M, cudaMemcpyHostToDevice, st));
        k_trn_elem_error<<<nblk(T, kTrnThreads), kTrnThreads, 0, st>>>(c->dm, c->H(0), c->U(0), c->Vv(0),
                                                                        c->tlevel(k, 0), c->tlevel(k, 1), c->dt,
                                                                        tol.p, raw.p, elem.p);
        if (node_error) {   // the raw values averaged over each node's elements, in element order
            k_node_error<<<nblk(V, 256), 256, 0, st>>>(c->dm, raw.p, nodal.p);
            CK(cudaMemcpyAsync(node_error + (size_t)k * V, nodal.p, sizeof(double) * V, cudaMemcpyDeviceToHost, st));
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));   // tol is rewritten for the next constituent
    }
    CK(cudaMemcpyAsync(elem_error, elem.p, sizeof(double) * T, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SW2GPU_OK;
}

int sw2gpu_set_dt(sw2gpu_ctx* c, double dt, const double* series) {
    if (!c || !(dt > 0.0)) return fail(SW2GPU_E_ARG, "bad context or dt");
    c->dt = dt;
    return upload_step_tables(c, series, c->stream);
}

int sw2gpu_resid(sw2gpu_ctx* c, double* resid) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    Runner& R = *c->self;
    const std::vector<int> one(1, 0);
    int rc = runner_tables(R, 1);
    if (!rc) rc = launch_resid(R, one);
    if (!rc) rc = read_results(R, one);
    if (rc) return rc;
    if (resid) CK(cudaMemcpyAsync(resid, c->R.p, sizeof(double) * 3 * c->V, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_load(sw2gpu_ctx* c, int32_t* nnzb, int32_t* row_ptr, int32_t* col, double* val, double* resid) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    if (nnzb) *nnzb = c->nnzb;
    if (!val && !resid && !row_ptr && !col) return SW2GPU_OK;
    Runner& R = *c->self;
    const std::vector<int> one(1, 0);
    int rc = runner_tables(R, 1);
    if (rc) return rc;
    // element classification for the two Jacobian kernels (sw2gpu_step takes it from the
    // residual pass at the same state); R is the last sw2gpu_resid's, as in fe_newton
    if ((rc = launch_map(R, one, 256, [&](int) { return nblk(c->T, 256); }, SW2_GO(k_classify<std::decay_t<decltype(src)>>)))) return rc;
    CK(cudaMemcpyAsync(&R.norms.p[0].ngeneral, c->gcount.p, sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->ngen.p, c->gcount.p, sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemsetAsync(c->gcount.p, 0, sizeof(int), c->stream));
    if ((rc = read_results(R, one))) return rc;
    if ((rc = launch_jacobian(R, one))) return rc;
    if ((rc = launch_map(R, one, 256, [&](int) { return nblk(c->V, 256); }, SW2_GO(k_rowscale<std::decay_t<decltype(src)>>, 1)))) return rc;
    if (row_ptr) memcpy(row_ptr, c->rowptr_h.data(), sizeof(int) * (c->V + 1));
    if (col) memcpy(col, c->col_h.data(), sizeof(int) * c->nnzb);
    if (val) CK(cudaMemcpyAsync(val, c->val.p, sizeof(double) * 9 * (size_t)c->nnzb, cudaMemcpyDeviceToHost, c->stream));
    if (resid) CK(cudaMemcpyAsync(resid, c->R.p, sizeof(double) * 3 * c->V, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SW2GPU_OK;
}

int sw2gpu_linear_solve(sw2gpu_ctx* c, const double* val, const double* rhs, double* x, int32_t* iterations) {
    if (!c || !val || !rhs || !x) return fail(SW2GPU_E_ARG, "null argument");
    Runner& R = *c->self;
    const std::vector<int> one(1, 0);
    CK(cudaMemcpyAsync(c->val.p, val, sizeof(double) * 9 * (size_t)c->nnzb, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->R.p, rhs, sizeof(double) * 3 * c->V, cudaMemcpyHostToDevice, c->stream));
    int rc = runner_tables(R, 0);
    if (!rc) rc = launch_linear(R, one, std::vector<double>(1, c->p.lin_rtol));
    if (rc) return rc;
    CK(cudaMemcpyAsync(x, c->sol.p, sizeof(double) * 3 * c->V, cudaMemcpyDeviceToHost, c->stream));
    if ((rc = read_results(R, {}))) return rc;
    const KrylovCtl& q = R.ctl_h[0];
    if (iterations) *iterations = q.iterations;
    if (q.err) return fail(SW2GPU_E_TIMEOUT, "Krylov barrier or tile-copy wait ran out");
    return q.converged ? SW2GPU_OK : fail(SW2GPU_E_LINEAR, "BiCGSTAB reached max_lin_it");
}

int sw2gpu_set_variant(sw2gpu_ctx* c, int32_t jac_minb, int32_t stages) {
    if (!c || (jac_minb != 1 && jac_minb != 2) || (stages != 0 && stages != 2 && stages != 3))
        return fail(SW2GPU_E_ARG, "variant: jac_minb 1|2, stages 0|2|3");
    c->tune_jac_minb = jac_minb;
    c->tune_stages = stages;
    c->drop_graphs();
    return runner_set(*c->self, c->self->ctx);
}

int sw2gpu_get_variant(const sw2gpu_ctx* c, int32_t* jac_minb, int32_t* stages) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    if (jac_minb) *jac_minb = c->self->jac_minb;
    if (stages) *stages = c->self->stages;
    return SW2GPU_OK;
}

// Times every launch variant on the context's own mesh and current state and keeps the
// fastest: the wet-Jacobian register budget (1 or 2 CTAs per SM) and the Krylov tile-ring
// depth (0, 2 or 3 stages).  The variants compute the same bits; the state is left as found.
int sw2gpu_autotune(sw2gpu_ctx* c, int32_t* jac_minb, int32_t* stages) {
    if (!c) return fail(SW2GPU_E_ARG, "null context");
    Runner& R = *c->self;
    const std::vector<int> one(1, 0);
    const size_t nb = sizeof(double) * c->V;
    cudaStream_t st = R.stream;
    // the residual zeroes old-dry nodes' velocities of the current level: keep a copy (on the
    // host -- every device work array is written by the kernels being timed)
    std::vector<double> keep(2 * (size_t)c->V);
    CK(cudaMemcpyAsync(keep.data(), c->U(0), nb, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(keep.data() + c->V, c->Vv(0), nb, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int rc = runner_tables(R, 0);
    if (!rc) rc = launch_resid(R, one);
    if (!rc) rc = read_results(R, one);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto timed = [&](auto&& fn, float& best) -> int {
        int r = fn();   // warm
        if (r) return r;
        for (int rep = 0; rep < 2; rep++) {
            CK(cudaEventRecord(e0, st));
            if ((r = fn())) return r;
            CK(cudaEventRecord(e1, st));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        return 0;
    };
    int best_j = c->tune_jac_minb;
    float tb = 1e30f;
    for (int m : {1, 2}) {
        if (!R.jac_ctas[m - 1]) continue;   // does not fit on this device
        R.jac_minb = m;
        float t = 1e30f;
        if ((rc = timed([&] { return launch_jacobian(R, one); }, t))) break;
        if (t < tb) { tb = t; best_j = m; }
    }
    c->tune_jac_minb = best_j;
    int best_s = c->tune_stages;
    tb = 1e30f;
    const std::vector<double> eta(1, c->p.lin_rtol);
    for (int sg : {0, 2, 3}) {
        if (rc) break;
        c->tune_stages = sg;
        if ((rc = runner_set(R, R.ctx))) break;
        if (R.stages != sg) continue;   // this mesh's tiles do not fit that ring
        float t = 1e30f;
        if ((rc = timed([&] { return launch_linear(R, one, eta); }, t))) break;
        if (t < tb) { tb = t; best_s = sg; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tune_stages = best_s;
    c->drop_graphs();
    if (!rc) rc = runner_set(R, R.ctx);
    CK(cudaMemcpyAsync(c->U(0), keep.data(), nb, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->Vv(0), keep.data() + c->V, nb, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    if (rc) return rc;
    if (jac_minb) *jac_minb = R.jac_minb;
    if (stages) *stages = R.stages;
    return SW2GPU_OK;
}

int sw2gpu_set_wait_limits(sw2gpu_ctx* c, int64_t barrier_polls, int64_t copy_polls) {
    if (!c || barrier_polls < 0 || copy_polls < 0) return fail(SW2GPU_E_ARG, "bad context or wait limit");
    c->wait_barrier = barrier_polls;
    c->wait_copy = copy_polls;
    c->drop_graphs();   // the limits travel in the Krylov launch's parameters
    return SW2GPU_OK;
}

int sw2gpu_set_graphs(sw2gpu_ctx* c, int32_t enable) {
    if (!c || enable < 0 || enable > 2) return fail(SW2GPU_E_ARG, "bad context or graph mode");
    c->drop_graphs();
    c->use_graphs = enable == 1;
    c->loop_graphs = enable == 2;
    return SW2GPU_OK;
}

int sw2gpu_step(sw2gpu_ctx* c, double dt, const double* series, sw2gpu_stats* stats) {
    if (!c || !(dt > 0.0)) return fail(SW2GPU_E_ARG, "bad context or dt");
    const double* ser[1] = {series};
    int status = 0;
    int rc = c->loop_graphs  ? loop_step(c, dt, ser[0], stats, &status)
             : c->use_graphs ? graph_step(c, dt, ser[0], stats, &status)
                             : runner_step(*c->self, &dt, ser, stats, &status);
    if (rc) return rc;
    if (status != SW2GPU_OK)
        fail(status, "step failed (Newton %d iterations, max residual %g)", stats ? stats->newton_its : -1,
             stats ? stats->resid_max : 0.0);
    return status;
}

int sw2gpu_batch_create(sw2gpu_ctx** ctxs, int32_t n, void* stream, sw2gpu_batch** out) {
    if (!ctxs || n <= 0 || !out) return fail(SW2GPU_E_ARG, "bad batch arguments");
    if (n > kMaxBatch) return fail(SW2GPU_E_ARG, "batch of %d instances exceeds %d", n, kMaxBatch);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++)
            if (ctxs[i] == ctxs[j] || !ctxs[i]) return fail(SW2GPU_E_ARG, "batch instance %d repeated or null", i);
    *out = nullptr;
    auto* b = new sw2gpu_batch();
    std::unique_ptr<sw2gpu_batch> guard(b);
    b->run.reset(new Runner());
    cudaStream_t st = (cudaStream_t)stream;
    bool own = false;
    if (!st) {
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        own = true;
    }
    b->own_stream = own;
    int rc = runner_init(*b->run, std::vector<sw2gpu_ctx*>(ctxs, ctxs + n), st);
    if (rc) {
        if (own) cudaStreamDestroy(st);
        return rc;
    }
    *out = guard.release();
    return SW2GPU_OK;
}

int sw2gpu_batch_step(sw2gpu_batch* b, const double* dt, const double* const* series, sw2gpu_stats* stats) {
    if (!b || !dt) return fail(SW2GPU_E_ARG, "bad batch arguments");
    const int K = (int)b->run->ctx.size();
    std::vector<int> status(K, 0);
    std::vector<sw2gpu_stats> st(K);
    // instances' own streams may still hold work (state uploads): order it before the batch
    for (auto* c : b->run->ctx) CK(cudaStreamSynchronize(c->stream));
    int rc = runner_step(*b->run, dt, series, stats ? stats : st.data(), status.data());
    if (rc) return rc;
    for (int k = 0; k < K; k++)
        if (status[k] != SW2GPU_OK) return fail(status[k], "instance %d: step failed", k);
    return SW2GPU_OK;
}

int sw2gpu_batch_set_graphs(sw2gpu_batch* b, int32_t enable) {
    if (!b) return fail(SW2GPU_E_ARG, "null batch");
    b->run->use_graphs = enable != 0;
    if (!enable) b->run->drop_batch_graphs();
    return SW2GPU_OK;
}

int sw2gpu_batch_destroy(sw2gpu_batch* b) {
    if (!b) return SW2GPU_OK;
    cudaStream_t st = b->run->stream;
    cudaStreamSynchronize(st);
    b->run.reset();
    if (b->own_stream) cudaStreamDestroy(st);
    delete b;
    return SW2GPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// continuous batching engine

namespace {

struct EngInst {
    sw2gpu_ctx* c = nullptr;
    int64_t id = 0;
    double t = 0.0, dt = 0.0, dt0 = 0.0;   // current and base time step
    int nsteps = 0, steps = 0, failures = 0, consecutive = 0, max_retries = 0, ticks = 0, last_status = 0;
    long newton = 0, linear = 0;
    std::vector<PwlSeries> ser;
    bool in_step = false;
    NState ns;
};

}  // namespace

struct sw2gpu_engine {
    std::unique_ptr<Runner> R;
    std::vector<EngInst> inst;     // slot k of the runner = inst[k]
    bool dirty = true;             // membership changed since the runner last saw it
    bool own_stream = false;
    int precision = SW2GPU_FP64;
    sw2gpu_stats last{};           // the last tick (see sw2gpu_engine_last_tick)
};

extern "C" {

int sw2gpu_engine_create(int32_t precision, void* stream, sw2gpu_engine** out) {
    if (!out || (precision != SW2GPU_FP64 && precision != SW2GPU_MIXED)) return fail(SW2GPU_E_ARG, "bad engine arguments");
    *out = nullptr;
    auto* e = new sw2gpu_engine();
    std::unique_ptr<sw2gpu_engine> guard(e);
    cudaStream_t st = (cudaStream_t)stream;
    if (!st) {
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        e->own_stream = true;
    }
    e->precision = precision;
    e->R.reset(new Runner());
    int rc = runner_alloc(*e->R, st, precision == SW2GPU_MIXED, kMaxBatch);
    if (rc) {
        if (e->own_stream) cudaStreamDestroy(st);
        return rc;
    }
    *out = guard.release();
    return SW2GPU_OK;
}

int sw2gpu_engine_add(sw2gpu_engine* e, sw2gpu_ctx* ctx, int64_t id, double t0, double dt, int32_t nsteps,
                      int32_t max_retries, int32_t nseries, const int32_t* series_len, const double* series_t,
                      const double* series_v) {
    if (!e || !ctx || !(dt > 0.0) || nsteps <= 0 || max_retries < 0 || nseries < 0)
        return fail(SW2GPU_E_ARG, "bad engine_add arguments");
    if ((int)e->inst.size() >= kMaxBatch) return fail(SW2GPU_E_ARG, "engine holds %d instances already", kMaxBatch);
    if (ctx->p.precision != e->precision) return fail(SW2GPU_E_ARG, "instance precision differs from the engine's");
    for (auto& x : e->inst)
        if (x.c == ctx || x.id == id) return fail(SW2GPU_E_ARG, "instance or id already in the engine");
    if (nseries < ctx->NS) return fail(SW2GPU_E_ARG, "instance reads %d series, %d given", ctx->NS, nseries);
    EngInst x;
    x.c = ctx;
    x.id = id;
    x.t = t0;
    x.dt = x.dt0 = dt;
    x.nsteps = nsteps;
    x.max_retries = max_retries;
    size_t off = 0;
    for (int s = 0; s < nseries; s++) {
        const int n = series_len[s];
        if (n <= 0) return fail(SW2GPU_E_ARG, "series %d is empty", s);
        PwlSeries ps;
        ps.t.assign(series_t + off, series_t + off + n);
        ps.v.assign(series_v + off, series_v + off + n);
        for (int i = 1; i < n; i++)
            if (!(ps.t[i] > ps.t[i - 1])) return fail(SW2GPU_E_ARG, "series %d: times not increasing", s);
        off += n;
        x.ser.push_back(std::move(ps));
    }
    // the instance's own stream may still hold its state uploads: order them first
    CK(cudaStreamSynchronize(ctx->stream));
    e->inst.push_back(std::move(x));
    e->dirty = true;
    return SW2GPU_OK;
}

int32_t sw2gpu_engine_active(const sw2gpu_engine* e) { return e ? (int32_t)e->inst.size() : 0; }

int sw2gpu_engine_last_tick(const sw2gpu_engine* e, sw2gpu_stats* out) {
    if (!e || !out) return fail(SW2GPU_E_ARG, "null argument");
    *out = e->last;
    return SW2GPU_OK;
}

int sw2gpu_engine_set_rebalance(sw2gpu_engine* e, int32_t rounds, double fraction) {
    if (!e || rounds < 1 || rounds > Runner::kMaxRounds || !(fraction >= 0.0 && fraction <= 1.0))
        return fail(SW2GPU_E_ARG, "rebalance: rounds in [1, %d], fraction in [0, 1]", Runner::kMaxRounds);
    e->R->rb_rounds = rounds;
    e->R->rb_frac = fraction;
    return SW2GPU_OK;
}

int sw2gpu_engine_tick(sw2gpu_engine* e, sw2gpu_run_stats* finished, int32_t max_finished, int32_t* nfinished) {
    if (!e || !nfinished || (max_finished > 0 && !finished)) return fail(SW2GPU_E_ARG, "bad engine_tick arguments");
    *nfinished = 0;
    const int K = (int)e->inst.size();
    if (K == 0) return SW2GPU_OK;
    if (max_finished < K) return fail(SW2GPU_E_ARG, "room for %d finished instances needed", K);
    Runner& R = *e->R;
    int rc = 0;
    if (e->dirty) {
        std::vector<sw2gpu_ctx*> cs;
        for (auto& x : e->inst) cs.push_back(x.c);
        if ((rc = runner_set(R, cs))) return rc;
        e->dirty = false;
    }
    R.launches = 0;
    R.nphase = 0;
    CK(cudaEventRecord(R.ev0, R.stream));
    // instances between steps start one: dt, step-averaged series, level rotation
    std::vector<int> S;
    for (int k = 0; k < K; k++) {
        EngInst& x = e->inst[k];
        if (x.in_step) continue;
        std::vector<double> sv(x.ser.size());
        for (size_t q = 0; q < x.ser.size(); q++) sv[q] = x.ser[q].avg(x.t, x.t + x.dt);
        if ((rc = step_begin(R, k, x.dt, sv.empty() ? nullptr : sv.data()))) return rc;
        S.push_back(k);
    }
    if ((rc = runner_tables(R, 1))) return rc;
    if (!S.empty()) {
        if ((rc = launch_init(R, S))) return rc;
        if ((rc = launch_resid(R, S))) return rc;
        if ((rc = read_results(R, S))) return rc;
        for (int k : S) {
            newton_begin(R, k, e->inst[k].ns);
            e->inst[k].in_step = true;
        }
    }
    // one Newton iteration of every instance inside a step
    std::vector<int> N;
    for (int k = 0; k < K; k++)
        if (e->inst[k].in_step && !e->inst[k].ns.done) N.push_back(k);
    if (!N.empty()) {
        std::vector<NState> ns(K);
        for (int k = 0; k < K; k++) ns[k] = e->inst[k].ns;
        if ((rc = newton_iteration(R, N, ns))) return rc;
        for (int k : N) e->inst[k].ns = ns[k];
    }
    // steps that ended: advance, or reset to the old level and retry with dt / 4
    std::vector<int> failed;
    for (int k = 0; k < K; k++) {
        EngInst& x = e->inst[k];
        x.ticks++;
        if (!x.in_step || !x.ns.done) continue;
        const int st = newton_status(x.ns, x.c->p);
        x.newton += x.ns.it;
        x.linear += x.ns.lin;
        x.in_step = false;
        if (st == SW2GPU_OK) {   // dt doubles back toward the base dt (tc_end, src/tools/tc_end.c:55-66)
            x.steps++;
            x.t += x.dt;
            x.dt = std::min(2.0 * x.dt, x.dt0);
            x.consecutive = 0;
        } else {
            x.failures++;
            x.consecutive++;
            x.last_status = st;
            x.dt *= 0.25;
            failed.push_back(k);
        }
    }
    if (!failed.empty() && (rc = launch_init(R, failed))) return rc;
    CK(cudaEventRecord(R.ev1, R.stream));
    CK(cudaEventSynchronize(R.ev1));
    {
        sw2gpu_stats& L = e->last;
        memset(&L, 0, sizeof(L));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, R.ev0, R.ev1);
        double ph[3];
        phase_times(R, ph);
        L.newton_its = (int32_t)N.size();
        L.linesearch_cuts = (int32_t)S.size();
        L.wd_elems = K;
        for (int k : N) L.linear_its = std::max<int32_t>(L.linear_its, R.ctl_h[k].iterations);
        L.device_ms = ms;
        L.kernel_launches = R.launches;
        L.jac_ms = ph[kPhJac];
        L.krylov_ms = ph[kPhKrylov];
        L.resid_ms = ph[kPhResid];
        L.other_ms = ms - ph[0] - ph[1] - ph[2];
    }
    // instances done with their steps (or out of retries) leave the engine
    std::vector<EngInst> keep;
    for (auto& x : e->inst) {
        const bool gave_up = x.consecutive > x.max_retries;
        if (x.steps >= x.nsteps || gave_up) {
            sw2gpu_run_stats& o = finished[(*nfinished)++];
            memset(&o, 0, sizeof(o));
            o.id = x.id;
            o.status = gave_up ? x.last_status : SW2GPU_OK;
            o.steps = x.steps;
            o.failures = x.failures;
            o.newton_its = (int32_t)x.newton;
            o.linear_its = (int32_t)x.linear;
            o.ticks = x.ticks;
            o.t = x.t;
            o.dt = x.dt;
            e->dirty = true;
        } else {
            keep.push_back(std::move(x));
        }
    }
    e->inst.swap(keep);
    return SW2GPU_OK;
}

int sw2gpu_engine_destroy(sw2gpu_engine* e) {
    if (!e) return SW2GPU_OK;
    cudaStream_t st = e->R->stream;
    cudaStreamSynchronize(st);
    e->R.reset();
    if (e->own_stream) cudaStreamDestroy(st);
    delete e;
    return SW2GPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// request server: admission by free device memory, continuous batching, latencies

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// a request's own copy of everything it was submitted with
struct Request {
    int64_t id = 0;
    // mesh arrays
    int32_t nnodes = 0, nelems2d = 0, nelems1d = 0, nstrings = 0, nmats = 0, nseries = 0;
    std::vector<double> x, y, z, rough, ev, eevc, cor;
    std::vector<int32_t> node_string, e2n, e2m, e1n, e1s, e1p, bc, isg, ivx, ivy, iu0, eevm;
    sw2gpu_params prm{};
    std::vector<double> h0, u0, v0;
    double t0 = 0, dt = 0;
    int32_t nsteps = 0;
    std::vector<int32_t> slen;
    std::vector<double> st, sv;
    size_t est_bytes = 0;
    sw2gpu_ctx* ctx = nullptr;
    Clock::time_point submitted, admitted, finished;
    // result
    sw2gpu_request_stats stats{};
    std::vector<double> h, u, v;
    std::string error;
    bool done = false;
    sw2gpu_mesh mesh() const {
        sw2gpu_mesh m;
        m.nnodes = nnodes; m.nelems2d = nelems2d; m.nelems1d = nelems1d; m.nstrings = nstrings;
        m.nmats = nmats; m.nseries = nseries;
        m.x = x.data(); m.y = y.data(); m.z = z.data(); m.node_string = node_string.data();
        m.elem2d_nodes = e2n.data(); m.elem2d_mat = e2m.data();
        m.elem1d_nodes = e1n.data(); m.elem1d_string = e1s.data(); m.elem1d_parent = e1p.data();
        m.str_bc_flag = bc.data(); m.str_isigma = isg.data(); m.str_ivx = ivx.data(); m.str_ivy = ivy.data();
        m.str_iu0 = iu0.data(); m.str_rough_height = rough.data();
        m.mat_eev_mode = eevm.data(); m.mat_ev = ev.data(); m.mat_eev_coef = eevc.data(); m.mat_coriolis = cor.data();
        return m;
    }
};

template <typename T>
std::vector<T> vcopy(const T* p, size_t n) {
    return p && n ? std::vector<T>(p, p + n) : std::vector<T>(std::max<size_t>(n, 0));
}

// device bytes of a request before its context exists: per triangle the element arrays, the
// 81-value FD Jacobian records and ~3.5 BCSR blocks; per node the three state levels, the
// Krylov vectors and the row data (measured contexts hold ~1.6 KB per triangle)
size_t estimate_bytes(const Request& q) {
    return (size_t)q.nelems2d * 1800 + (size_t)q.nnodes * 640 + (size_t)q.nelems1d * 400 + (1u << 20);
}

}  // namespace

struct sw2gpu_server {
    int precision = SW2GPU_FP64;
    size_t budget = 0;                 // device bytes the admitted requests may hold
    int max_active = kMaxBatch;
    std::mutex mu;
    std::condition_variable cv;        // new work, admission room, results
    std::deque<std::shared_ptr<Request>> queue;     // submitted, not yet admitted
    std::deque<std::shared_ptr<Request>> ready;     // context built, not yet in the engine
    std::map<int64_t, std::shared_ptr<Request>> live;   // admitted, not yet collected
    size_t in_use = 0;                 // device bytes of admitted requests
    int admitted_active = 0;           // admitted and not finished
    int64_t next_id = 1;
    bool stop = false;
    std::string fatal;                 // error that stopped the worker
    sw2gpu_engine* eng = nullptr;
    cudaStream_t stream = nullptr;
    int device = 0;
    std::vector<std::thread> loaders;   // build admitted requests' contexts in parallel
    std::thread worker;

    void load_loop();
    void work_loop();
};

void sw2gpu_server::load_loop() {
    cudaSetDevice(device);
    for (;;) {
        std::shared_ptr<Request> q;
        {
            std::unique_lock<std::mutex> lk(mu);
            // FIFO admission: the head request waits until its bytes fit the budget
            cv.wait(lk, [&] {
                if (stop) return true;
                if (queue.empty()) return false;
                const auto& h = queue.front();
                return admitted_active < max_active && (in_use + h->est_bytes <= budget || admitted_active == 0);
            });
            if (stop) return;
            q = queue.front();
            queue.pop_front();
            in_use += q->est_bytes;
            admitted_active++;
        }
        q->admitted = Clock::now();
        const sw2gpu_mesh m = q->mesh();
        sw2gpu_ctx* c = nullptr;
        int rc = sw2gpu_create(&m, &q->prm, nullptr, &c);
        if (!rc) rc = sw2gpu_set_state(c, 0, q->h0.data(), q->u0.data(), q->v0.data());
        if (!rc) rc = sw2gpu_set_state(c, 1, q->h0.data(), q->u0.data(), q->v0.data());
        if (!rc) rc = sw2gpu_set_state(c, 2, q->h0.data(), q->u0.data(), q->v0.data());
        std::lock_guard<std::mutex> lk(mu);
        if (rc) {   // the request fails on its own; the server goes on
            q->error = g_err;
            q->stats.status = rc;
            q->done = true;
            q->finished = Clock::now();
            if (c) sw2gpu_destroy(c);
            in_use -= q->est_bytes;
            admitted_active--;
        } else {
            q->ctx = c;
            in_use = in_use - q->est_bytes + c->bytes;   // the context's measured size
            q->est_bytes = c->bytes;
            ready.push_back(q);
        }
        cv.notify_all();
    }
}

void sw2gpu_server::work_loop() {
    cudaSetDevice(device);
    std::map<int64_t, std::shared_ptr<Request>> running;
    std::vector<sw2gpu_run_stats> fin(kMaxBatch);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return stop || !ready.empty() || !running.empty(); });
            if (stop) break;
            // requests that arrived while others run join the engine between ticks
            while (!ready.empty() && sw2gpu_engine_active(eng) < kMaxBatch) {
                auto q = ready.front();
                ready.pop_front();
                std::vector<int32_t> len = q->slen;
                const int rc = sw2gpu_engine_add(eng, q->ctx, q->id, q->t0, q->dt, q->nsteps, 8, (int32_t)len.size(),
                                                 len.empty() ? nullptr : len.data(), q->st.data(), q->sv.data());
                if (rc) {
                    q->error = g_err;
                    q->stats.status = rc;
                    q->done = true;
                    q->finished = Clock::now();
                    sw2gpu_destroy(q->ctx);
                    q->ctx = nullptr;
                    in_use -= q->est_bytes;
                    admitted_active--;
                    cv.notify_all();
                    continue;
                }
                running[q->id] = q;
            }
        }
        if (running.empty()) continue;
        int32_t nf = 0;
        const int rc = sw2gpu_engine_tick(eng, fin.data(), (int32_t)fin.size(), &nf);
        if (rc) {   // a device-level failure: fail every running request and stop
            std::lock_guard<std::mutex> lk(mu);
            fatal = g_err;
            for (auto& kv : running) {
                kv.second->error = fatal;
                kv.second->stats.status = rc;
                kv.second->done = true;
                kv.second->finished = Clock::now();
            }
            stop = true;
            cv.notify_all();
            break;
        }
        for (int i = 0; i < nf; i++) {
            auto it = running.find(fin[i].id);
            if (it == running.end()) continue;
            auto q = it->second;
            running.erase(it);
            q->h.resize(q->nnodes);
            q->u.resize(q->nnodes);
            q->v.resize(q->nnodes);
            sw2gpu_get_state(q->ctx, 0, q->h.data(), q->u.data(), q->v.data());
            sw2gpu_destroy(q->ctx);
            q->ctx = nullptr;
            q->finished = Clock::now();
            sw2gpu_request_stats& st = q->stats;
            st.id = q->id;
            st.status = fin[i].status;
            st.steps = fin[i].steps;
            st.failures = fin[i].failures;
            st.newton_its = fin[i].newton_its;
            st.linear_its = fin[i].linear_its;
            st.t = fin[i].t;
            st.queue_ms = ms_between(q->submitted, q->admitted);
            st.run_ms = ms_between(q->admitted, q->finished);
            st.latency_ms = ms_between(q->submitted, q->finished);
            st.device_bytes = (int64_t)q->est_bytes;
            std::lock_guard<std::mutex> lk(mu);
            q->done = true;
            in_use -= q->est_bytes;
            admitted_active--;
            cv.notify_all();
        }
    }
    // stopping: contexts of requests still in the engine are released here
    for (auto& kv : running)
        if (kv.second->ctx) {
            sw2gpu_destroy(kv.second->ctx);
            kv.second->ctx = nullptr;
        }
}

extern "C" {

int sw2gpu_server_create(int32_t precision, double hbm_fraction, int32_t max_active, sw2gpu_server** out) {
    if (!out || !(hbm_fraction > 0.0 && hbm_fraction <= 1.0) || max_active <= 0 ||
        (precision != SW2GPU_FP64 && precision != SW2GPU_MIXED))
        return fail(SW2GPU_E_ARG, "bad server arguments");
    *out = nullptr;
    auto* S = new sw2gpu_server();
    std::unique_ptr<sw2gpu_server> guard(S);
    CK(cudaGetDevice(&S->device));
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    S->budget = (size_t)(hbm_fraction * (double)fr);
    S->precision = precision;
    S->max_active = std::min<int>(max_active, kMaxBatch);
    CK(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    int rc = sw2gpu_engine_create(precision, S->stream, &S->eng);
    if (rc) {
        cudaStreamDestroy(S->stream);
        return rc;
    }
    const int nload = std::max(1, std::min(4, (int)std::thread::hardware_concurrency() / 2));
    for (int i = 0; i < nload; i++) S->loaders.emplace_back([S] { S->load_loop(); });
    S->worker = std::thread([S] { S->work_loop(); });
    *out = guard.release();
    return SW2GPU_OK;
}

int sw2gpu_server_submit(sw2gpu_server* S, const sw2gpu_mesh* m, const sw2gpu_params* prm, const double* h0,
                         const double* u0, const double* v0, double t0, double dt, int32_t nsteps, int32_t nseries,
                         const int32_t* series_len, const double* series_t, const double* series_v, int64_t* id) {
    if (!S || !m || !prm || !h0 || !u0 || !v0 || !id || !(dt > 0.0) || nsteps <= 0 || nseries < 0)
        return fail(SW2GPU_E_ARG, "bad submit arguments");
    auto q = std::make_shared<Request>();
    q->nnodes = m->nnodes; q->nelems2d = m->nelems2d; q->nelems1d = m->nelems1d;
    q->nstrings = m->nstrings; q->nmats = m->nmats; q->nseries = m->nseries;
    const size_t V = m->nnodes, T = m->nelems2d, E = m->nelems1d, NS = m->nstrings, NM = m->nmats;
    q->x = vcopy(m->x, V); q->y = vcopy(m->y, V); q->z = vcopy(m->z, V); q->node_string = vcopy(m->node_string, V);
    q->e2n = vcopy(m->elem2d_nodes, 3 * T); q->e2m = vcopy(m->elem2d_mat, T);
    q->e1n = vcopy(m->elem1d_nodes, 2 * E); q->e1s = vcopy(m->elem1d_string, E); q->e1p = vcopy(m->elem1d_parent, E);
    q->bc = vcopy(m->str_bc_flag, NS); q->isg = vcopy(m->str_isigma, NS); q->ivx = vcopy(m->str_ivx, NS);
    q->ivy = vcopy(m->str_ivy, NS); q->iu0 = vcopy(m->str_iu0, NS); q->rough = vcopy(m->str_rough_height, NS);
    q->eevm = vcopy(m->mat_eev_mode, NM); q->ev = vcopy(m->mat_ev, 3 * NM); q->eevc = vcopy(m->mat_eev_coef, NM);
    q->cor = vcopy(m->mat_coriolis, NM);
    q->prm = *prm;
    q->prm.precision = S->precision;
    q->h0 = vcopy(h0, V); q->u0 = vcopy(u0, V); q->v0 = vcopy(v0, V);
    q->t0 = t0; q->dt = dt; q->nsteps = nsteps;
    size_t npts = 0;
    for (int i = 0; i < nseries; i++) npts += (size_t)series_len[i];
    q->slen = vcopy(series_len, (size_t)nseries);
    q->st = vcopy(series_t, npts);
    q->sv = vcopy(series_v, npts);
    if (q->st.empty()) { q->st.push_back(0.0); q->sv.push_back(0.0); }
    q->est_bytes = estimate_bytes(*q);
    q->submitted = Clock::now();
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return fail(SW2GPU_E_CUDA, "server stopped: %s", S->fatal.c_str());
    q->id = S->next_id++;
    *id = q->id;
    S->live[q->id] = q;
    S->queue.push_back(q);
    S->cv.notify_all();
    return SW2GPU_OK;
}

int sw2gpu_server_wait(sw2gpu_server* S, int64_t id, double timeout_s, sw2gpu_request_stats* st, double* h,
                       double* u, double* v) {
    if (!S) return fail(SW2GPU_E_ARG, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->live.find(id);
    if (it == S->live.end()) return fail(SW2GPU_E_ARG, "unknown or collected request %lld", (long long)id);
    auto q = it->second;
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                              std::chrono::duration<double>(std::max(timeout_s, 0.0)));
    if (!S->cv.wait_until(lk, deadline, [&] { return q->done; })) return SW2GPU_PENDING;
    if (st) *st = q->stats;
    if (!q->h.empty()) {
        const size_t nb = sizeof(double) * q->nnodes;
        if (h) memcpy(h, q->h.data(), nb);
        if (u) memcpy(u, q->u.data(), nb);
        if (v) memcpy(v, q->v.data(), nb);
    }
    S->live.erase(it);
    if (!q->error.empty()) return fail(q->stats.status ? q->stats.status : SW2GPU_E_CUDA, "%s", q->error.c_str());
    return SW2GPU_OK;
}

int sw2gpu_server_status(sw2gpu_server* S, int32_t* queued, int32_t* active, int64_t* bytes_in_use,
                         int64_t* budget) {
    if (!S) return fail(SW2GPU_E_ARG, "null server");
    std::lock_guard<std::mutex> lk(S->mu);
    if (queued) *queued = (int32_t)S->queue.size();
    if (active) *active = S->admitted_active;
    if (bytes_in_use) *bytes_in_use = (int64_t)S->in_use;
    if (budget) *budget = (int64_t)S->budget;
    return S->fatal.empty() ? SW2GPU_OK : fail(SW2GPU_E_CUDA, "server stopped: %s", S->fatal.c_str());
}

int sw2gpu_server_destroy(sw2gpu_server* S) {
    if (!S) return SW2GPU_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    for (auto& t : S->loaders)
        if (t.joinable()) t.join();
    if (S->worker.joinable()) S->worker.join();
    for (auto& q : S->ready)
        if (q->ctx) sw2gpu_destroy(q->ctx);
    sw2gpu_engine_destroy(S->eng);
    cudaStreamDestroy(S->stream);
    delete S;
    return SW2GPU_OK;
}

}  // extern "C"
