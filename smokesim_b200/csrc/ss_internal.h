// ss_internal.h - device state of one grid and the kernel launchers.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/smokesim.h"

namespace ss {

// Launch a kernel, with programmatic dependent launch allowed when `pdl` is
// set: the kernel may then be scheduled while the kernel before it on the
// stream (or in the captured graph) drains.  Every kernel launched this way
// calls pdl_entry() (common.cuh) before it touches global memory; that waits
// until the preceding kernel has completed and its writes are visible, so the
// results are those of a plain launch.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(bool pdl, dim3 grid, dim3 block, size_t smem, cudaStream_t st, void (*kernel)(KArgs...),
                            Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

struct Level {
    int n[3];
    float h;    // cell size of the level: h * 2^L
    float hh;   // h*h
};

// Launch-time constants of a step (all derived on the host in FP32 exactly as
// the oracle derives them).
struct StepConsts {
    float dt, rho, t_amb, alpha, beta, eps;
    float wind[3];
    float cfl;      // dt / h
    float rho_h;    // rho * h       (smoother right-hand side)
    float dt_h;     // dt * h        (residual right-hand side)
    float k_upd;    // -dt / (rho*h) (projection update)
    float vort_k;   // unused scaling helper
};

struct ReduceSlots {
    double* partial;      // per-block partial sums (device scratch)
    double* partial_max = nullptr;  // per-block maxima (mixed-precision solve)
    double* partial2 = nullptr;     // second-stage partials: sums, then maxima (2 * stage2 entries)
    unsigned int* ticket = nullptr; // blocks finished in the refinement residual (the last one folds)
    int stage2 = 0;
    double* out;          // reduction results (device), SLOT_* below
    double* host;         // pinned mirror of out
    int max_blocks;
};
// SLOT_STEPS: refinement steps a device-side tolerance loop took (a double);
// SLOT_ERR: the device error word (an int at the start of the slot), so that
// one copy of the slots brings both back
enum { SLOT_DIV_BEFORE = 0, SLOT_RESIDUAL = 1, SLOT_DIV_AFTER = 2, SLOT_AMAX = 3, SLOT_STEPS = 4, SLOT_ERR = 7,
       SLOT_COUNT = 8 };

// Convergence test of the mixed solve's tolerance loop, folded into the last
// block of the refinement residual (k_ir_residual): it records k, the
// refinement steps done, in SLOT_STEPS and, where more is set and the
// residual norm is above tol times the pre-solve divergence norm, sets the
// condition of the graph node that runs the next refinement step.
struct IrDecide {
    cudaGraphConditionalHandle next = 0;
    double tol = 0.0;
    int k = 0;
    int more = 0;
    int active = 0;
};

struct TensorMapEntry {
    CUtensorMap map;
    const void* ptr;
    bool bytes;
    int dims[3];
    int box[3];
};

}  // namespace ss

struct ss_sim {
    int dim, nx, ny, nz, nch, enclosed, min_coarse;
    float h, t_amb0;
    size_t ncell, nv[3];

    float* vel[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
    int vi[3] = {0, 0, 0};
    float* dens[2] = {nullptr, nullptr};   // nch planes of ncell, channel-major
    float* temp[2] = {nullptr, nullptr};
    int si = 0;

    uint8_t* solid = nullptr;      // level-0: 1 solid / 0 fluid (rasteriser output)
    uint8_t* flags = nullptr;      // level-0 flag byte with neighbour bits
    uint8_t* fmask = nullptr;      // level-0 fluid mask (M_* bits); null when nx is odd
    float* svel[3] = {nullptr, nullptr, nullptr};   // solid velocity (FP16-rounded); null = all zero
    int svel_active = 0;

    int levels = 0;
    int bottom = 0;            // first level solved by the single-block bottom kernel (== levels: none)
    ss::Level lv[SS_MAX_LEVELS];
    float* p[SS_MAX_LEVELS] = {};
    float* r[SS_MAX_LEVELS] = {};
    float* p_alt[SS_MAX_LEVELS] = {};   // second buffer of the tiled sweep (p_in -> p_out)
    float* r_alt[SS_MAX_LEVELS] = {};   // second buffer of the fused in-place residual (L >= 1)
    float* alpha[SS_MAX_LEVELS] = {};   // coarse solid fraction (L >= 1), FP16-rounded values
    float* div0 = nullptr;              // level-0 divergence, smoother boundary rule
    float* div0r = nullptr;             // residual boundary rule (== div0 when enclosed)
    float* vort = nullptr;              // 3*ncell (2D: ncell) vorticity scratch
    float* rhs_s = nullptr;             // level-0 rho*h*div/dt of the current solve, colour-split (k_rb.cu)
    float* rhs_r = nullptr;             // level-0 rho*div/(dt*h) of the current solve, colour-split
    int rhs_r_is_s = 0;                 // the mixed solve's residual right-hand side equals rhs_s (h^2 == 1): rhs_r unused
    uint8_t* rb_mask = nullptr;         // colour-split copy of fmask
    float* rb_pw = nullptr;             // level-0 prolongation weights per axis (x, then y, then z)
    // mixed-precision solve: FP64 level-0 pressure, FP16/BF16 coarse levels
    double* p64 = nullptr;
    double* p64b = nullptr;             // ping-pong partner of p64 (update + residual in one pass)
    double* p64c = nullptr;             // the extrapolated warm start's p(n-2) (warm_start 1)
    int prev_ok = 0;                    // p64c holds the pressure the current p64 was solved from
    int p64_parity = 0;                 // which of the two allocations p64 currently is
    int p64_valid = 0;                  // p64 holds the current pressure (else p[0] does)
    int cstore = 0;                     // storage type of cp/cr (SS_PREC_MIXED or SS_PREC_MIXED_BF16)
    void* cp[SS_MAX_LEVELS] = {};       // coarse pressure, 2 bytes per cell (L >= 1)
    void* cr[SS_MAX_LEVELS] = {};       // coarse right-hand side / residual
    float* d_scale = nullptr;           // [scale, 1/scale] of the coarse storage (device)
    float force[3] = {0.f, 0.f, 0.f};   // control force on the faces inside active emitters
    float* ffield = nullptr;            // coarse control force field, 3 * ff_n^3 (none: ff_n == 0)
    int ff_n = 0;
    void* render_buf = nullptr;         // device image of ss_render with a host destination
    size_t render_bytes = 0;
    int rb_vec = 0;                     // level-0 kernels may work on 4 cells per thread (nx % 8 == 0)
    int rb_prolong_vec = 0;             // ... and the prolongation too (even sizes, table pattern checked)
    ss::ReduceSlots red{};

    std::vector<ss_emitter> em;
    std::vector<ss_obstacle> ob;
    std::vector<ss_box> bx;
    ss_emitter* d_em = nullptr;
    ss_obstacle* d_ob = nullptr;
    ss_box* d_bx = nullptr;
    int cap_em = 0, cap_ob = 0, cap_bx = 0;
    int pyramid_dirty = 1;

    ss_stats st{};
    long long nlaunch = 0;     // kernels launched since the counter was reset
    int* d_err = nullptr;      // device error word (in red.out[SLOT_ERR]): bit 0 = a bounded barrier wait gave up
    int err_armed = 0;         // a kernel that can set the error word ran since the word was last read
    int use_tma = 1;           // TMA tile loads of the coarse-level tiled sweeps (0: per-thread loads)
    // mixed solve: the coarsest level by its response matrix instead of its
    // n_coarse sweeps (levels of at most kCoarseResponseMax cells)
    int coarse_matrix = 1;       // SMOKESIM_COARSE_SWEEPS=1 sets 0
    float* cmat = nullptr;       // cmat_n^2: E[i n + j] = dp_j / dr_i
    float* cmat_alpha = nullptr; // solid fractions it was built for
    int* cmat_state = nullptr;   // device: [0] iteration count it was built for, [1] rebuild flag
    float* cmat_part = nullptr;  // the product's slice sums (kProductLanes floats)
    int cmat_n = 0, cmat_iters = -1, cmat_dirty = 1;
    // The multigrid part of a solve recorded once as a CUDA graph and replayed
    // (api.cpp, run_graph): slot 0 fixed-count FP32 V-cycles, 1 one FP32
    // tolerance cycle, 2/3 one mixed refinement step per FP64 buffer parity,
    // 4/5 the mixed tolerance loop on the device per starting parity.
    struct SolveGraph {
        cudaGraphExec_t exec = nullptr;
        unsigned char key[96] = {};
        long long launches = 0;        // kernels of one replay (4/5: of the first residual)
        long long step_launches = 0;   // 4/5: kernels of one refinement step
    };
    SolveGraph graphs[6];
    int use_graphs = 1;
    // mixed solve to a tolerance: the first chain_depth refinement steps as
    // nested conditional graph nodes, the convergence test on the device
    // (SMOKESIM_DEVICE_LOOP=0 sets 0: a host round trip per step)
    int device_loop = 1;
    cudaStream_t chain_stream = nullptr;   // records the nested step graphs
    // programmatic dependent launch of the solve's kernel chain (SMOKESIM_PDL=0 sets 0)
    int pdl = 1;
    // mixed solve: the levels from cluster_from down in one thread-block
    // cluster launch (k_coarse_cluster) of cluster_ctas CTAs; -1 = not yet
    // probed, 0 = per-level launches (SMOKESIM_CLUSTER=0 sets use_cluster 0)
    int use_cluster = 1;
    int cluster_from = 0;
    int cluster_ctas = -1;
    float* cluster_fine = nullptr;   // a cluster level's residuals (kClusterCells floats)
    int rb_active = 0;         // level-0 pressure currently lives colour-split in p_alt[0]
    std::vector<ss::TensorMapEntry> tmaps;
    cudaStream_t stream0 = nullptr;
};

namespace ss {

// error helpers (api.cpp)
int set_error(int code, const std::string& msg);
int check_cuda(cudaError_t e, const char* what);

StepConsts make_consts(const ss_sim* s, const ss_params* p);

// ---- fluid kernels (k_fluid.cu) ----
int launch_emitters(ss_sim* s, const StepConsts& c, cudaStream_t st);
int launch_advect_velocities(ss_sim* s, const StepConsts& c, bool fuse_buoyancy, cudaStream_t st);
int launch_buoyancy(ss_sim* s, const StepConsts& c, cudaStream_t st);
int launch_vorticity(ss_sim* s, const StepConsts& c, cudaStream_t st);
int launch_update_velocities(ss_sim* s, const StepConsts& c, cudaStream_t st);
// div_slot >= 0: also fold the squared divergence of the current velocities
// into that statistics slot (the k_divergence operator, no right-hand sides)
int launch_advect_smoke(ss_sim* s, const StepConsts& c, cudaStream_t st, int div_slot = -1);
// divergence of the current velocities into div0 (+div0r); optional ||div||^2 into slot
// with sc and quirks >= 0 also the level-0 right-hand sides rhs_s / rhs_r of that boundary rule;
// with ep / eq also the extrapolated warm start of the mixed solve in the same pass
// (every cell: ep = 2 ep - eq, eq = the old ep)
int launch_divergence(ss_sim* s, bool write, int slot, cudaStream_t st, const StepConsts* sc = nullptr,
                      int quirks = -1, double* ep = nullptr, double* eq = nullptr);

// ---- multigrid kernels (k_mg.cu) ----
int launch_smooth(ss_sim* s, const StepConsts& c, int L, int iterations, int quirks, cudaStream_t st);
int launch_residual(ss_sim* s, const StepConsts& c, int L, bool write_fine, bool write_coarse, int quirks,
                    cudaStream_t st);
int launch_restrict(ss_sim* s, int L, cudaStream_t st);
int launch_prolong(ss_sim* s, int L, cudaStream_t st);
int launch_projected_residual_norm(ss_sim* s, const StepConsts& c, int slot, cudaStream_t st);
int launch_solid_pyramid(ss_sim* s, cudaStream_t st);
// levels Lb..coarsest of the V-cycle in one thread block (shared memory)
constexpr int kBottomSmemBytes = 160 * 1024;
int bottom_start(const ss_sim* s);
int launch_bottom(ss_sim* s, const ss_mg_schedule& mg, int L, cudaStream_t st);
// one red-black sweep per launch, tiled in shared memory (k_rbgs.cu)
int launch_rbgs_sweep(ss_sim* s, const StepConsts& c, int L, int quirks, bool prolong, bool resid,
                      cudaStream_t st);
// the same sweep with the tile fetched by TMA (k_rbgs_tma.cu); 3D, nx % 16 == 0
bool tma_sweep_supported(const ss_sim* s, int L);
int launch_rbgs_sweep_tma(ss_sim* s, const StepConsts& c, int L, int quirks, bool resid, cudaStream_t st);
// level 0 on colour-split arrays during a solve (k_rb.cu)
bool rb_supported(const ss_sim* s, int quirks);
int launch_rb_convert(ss_sim* s, bool split, cudaStream_t st);
int launch_rb_split_mask(ss_sim* s, cudaStream_t st);
// zero: the select-free half-sweep (every non-fluid cell of the other colour holds +0)
// from_zero: the sweeps start from a zero level-0 pressure (cleared here or
// by the first half-sweep)
int launch_rb_sweep(ss_sim* s, int iterations, cudaStream_t st, bool zero = false, bool from_zero = false);
bool rb_zero_form(const ss_sim* s);
int launch_rb_residual_restrict(ss_sim* s, cudaStream_t st);
int launch_rb_prolong(ss_sim* s, cudaStream_t st);
int rb_init_vector_paths(ss_sim* s, cudaStream_t st);

// mixed-precision correction solve (k_mg.cu, k_rb.cu, k_mixed.cu)
int coarse_smooth(ss_sim* s, const StepConsts& c, int L, int iterations, int prec, cudaStream_t st);
int coarse_residual_restrict(ss_sim* s, const StepConsts& c, int L, int prec, cudaStream_t st);
int coarse_prolong(ss_sim* s, int L, int prec, cudaStream_t st);
int coarse_bottom(ss_sim* s, const ss_mg_schedule& mg, int L, int prec, cudaStream_t st);
int coarse_cluster_from(const ss_sim* s);
int coarse_cluster_setup(ss_sim* s);
int coarse_cluster(ss_sim* s, const ss_mg_schedule& mg, int L, int prec, cudaStream_t st);
int launch_rb_residual_restrict_mixed(ss_sim* s, int prec, cudaStream_t st);

int launch_rb_prolong_mixed(ss_sim* s, int prec, cudaStream_t st);
int launch_p64_from_p0(ss_sim* s, cudaStream_t st);
int launch_p0_from_p64(ss_sim* s, cudaStream_t st);
int launch_ir_residual(ss_sim* s, const StepConsts& c, int slot, bool accumulate, cudaStream_t st,
                       const IrDecide* dec = nullptr);
int launch_ir_accumulate(ss_sim* s, cudaStream_t st);
// p0_out: when given, the FP32 copy of the FP64 pressure is written there too
int launch_update_velocities_p64(ss_sim* s, const StepConsts& c, cudaStream_t st, float* p0_out = nullptr);
// first stage of a deterministic reduction over n per-block partials: sums
// (or maxima) of consecutive groups of 1024; *res / *nres describe what is
// left for a single final block (the input itself when n <= 1024)
int reduce_stage1(ss_sim* s, const double* in, int n, bool is_max, const double** res, int* nres, cudaStream_t st);

// Forward state copies a step can leave for its adjoint (api.cpp, run_step):
// any pointer may be null.
struct StepSaves {
    float* emit_vel[3];      // velocity after handle_emitters
    float* emit_dens;        // smoke after handle_emitters (nch * ncell)
    float* emit_temp;
    float* force_vel[3];     // velocity after advection (+ buoyancy), before vorticity confinement
    float* proj_vel[3];      // velocity after the projection update
    int vcycles;             // out: V-cycles (or refinement steps) the solve ran
    // the projection's result: pres_save receives the solved pressure (FP64
    // with the mixed-precision solve, else FP32); with pres_restore set the
    // step skips the solve and takes that pressure and vcycles_restore instead
    void* pres_save;
    const void* pres_restore;
    int vcycles_restore;
};
int run_step(ss_sim* s, const ss_params* p, cudaStream_t st, StepSaves* saves);
// z planes a thread (or a block) of a z-marching kernel takes: at most
// max_planes (the figure tuned at 256^3), and few enough that small grids
// still fill the GPU - about `target` blocks for `tiles` blocks a z slab
inline int z_planes(long long tiles, int nz, int max_planes, int min_planes = 1, long long target = 148LL * 8) {
    long long p = (tiles * nz + target - 1) / target;
    if (p > max_planes) p = max_planes;
    if (p < min_planes) p = min_planes;
    return (int)p;
}
int launch_force_field(ss_sim* s, const StepConsts& c, cudaStream_t st);
int launch_vorticity_field(ss_sim* s, const StepConsts& c, const float* const vel[3], float* out, cudaStream_t st);

// adjoint kernels (k_adjoint.cu)
struct AdjScratch {
    float* pbar[SS_MAX_LEVELS];
    float* bbar[SS_MAX_LEVELS];
    float* T[SS_MAX_LEVELS];
    // response matrix of the coarsest level's sweeps (launch_coarse_response);
    // null: the bottom solve's adjoint transposes the sweeps one by one
    const float* cresp;
};
// coarsest levels up to this many cells get a response matrix (4 MiB)
constexpr int kCoarseResponseMax = 1024;
// lanes of the coarsest level's matrix product (k_mg.cu, coarse_parts): one
// 16-block cluster of 1024 threads
constexpr int kProductLanes = 16384;
int launch_coarse_response(ss_sim* s, int iters, float* D, cudaStream_t st);
int update_coarse_matrix(ss_sim* s, const ss_mg_schedule& mg, cudaStream_t st);
// Scratch of the deterministic (owner-computes) adjoint scatters; a null
// AdjOwner selects the atomic scatter-adds.
struct AdjOwner {
    void* tr[3];   // float4 per face of each axis: clamped back-traced point, w = weight of the source (the smoke pass uses tr[0])
    void* vq[3];   // float4 per face of each axis: position gradient, w = value the face keeps
    int* win;      // tap reaches: 6 per face axis (the smoke pass uses the first 6); win[23]: error word
};
int adj_force_field(ss_sim* s, const StepConsts& c, float* const ub[3], float* grad, cudaStream_t st,
                    const AdjOwner* own = nullptr);
#define TRY_ADJ(x)                          \
    do {                                    \
        int _rc = (x);                      \
        if (_rc != SS_OK) return _rc;       \
    } while (0)
int adj_advect_smoke(ss_sim* s, const StepConsts& c, const float* const vel[3], const float* dens, const float* temp,
                     const float* dout, const float* tout, float* din, float* tin, float* vcb, float* const vb[3],
                     cudaStream_t st, const AdjOwner* own = nullptr);
int adj_update(ss_sim* s, const StepConsts& c, float* const vb[3], float* pbar, cudaStream_t st);
int adj_divergence(ss_sim* s, const float* dbar, float* const vb[3], cudaStream_t st);
int adj_v_cycle(ss_sim* s, const StepConsts& c, const ss_mg_schedule& mg, const AdjScratch& w, cudaStream_t st);
int adj_apply_laplacian(ss_sim* s, const float* rb, float k, float* pbar, cudaStream_t st);
int adj_vorticity(ss_sim* s, const StepConsts& c, const float* vort, float* const vb[3], float* wdir, float* dbar,
                  float* wbar, cudaStream_t st);
int adj_advect_velocity(ss_sim* s, const StepConsts& c, bool buoy, const float* const vel[3], const float* dens,
                        const float* temp, const float* const gin[3], float* const vb[3], float* dbar, float* tbar,
                        cudaStream_t st, const AdjOwner* own = nullptr);
int adj_buoyancy(ss_sim* s, const StepConsts& c, float* vbar, float* dbar, float* tbar, cudaStream_t st,
                 const AdjOwner* own = nullptr);
int adj_emitters(ss_sim* s, const StepConsts& c, int forced, float* const vb[3], double* fpart, double* fout,
                 const ss_emitter* em, int ne, cudaStream_t st);
int adj_force_blocks(const ss_sim* s);

// ---- scene kernels (k_scene.cu) ----
int launch_rasterize(ss_sim* s, cudaStream_t st);
int launch_flags(ss_sim* s, cudaStream_t st);
int launch_fill(float* a, size_t n, float v, cudaStream_t st);

// ---- reductions ----
int launch_reduce_final(ss_sim* s, int nblocks, int slot, cudaStream_t st);

}  // namespace ss
