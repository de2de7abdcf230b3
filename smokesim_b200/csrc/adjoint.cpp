// adjoint.cpp - reverse pass of a rollout, with checkpointing (C ABI).
//
// The forward rollout saves the full simulation state every `every` steps.
// The reverse pass walks the segments backwards: it restores a segment's
// checkpoint and recomputes the segment once, keeping for each step the
// intermediate velocities, smoke and vorticity its stages read (run_step's
// StepSaves); then, last step first, it applies the stages' adjoint kernels
// (k_adjoint.cu) in reverse stage order.  The forward pass keeps the last
// segment's intermediates itself, so every step but those is run twice
// (forward pass, segment recomputation) plus its adjoint - and with one
// segment (checkpoint_every >= nsteps) nothing is recomputed.  Memory is
// nsteps/every states plus `every` steps of intermediates.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ss_internal.h"

using namespace ss;

namespace {

struct State {
    float* vel[3] = {nullptr, nullptr, nullptr};
    float* v_other = nullptr;   // the y ping-pong partner (stand-alone buoyancy leaves faces unwritten)
    float* dens = nullptr;
    float* temp = nullptr;
    float* p = nullptr;
    double* p64 = nullptr;      // the mixed solve's FP64 pressure (allocated when a mixed forward saves one)
    bool p64_valid = false;
    std::vector<ss_emitter> em;
    std::vector<ss_obstacle> ob;
};

// what one step's adjoint reads of its forward pass
struct Record {
    float* ue[3] = {nullptr, nullptr, nullptr};   // velocity after handle_emitters
    float* ua[3] = {nullptr, nullptr, nullptr};   // after advection (+ buoyancy)
    float* un[3] = {nullptr, nullptr, nullptr};   // after the projection update
    float* dens_e = nullptr;                      // smoke after handle_emitters
    float* temp_e = nullptr;
    float* vort = nullptr;                        // vorticity of ua
    int vcycles = 0;
    std::vector<ss_emitter> em;                   // emitter records the step used
};

}  // namespace

struct ss_adjoint {
    ss_sim* s = nullptr;
    int n = 0, every = 1;
    std::vector<State> ckpt;
    std::vector<Record> rec;
    std::vector<float> forces;
    float* ub[3] = {}, *ub2[3] = {};
    float* db = nullptr, *db2 = nullptr, *tb = nullptr, *tb2 = nullptr;
    AdjScratch w{};
    float* vc3 = nullptr, *wdir = nullptr, *dbar3 = nullptr, *wbar = nullptr;
    double* fpart = nullptr;
    double* fgrad = nullptr;   // nsteps * 3
    float* ffgrad = nullptr;   // dL/d(coarse force field), 3 * ff_n^3
    int ffgrad_n = 0;          // ff_n that ffgrad was sized and last filled for
    std::vector<void*> allocs;
    long long launches = 0, ckpt_bytes = 0, work_bytes = 0;
    float* cresp = nullptr;        // response matrix of the coarsest level's sweeps, cresp_n^2
    int cresp_n = 0;
    AdjOwner own{};                // owner-computes scratch (allocated when first enabled)
    bool deterministic = false;    // owner-computes scatters instead of atomics
    bool forward_done = false;
    bool last_recorded = false;   // rec holds the last segment, written by the forward pass
    // optional: the solved pressure of every step (FP64 with the mixed solve),
    // so that recomputing a segment replays it instead of solving again
    bool store_p = false;
    std::vector<void*> pstore;
    std::vector<int> pstore_vc;
    size_t pstore_elem = 0;        // bytes per cell of the stored pressures
    long long pstore_bytes = 0;
    // the transposed V-cycles of one step, recorded once as a CUDA graph
    cudaGraphExec_t vgraph = nullptr;
    unsigned char vkey[64] = {};
    long long vlaunches = 0;
};

static int amalloc(ss_adjoint* A, void** p, size_t bytes, long long* counter) {
    cudaError_t e = cudaMalloc(p, bytes > 0 ? bytes : 16);
    if (e != cudaSuccess) return check_cuda(e, "cudaMalloc (adjoint)");
    A->allocs.push_back(*p);
    *counter += (long long)bytes;
    return SS_OK;
}

static void free_adjoint(ss_adjoint* A) {
    if (A->vgraph) cudaGraphExecDestroy(A->vgraph);
    cudaFree(A->ffgrad);
    for (void* p : A->allocs) cudaFree(p);
    for (void* p : A->pstore) cudaFree(p);
    delete A;
}

static int alloc_state(ss_adjoint* A, State& S) {
    ss_sim* s = A->s;
    for (int d = 0; d < s->dim; ++d) TRY_ADJ(amalloc(A, (void**)&S.vel[d], s->nv[d] * 4, &A->ckpt_bytes));
    TRY_ADJ(amalloc(A, (void**)&S.v_other, s->nv[1] * 4, &A->ckpt_bytes));
    TRY_ADJ(amalloc(A, (void**)&S.dens, s->ncell * s->nch * 4, &A->ckpt_bytes));
    TRY_ADJ(amalloc(A, (void**)&S.temp, s->ncell * 4, &A->ckpt_bytes));
    TRY_ADJ(amalloc(A, (void**)&S.p, s->ncell * 4, &A->ckpt_bytes));
    return SS_OK;
}

static int alloc_record(ss_adjoint* A, Record& R) {
    ss_sim* s = A->s;
    for (int d = 0; d < s->dim; ++d) {
        TRY_ADJ(amalloc(A, (void**)&R.ue[d], s->nv[d] * 4, &A->ckpt_bytes));
        TRY_ADJ(amalloc(A, (void**)&R.ua[d], s->nv[d] * 4, &A->ckpt_bytes));
        TRY_ADJ(amalloc(A, (void**)&R.un[d], s->nv[d] * 4, &A->ckpt_bytes));
    }
    TRY_ADJ(amalloc(A, (void**)&R.dens_e, s->ncell * s->nch * 4, &A->ckpt_bytes));
    TRY_ADJ(amalloc(A, (void**)&R.temp_e, s->ncell * 4, &A->ckpt_bytes));
    TRY_ADJ(amalloc(A, (void**)&R.vort, s->ncell * (s->dim == 3 ? 4 : 1) * 4, &A->ckpt_bytes));
    return SS_OK;
}

static int copy_d2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    return check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st), "state copy");
}

static int save_state(ss_adjoint* A, State& S, cudaStream_t st) {
    ss_sim* s = A->s;
    for (int d = 0; d < s->dim; ++d) TRY_ADJ(copy_d2d(S.vel[d], s->vel[d][s->vi[d]], s->nv[d] * 4, st));
    TRY_ADJ(copy_d2d(S.v_other, s->vel[1][1 - s->vi[1]], s->nv[1] * 4, st));
    TRY_ADJ(copy_d2d(S.dens, s->dens[s->si], s->ncell * s->nch * 4, st));
    TRY_ADJ(copy_d2d(S.temp, s->temp[s->si], s->ncell * 4, st));
    TRY_ADJ(copy_d2d(S.p, s->p[0], s->ncell * 4, st));
    // the mixed solve warm-starts from its FP64 pressure: keep it exactly, so
    // that a recomputed segment repeats the forward pass bit for bit
    S.p64_valid = s->p64_valid && s->p64;
    if (S.p64_valid) {
        if (!S.p64) TRY_ADJ(amalloc(A, (void**)&S.p64, s->ncell * sizeof(double), &A->ckpt_bytes));
        TRY_ADJ(copy_d2d(S.p64, s->p64, s->ncell * sizeof(double), st));
    }
    S.em = s->em;
    S.ob = s->ob;
    return SS_OK;
}

static int restore_state(ss_sim* s, const State& S, cudaStream_t st) {
    for (int d = 0; d < s->dim; ++d) TRY_ADJ(copy_d2d(s->vel[d][s->vi[d]], S.vel[d], s->nv[d] * 4, st));
    TRY_ADJ(copy_d2d(s->vel[1][1 - s->vi[1]], S.v_other, s->nv[1] * 4, st));
    TRY_ADJ(copy_d2d(s->dens[s->si], S.dens, s->ncell * s->nch * 4, st));
    TRY_ADJ(copy_d2d(s->temp[s->si], S.temp, s->ncell * 4, st));
    TRY_ADJ(copy_d2d(s->p[0], S.p, s->ncell * 4, st));
    s->p64_valid = 0;
    if (S.p64_valid && s->p64) {
        TRY_ADJ(copy_d2d(s->p64, S.p64, s->ncell * sizeof(double), st));
        s->p64_valid = 1;
        s->prev_ok = 0;
    }
    s->em = S.em;
    s->ob = S.ob;
    return SS_OK;
}

static void set_force(ss_adjoint* A, int k) {
    for (int d = 0; d < 3; ++d) A->s->force[d] = A->forces[3 * (size_t)k + d];
}

static int check_adjoint_params(const ss_adjoint* A, const ss_params* p) {
    if (!A || !p) return set_error(SS_E_INVALID, "NULL argument");
    if (p->stage_mask & SS_STAGE_RESOLVE_PRESSURE) {
        if (p->mg.ref_quirks) return set_error(SS_E_UNSUPPORTED, "the adjoint transposes the corrected operators (ref_quirks = 0)");
        // The mixed-precision solve's refinement steps are, in exact
        // arithmetic, the same V-cycles on the pressure as the FP32 solve's
        // (a linear V-cycle applied to the correction with the residual as its
        // right-hand side), so the recorded count of them is transposed with
        // the FP32 adjoint V-cycle: the gradient of the exact-arithmetic map at
        // the states the mixed forward produced.
        if (p->mg.precision != SS_PREC_FP32 && p->mg.precision != SS_PREC_MIXED &&
            p->mg.precision != SS_PREC_MIXED_BF16)
            return set_error(SS_E_INVALID, "unknown precision mode");
        // the extrapolated warm start makes a step's pressure depend on the
        // two before it; the reverse pass transposes the one-step warm start
        if (p->mg.warm_start != 0)
            return set_error(SS_E_UNSUPPORTED, "the adjoint needs warm_start = 0 (the previous step's pressure)");
    }
    return SS_OK;
}

// The transposed V-cycles of one step (adjoint of the right-hand side in
// w.bbar[0], of the warm-start pressure in w.pbar[0]).  Every step runs the
// same launches on the same buffers, so they are recorded once as a CUDA
// graph and replayed (directly on the legacy stream or inside a caller's
// capture).
static int adj_solve(ss_adjoint* A, const ss_params* p, const StepConsts& c, int vcycles, cudaStream_t st) {
    ss_sim* s = A->s;
    auto body = [&]() -> int {
        TRY_ADJ(check_cuda(cudaMemsetAsync(A->w.bbar[0], 0, s->ncell * 4, st), "memset"));
        for (int i = 0; i < vcycles; ++i) TRY_ADJ(adj_v_cycle(s, c, p->mg, A->w, st));
        return SS_OK;
    };
    if (st == nullptr) return body();
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    TRY_ADJ(check_cuda(cudaStreamIsCapturing(st, &cs), "cudaStreamIsCapturing"));
    if (cs != cudaStreamCaptureStatusNone) return body();
    struct Key { int vcycles; ss_mg_schedule mg; float dt, rho; } key;
    std::memset(&key, 0, sizeof key);
    key.vcycles = vcycles; key.mg = p->mg; key.dt = p->time_step; key.rho = p->density;
    static_assert(sizeof(Key) <= sizeof(A->vkey), "graph key size");
    unsigned char kb[sizeof(A->vkey)] = {};
    std::memcpy(kb, &key, sizeof key);
    if (A->vgraph && std::memcmp(kb, A->vkey, sizeof kb) == 0) {
        s->nlaunch += A->vlaunches;
        return check_cuda(cudaGraphLaunch(A->vgraph, st), "cudaGraphLaunch");
    }
    if (A->vgraph) {
        cudaGraphExecDestroy(A->vgraph);
        A->vgraph = nullptr;
    }
    const long long before = s->nlaunch;
    TRY_ADJ(check_cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture"));
    const int rc = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc != SS_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    TRY_ADJ(check_cuda(e, "cudaStreamEndCapture"));
    const cudaError_t ei = cudaGraphInstantiate(&A->vgraph, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        A->vgraph = nullptr;
        return check_cuda(ei, "cudaGraphInstantiate");
    }
    std::memcpy(A->vkey, kb, sizeof kb);
    A->vlaunches = s->nlaunch - before;
    return check_cuda(cudaGraphLaunch(A->vgraph, st), "cudaGraphLaunch");
}

// Size the per-step pressure store for this forward pass's precision.
static int ensure_pstore(ss_adjoint* A, const ss_params* p) {
    if (!A->store_p || !(p->stage_mask & SS_STAGE_RESOLVE_PRESSURE)) return SS_OK;
    const size_t elem = p->mg.precision != SS_PREC_FP32 ? sizeof(double) : sizeof(float);
    if (A->pstore_elem == elem && (int)A->pstore.size() == A->n) return SS_OK;
    for (void* q : A->pstore) cudaFree(q);
    A->pstore.clear();
    A->pstore_bytes = 0;
    A->pstore_elem = 0;
    A->pstore.assign(A->n, nullptr);
    A->pstore_vc.assign(A->n, 0);
    for (int k = 0; k < A->n; ++k) {
        const cudaError_t e = cudaMalloc(&A->pstore[k], A->s->ncell * elem);
        if (e != cudaSuccess) {
            for (void* q : A->pstore) cudaFree(q);
            A->pstore.clear();
            return check_cuda(e, "cudaMalloc(pressure store)");
        }
        A->pstore_bytes += (long long)(A->s->ncell * elem);
    }
    A->pstore_elem = elem;
    return SS_OK;
}

// the pressure-store part of a step's saves: save in the forward pass,
// replay when a segment is recomputed
static void pstore_saves(ss_adjoint* A, int k, bool replay, StepSaves& sv) {
    if (!A->store_p || A->pstore.empty()) return;
    if (replay) {
        sv.pres_restore = A->pstore[k];
        sv.vcycles_restore = A->pstore_vc[k];
    } else {
        sv.pres_save = A->pstore[k];
    }
}

// Forward step k keeping what its adjoint reads.
static int record_step(ss_adjoint* A, const ss_params* p, int k, Record& R, cudaStream_t st, bool replay = false) {
    ss_sim* s = A->s;
    StepSaves sv{};
    pstore_saves(A, k, replay, sv);
    for (int d = 0; d < s->dim; ++d) {
        sv.emit_vel[d] = R.ue[d];
        sv.force_vel[d] = R.ua[d];
        sv.proj_vel[d] = R.un[d];
    }
    sv.emit_dens = R.dens_e;
    sv.emit_temp = R.temp_e;
    set_force(A, k);
    TRY_ADJ(run_step(s, p, st, &sv));
    R.vcycles = sv.vcycles;
    if (!replay && !A->pstore.empty()) A->pstore_vc[k] = sv.vcycles;
    R.em = s->em;
    if (p->stage_mask & SS_STAGE_APPLY_VORTICITY) {
        const float* ua[3] = {R.ua[0], R.ua[1], R.ua[2]};
        TRY_ADJ(launch_vorticity_field(s, make_consts(s, p), ua, R.vort, st));
    }
    return SS_OK;
}

// Reverse of one step from its record: on entry ub/db/tb/pbar[0] hold the
// adjoint of the step's end state, on return that of its start state.
static int adj_step(ss_adjoint* A, const ss_params* p, int k, const Record& R, cudaStream_t st) {
    ss_sim* s = A->s;
    const StepConsts c = make_consts(s, p);
    const int m = p->stage_mask;
    const size_t ncell = s->ncell;
    const AdjOwner* own = A->deterministic ? &A->own : nullptr;
    if (m & SS_STAGE_ADVECT_SMOKE) {
        TRY_ADJ(check_cuda(cudaMemsetAsync(A->db2, 0, ncell * s->nch * 4, st), "memset"));
        TRY_ADJ(check_cuda(cudaMemsetAsync(A->tb2, 0, ncell * 4, st), "memset"));
        const float* vel[3] = {R.un[0], R.un[1], R.un[2]};
        TRY_ADJ(adj_advect_smoke(s, c, vel, R.dens_e, R.temp_e, A->db, A->tb, A->db2, A->tb2, A->vc3, A->ub, st, own));
        std::swap(A->db, A->db2);
        std::swap(A->tb, A->tb2);
    }
    if (m & SS_STAGE_UPDATE_VELOCITIES) TRY_ADJ(adj_update(s, c, A->ub, A->w.pbar[0], st));
    if (m & SS_STAGE_RESOLVE_PRESSURE) {
        TRY_ADJ(adj_solve(A, p, c, R.vcycles, st));
        TRY_ADJ(adj_divergence(s, A->w.bbar[0], A->ub, st));
    }
    if (m & SS_STAGE_APPLY_VORTICITY) TRY_ADJ(adj_vorticity(s, c, R.vort, A->ub, A->wdir, A->dbar3, A->wbar, st));
    if (m & SS_STAGE_ADVECT_VELOCITIES) {
        for (int d = 0; d < s->dim; ++d)
            TRY_ADJ(check_cuda(cudaMemsetAsync(A->ub2[d], 0, s->nv[d] * 4, st), "memset"));
        const float* vel[3] = {R.ue[0], R.ue[1], R.ue[2]};
        const float* gin[3] = {A->ub[0], A->ub[1], A->ub[2]};
        TRY_ADJ(adj_advect_velocity(s, c, (m & SS_STAGE_APPLY_BUOYANCY) != 0, vel, R.dens_e, R.temp_e, gin, A->ub2,
                                    A->db, A->tb, st, own));
        for (int d = 0; d < 3; ++d) std::swap(A->ub[d], A->ub2[d]);
    } else if (m & SS_STAGE_APPLY_BUOYANCY) {
        TRY_ADJ(adj_buoyancy(s, c, A->ub[1], A->db, A->tb, st, own));
    }
    if (m & SS_STAGE_HANDLE_EMITTERS) {
        // the force field came after the emitters: its transpose first
        if (s->ff_n > 0) TRY_ADJ(adj_force_field(s, c, A->ub, A->ffgrad, st, own));
        // the emitter records of this step (their status changes over time)
        if (!R.em.empty())
            TRY_ADJ(check_cuda(cudaMemcpyAsync(s->d_em, R.em.data(), R.em.size() * sizeof(ss_emitter),
                                               cudaMemcpyHostToDevice, st), "emitter records"));
        TRY_ADJ(adj_emitters(s, c, 1, A->ub, A->fpart, A->fgrad + 3 * (size_t)k, R.em.data(), (int)R.em.size(), st));
    }
    return SS_OK;
}

extern "C" {

int ss_set_emitter_force(ss_sim* s, const float force[3]) {
    if (!s || !force) return set_error(SS_E_INVALID, "NULL argument");
    for (int d = 0; d < 3; ++d)
        if (!std::isfinite(force[d])) return set_error(SS_E_NONFINITE, "force");
    for (int d = 0; d < 3; ++d) s->force[d] = d < s->dim ? force[d] : 0.f;
    return SS_OK;
}

int ss_adjoint_create(ss_sim* s, int nsteps, int every, ss_adjoint** out) {
    if (!s || !out || nsteps < 1) return set_error(SS_E_INVALID, "NULL argument or nsteps < 1");
    if (every <= 0) every = 1;
    if (every > nsteps) every = nsteps;
    ss_adjoint* A = new ss_adjoint();
    A->s = s;
    A->n = nsteps;
    A->every = every;
    A->forces.assign((size_t)nsteps * 3, 0.f);
    const int nseg = (nsteps + every - 1) / every;
    A->ckpt.resize(nseg);
    A->rec.resize(every);
    int rc = SS_OK;
    for (auto& S : A->ckpt) rc = rc ? rc : alloc_state(A, S);
    for (auto& R : A->rec) rc = rc ? rc : alloc_record(A, R);
    auto W = [&](void** p, size_t bytes) { if (!rc) rc = amalloc(A, p, bytes, &A->work_bytes); };
    for (int d = 0; d < s->dim; ++d) {
        W((void**)&A->ub[d], s->nv[d] * 4);
        W((void**)&A->ub2[d], s->nv[d] * 4);
    }
    W((void**)&A->db, s->ncell * s->nch * 4);
    W((void**)&A->db2, s->ncell * s->nch * 4);
    W((void**)&A->tb, s->ncell * 4);
    W((void**)&A->tb2, s->ncell * 4);
    W((void**)&A->vc3, s->ncell * 3 * 4);
    W((void**)&A->wdir, s->ncell * 3 * 4);
    W((void**)&A->dbar3, s->ncell * 3 * 4);
    W((void**)&A->wbar, s->ncell * 3 * 4);
    for (int l = 0; l < s->levels; ++l) {
        const size_t n = (size_t)s->lv[l].n[0] * s->lv[l].n[1] * s->lv[l].n[2];
        W((void**)&A->w.pbar[l], n * 4);
        W((void**)&A->w.bbar[l], n * 4);
        W((void**)&A->w.T[l], n * 4);
    }
    W((void**)&A->fpart, (size_t)adj_force_blocks(s) * 3 * sizeof(double));
    W((void**)&A->fgrad, (size_t)nsteps * 3 * sizeof(double));
    // the bottom solve's adjoint applies the coarsest sweeps as one matrix
    // (SMOKESIM_ADJ_COARSE_SWEEPS=1 transposes them sweep by sweep instead)
    {
        const ss::Level& lc = s->lv[s->levels - 1];
        const long long nc = (long long)lc.n[0] * lc.n[1] * lc.n[2];
        const char* e = getenv("SMOKESIM_ADJ_COARSE_SWEEPS");
        if (s->levels >= 2 && nc <= kCoarseResponseMax && !(e && atoi(e) != 0)) {
            W((void**)&A->cresp, (size_t)(nc * nc) * 4);
            A->cresp_n = (int)nc;
        }
    }
    if (rc) {
        free_adjoint(A);
        return rc;
    }
    *out = A;
    return SS_OK;
}

int ss_adjoint_destroy(ss_adjoint* A) {
    if (!A) return set_error(SS_E_INVALID, "NULL handle");
    cudaDeviceSynchronize();
    free_adjoint(A);
    return SS_OK;
}

int ss_adjoint_forward(ss_adjoint* A, const ss_params* p, const float* forces, void* stream) {
    TRY_ADJ(check_adjoint_params(A, p));
    ss_sim* s = A->s;
    cudaStream_t st = (cudaStream_t)stream;
    if (forces) {
        for (size_t i = 0; i < A->forces.size(); ++i)
            if (!std::isfinite(forces[i])) return set_error(SS_E_NONFINITE, "force");
        std::memcpy(A->forces.data(), forces, A->forces.size() * sizeof(float));
    } else {
        std::fill(A->forces.begin(), A->forces.end(), 0.f);
    }
    s->nlaunch = 0;
    A->last_recorded = false;
    TRY_ADJ(ensure_pstore(A, p));
    const int last0 = ((A->n - 1) / A->every) * A->every;   // first step of the last segment
    for (int k = 0; k < A->n; ++k) {
        if (k % A->every == 0) TRY_ADJ(save_state(A, A->ckpt[k / A->every], st));
        // the last segment keeps its intermediates now: the reverse pass
        // starts there without recomputing it
        if (k >= last0) TRY_ADJ(record_step(A, p, k, A->rec[k - last0], st));
        else {
            set_force(A, k);
            StepSaves sv{};
            pstore_saves(A, k, false, sv);
            TRY_ADJ(run_step(s, p, st, sv.pres_save ? &sv : nullptr));
            if (sv.pres_save) A->pstore_vc[k] = sv.vcycles;
        }
    }
    for (int d = 0; d < 3; ++d) s->force[d] = 0.f;
    A->forward_done = true;
    A->last_recorded = true;
    return check_cuda(cudaGetLastError(), "adjoint forward");
}

int ss_adjoint_backward(ss_adjoint* A, const ss_params* p, const float* grad_density, const float* grad_temperature,
                        const float* const grad_velocity[3], float* grad_forces, void* stream) {
    TRY_ADJ(check_adjoint_params(A, p));
    if (!A->forward_done) return set_error(SS_E_INVALID, "ss_adjoint_forward has not run");
    ss_sim* s = A->s;
    cudaStream_t st = (cudaStream_t)stream;
    s->nlaunch = 0;
    // adjoint of the final state
    for (int d = 0; d < s->dim; ++d) {
        if (grad_velocity && grad_velocity[d]) TRY_ADJ(copy_d2d(A->ub[d], grad_velocity[d], s->nv[d] * 4, st));
        else TRY_ADJ(check_cuda(cudaMemsetAsync(A->ub[d], 0, s->nv[d] * 4, st), "memset"));
    }
    if (grad_density) TRY_ADJ(copy_d2d(A->db, grad_density, s->ncell * s->nch * 4, st));
    else TRY_ADJ(check_cuda(cudaMemsetAsync(A->db, 0, s->ncell * s->nch * 4, st), "memset"));
    if (grad_temperature) TRY_ADJ(copy_d2d(A->tb, grad_temperature, s->ncell * 4, st));
    else TRY_ADJ(check_cuda(cudaMemsetAsync(A->tb, 0, s->ncell * 4, st), "memset"));
    TRY_ADJ(check_cuda(cudaMemsetAsync(A->w.pbar[0], 0, s->ncell * 4, st), "memset"));
    TRY_ADJ(check_cuda(cudaMemsetAsync(A->fgrad, 0, (size_t)A->n * 3 * sizeof(double), st), "memset"));
    if (s->ff_n > 0) {
        const size_t nff = (size_t)3 * s->ff_n * s->ff_n * s->ff_n;
        if (A->ffgrad_n != s->ff_n) {
            cudaFree(A->ffgrad);
            A->ffgrad = nullptr;
            A->ffgrad_n = 0;
            TRY_ADJ(check_cuda(cudaMalloc((void**)&A->ffgrad, nff * sizeof(float)), "cudaMalloc(force field gradient)"));
            A->ffgrad_n = s->ff_n;
        }
        TRY_ADJ(check_cuda(cudaMemsetAsync(A->ffgrad, 0, nff * sizeof(float), st), "memset"));
    }
    if (A->deterministic) TRY_ADJ(check_cuda(cudaMemsetAsync(A->own.win, 0, 24 * sizeof(int), st), "memset"));
    // this call's coarsest-level map (schedule and solid fractions as they are now)
    A->w.cresp = nullptr;
    if (A->cresp) {
        TRY_ADJ(launch_coarse_response(s, p->mg.n_coarse, A->cresp, st));
        A->w.cresp = A->cresp;
    }
    const int nseg = (A->n + A->every - 1) / A->every;
    for (int sg = nseg - 1; sg >= 0; --sg) {
        const int k0 = sg * A->every, k1 = std::min(A->n, k0 + A->every);
        if (!(sg == nseg - 1 && A->last_recorded)) {
            TRY_ADJ(restore_state(s, A->ckpt[sg], st));
            for (int k = k0; k < k1; ++k) TRY_ADJ(record_step(A, p, k, A->rec[k - k0], st, true));
        }
        A->last_recorded = false;   // rec now holds this segment
        for (int k = k1 - 1; k >= k0; --k) TRY_ADJ(adj_step(A, p, k, A->rec[k - k0], st));
    }
    TRY_ADJ(restore_state(s, A->ckpt[0], st));
    for (int d = 0; d < 3; ++d) s->force[d] = 0.f;
    A->launches = s->nlaunch;
    // the force-field gradient is read back with a plain copy afterwards
    if (s->ff_n > 0) TRY_ADJ(check_cuda(cudaStreamSynchronize(st), "adjoint sync"));
    if (grad_forces) {
        std::vector<double> g((size_t)A->n * 3);
        TRY_ADJ(check_cuda(cudaMemcpyAsync(g.data(), A->fgrad, g.size() * sizeof(double), cudaMemcpyDeviceToHost, st),
                           "force gradient"));
        TRY_ADJ(check_cuda(cudaStreamSynchronize(st), "adjoint sync"));
        for (size_t i = 0; i < g.size(); ++i) grad_forces[i] = (float)g[i];
    }
    if (A->deterministic) {
        int err = 0;
        TRY_ADJ(check_cuda(cudaMemcpyAsync(&err, A->own.win + 23, sizeof(int), cudaMemcpyDeviceToHost, st), "reach flag"));
        TRY_ADJ(check_cuda(cudaStreamSynchronize(st), "adjoint sync"));
        if (err)
            return set_error(SS_E_INVALID, "a back-traced point lies more than 8 cells from its source: the "
                                           "owner-computes scatters enumerate at most 8; use the atomic ones");
    }
    return check_cuda(cudaGetLastError(), "adjoint backward");
}

int ss_adjoint_field_device_ptr(ss_adjoint* A, int field, void** dptr, size_t* count) {
    if (!A || !dptr) return set_error(SS_E_INVALID, "NULL argument");
    ss_sim* s = A->s;
    void* d = nullptr;
    size_t n = 0;
    switch (field) {
    case SS_FIELD_VX: d = A->ub[0]; n = s->nv[0]; break;
    case SS_FIELD_VY: d = A->ub[1]; n = s->nv[1]; break;
    case SS_FIELD_VZ: if (s->dim == 3) { d = A->ub[2]; n = s->nv[2]; } break;
    case SS_FIELD_DENSITY: d = A->db; n = s->ncell * s->nch; break;
    case SS_FIELD_TEMPERATURE: d = A->tb; n = s->ncell; break;
    case SS_FIELD_PRESSURE: d = A->w.pbar[0]; n = s->ncell; break;
    default: break;
    }
    if (!d) return set_error(SS_E_INVALID, "no adjoint for this field");
    *dptr = d;
    if (count) *count = n;
    return SS_OK;
}

int ss_adjoint_get_field(ss_adjoint* A, int field, float* dst, size_t count, int dst_on_device, void* stream) {
    if (!A || !dst) return set_error(SS_E_INVALID, "NULL argument");
    void* d = nullptr;
    size_t n = 0;
    TRY_ADJ(ss_adjoint_field_device_ptr(A, field, &d, &n));
    if (count != n) return set_error(SS_E_INVALID, "element count does not match the field");
    cudaStream_t st = (cudaStream_t)stream;
    TRY_ADJ(check_cuda(cudaMemcpyAsync(dst, d, n * sizeof(float), dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st),
                       "adjoint field"));
    if (!dst_on_device) TRY_ADJ(check_cuda(cudaStreamSynchronize(st), "adjoint field sync"));
    return SS_OK;
}

int ss_adjoint_force_field_grad(ss_adjoint* A, float* dst, size_t count) {
    if (!A || !dst) return set_error(SS_E_INVALID, "NULL argument");
    const int n = A->ffgrad_n;
    if (n <= 0 || !A->ffgrad) return set_error(SS_E_INVALID, "no force field gradient (no field, or no backward pass yet)");
    const size_t nff = (size_t)3 * n * n * n;
    if (count != nff) return set_error(SS_E_INVALID, "count differs from 3 * n^3 of the force field");
    TRY_ADJ(check_cuda(cudaMemcpy(dst, A->ffgrad, nff * sizeof(float), cudaMemcpyDeviceToHost), "force field gradient"));
    return SS_OK;
}

int ss_adjoint_set_deterministic(ss_adjoint* A, int on) {
    if (!A) return set_error(SS_E_INVALID, "NULL handle");
    if (on && !A->own.win) {
        ss_sim* s = A->s;
        for (int d = 0; d < s->dim; ++d) {
            TRY_ADJ(amalloc(A, &A->own.tr[d], s->nv[d] * 16, &A->work_bytes));
            TRY_ADJ(amalloc(A, &A->own.vq[d], s->nv[d] * 16, &A->work_bytes));
        }
        TRY_ADJ(amalloc(A, (void**)&A->own.win, 24 * sizeof(int), &A->work_bytes));
    }
    A->deterministic = on != 0;
    return SS_OK;
}

int ss_adjoint_set_pressure_store(ss_adjoint* A, int on) {
    if (!A) return set_error(SS_E_INVALID, "NULL handle");
    A->store_p = on != 0;
    if (!A->store_p) {
        for (void* q : A->pstore) cudaFree(q);
        A->pstore.clear();
        A->pstore_vc.clear();
        A->pstore_bytes = 0;
        A->pstore_elem = 0;
    }
    A->forward_done = false;   // the next backward needs a forward that filled (or not) the store
    return SS_OK;
}

int ss_adjoint_info(ss_adjoint* A, long long* launches, long long* ckpt_bytes, long long* work_bytes) {
    if (!A) return set_error(SS_E_INVALID, "NULL handle");
    if (launches) *launches = A->launches;
    if (ckpt_bytes) *ckpt_bytes = A->ckpt_bytes + A->pstore_bytes;
    if (work_bytes) *work_bytes = A->work_bytes;
    return SS_OK;
}

}  // extern "C"
