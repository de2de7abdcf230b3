// api.cpp - the C ABI of libsmokesim.so (include/smokesim.h).
//
// Host orchestration of the smoke step: the order of run_physics_step
// (common/physics/physics.c:72-101), the recursive V-cycle of
// common/physics/grid.c:177-209, the emitter clock of
// update_emitters_status.comp and the rigid obstacles of obstacle_update.comp
// (both tiny, run on the host), and device memory ownership.
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "ss_internal.h"

using namespace ss;

namespace ss {

static thread_local std::string g_err;

int set_error(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return SS_OK;
    return set_error(e == cudaErrorMemoryAllocation ? SS_E_OOM : SS_E_CUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

StepConsts make_consts(const ss_sim* s, const ss_params* p) {
    StepConsts c{};
    c.dt = p->time_step;
    c.rho = p->density;
    c.t_amb = p->t_ambient;
    c.alpha = p->t_weight_coeff;
    c.beta = p->t_temp_coeff;
    c.eps = p->vorticity_confinement;
    for (int d = 0; d < 3; ++d) c.wind[d] = p->wind[d];
    c.cfl = c.dt / s->h;
    c.rho_h = c.rho * s->h;
    c.dt_h = c.dt * s->h;
    c.k_upd = -c.dt / (c.rho * s->h);
    c.vort_k = s->h;
    return c;
}

}  // namespace ss

#define TRY(x)                 \
    do {                       \
        int _rc = (x);         \
        if (_rc != SS_OK) return _rc; \
    } while (0)
#define CU(x, what) TRY(check_cuda((x), what))

static cudaStream_t as_stream(void* st) { return (cudaStream_t)st; }
extern "C" {
static int check_device_error(ss_sim* s, cudaStream_t st);
}

static int dalloc(void** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return check_cuda(e, "cudaMalloc");
    return SS_OK;
}

static void free_sim(ss_sim* s) {
    if (!s) return;
    for (int d = 0; d < 3; ++d)
        for (int b = 0; b < 2; ++b) cudaFree(s->vel[d][b]);
    for (int b = 0; b < 2; ++b) { cudaFree(s->dens[b]); cudaFree(s->temp[b]); }
    cudaFree(s->solid);
    cudaFree(s->flags);
    for (int d = 0; d < 3; ++d) cudaFree(s->svel[d]);
    for (int l = 0; l < s->levels; ++l) {
        cudaFree(s->p[l]); cudaFree(s->r[l]); cudaFree(s->alpha[l]);
        cudaFree(s->p_alt[l]); cudaFree(s->r_alt[l]);
    }
    cudaFree(s->div0);
    if (s->div0r != s->div0) cudaFree(s->div0r);
    cudaFree(s->vort);
    cudaFree(s->rhs_s);
    cudaFree(s->fmask);
    cudaFree(s->rb_mask);
    cudaFree(s->rb_pw);
    cudaFree(s->p64);
    cudaFree(s->p64b);
    cudaFree(s->p64c);
    cudaFree(s->render_buf);
    cudaFree(s->ffield);
    cudaFree(s->cmat);
    cudaFree(s->cmat_alpha);
    cudaFree(s->cmat_state);
    cudaFree(s->cmat_part);
    cudaFree(s->cluster_fine);
    for (auto& g : s->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    cudaFree(s->d_scale);
    cudaFree(s->red.partial_max);
    cudaFree(s->red.ticket);
    for (int l = 0; l < SS_MAX_LEVELS; ++l) { cudaFree(s->cp[l]); cudaFree(s->cr[l]); }
    cudaFree(s->rhs_r);
    cudaFree(s->red.partial);
    cudaFree(s->red.partial2);
    cudaFree(s->red.out);
    if (s->red.host) cudaFreeHost(s->red.host);
    cudaFree(s->d_em);
    cudaFree(s->d_ob);
    cudaFree(s->d_bx);
    if (s->chain_stream) cudaStreamDestroy(s->chain_stream);
    delete s;
}

static bool finite_params(const ss_params* p) {
    const float v[] = {p->time_step, p->density, p->t_ambient, p->t_weight_coeff, p->t_temp_coeff,
                       p->vorticity_confinement, p->wind[0], p->wind[1], p->wind[2], p->current_time};
    for (float x : v)
        if (!isfinite(x)) return false;
    return isfinite(p->mg.tol);
}

static int check_params(const ss_sim* s, const ss_params* p) {
    if (!s || !p) return set_error(SS_E_INVALID, "NULL handle or params");
    if (!finite_params(p)) return set_error(SS_E_NONFINITE, "non-finite parameter");
    if (!(p->time_step > 0.f) || !(p->density > 0.f)) return set_error(SS_E_INVALID, "time_step and density must be > 0");
    if (p->mg.n_pre < 0 || p->mg.n_post < 0 || p->mg.n_coarse < 0 || p->mg.n_vcycles < 0 || p->mg.tol < 0)
        return set_error(SS_E_INVALID, "negative multigrid schedule entry");
    if (p->mg.precision != SS_PREC_FP32 && p->mg.precision != SS_PREC_MIXED && p->mg.precision != SS_PREC_MIXED_BF16)
        return set_error(SS_E_INVALID, "unknown precision mode");
    return SS_OK;
}

extern "C" {

int ss_abi_version(void) { return SS_ABI_VERSION; }

const char* ss_strerror(int status) {
    switch (status) {
    case SS_OK: return "ok";
    case SS_E_INVALID: return "invalid argument";
    case SS_E_CUDA: return "CUDA error";
    case SS_E_OOM: return "out of memory";
    case SS_E_NOT_CONVERGED: return "pressure solve did not reach the tolerance";
    case SS_E_NONFINITE: return "non-finite input";
    case SS_E_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
    }
}

const char* ss_last_error_message(void) { return g_err.c_str(); }

void ss_default_params(ss_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    // reference get_default_p_settings (common/physics/physics.c:7-20)
    p->time_step = 1.0f / 120.0f;
    p->density = 1.0f;
    p->t_ambient = 293.0f;
    p->t_temp_coeff = 1.0f;
    p->t_weight_coeff = 0.07f;
    p->vorticity_confinement = 1.0f;
    p->stage_mask = SS_STAGE_ALL;
    p->collect_stats = 0;
    // reference v_cycle schedule (common/physics/grid.c:177-190)
    p->mg.n_pre = 16;
    p->mg.n_post = 16;
    p->mg.n_coarse = 80;
    p->mg.n_vcycles = 1;
    p->mg.tol = 0.0;
    p->mg.ref_quirks = 1;
    p->mg.precision = SS_PREC_FP32;
}

int ss_create(const ss_desc* d, void* stream, ss_sim** out) {
    if (!d || !out) return set_error(SS_E_INVALID, "NULL desc or out");
    *out = nullptr;
    if (d->dim != 2 && d->dim != 3) return set_error(SS_E_INVALID, "dim must be 2 or 3");
    const int nz = d->dim == 2 ? 1 : d->n[2];
    if (d->n[0] < 3 || d->n[1] < 3 || nz < 1 || (d->dim == 3 && nz < 3))
        return set_error(SS_E_INVALID, "grid must have at least 3 cells per axis");
    if (d->dim == 2 && d->n[2] != 1) return set_error(SS_E_INVALID, "2D grids need n[2] == 1");
    const double cells = (double)(d->n[0] + 1) * (d->n[1] + 1) * (nz + 1);
    if (cells >= 2147483647.0) return set_error(SS_E_INVALID, "grid too large (face arrays must index in 31 bits)");
    if (!(d->cell_size > 0.f) || !isfinite(d->cell_size)) return set_error(SS_E_INVALID, "cell_size must be > 0");
    if (d->density_channels != 1 && d->density_channels != 3) return set_error(SS_E_INVALID, "density_channels must be 1 or 3");
    if (!isfinite(d->t_ambient)) return set_error(SS_E_NONFINITE, "t_ambient");
    cudaStream_t st = as_stream(stream);

    ss_sim* s = new ss_sim();
    s->dim = d->dim;
    s->nx = d->n[0]; s->ny = d->n[1]; s->nz = nz;
    s->nch = d->density_channels;
    s->enclosed = d->enclosed ? 1 : 0;
    s->min_coarse = d->min_coarse > 0 ? d->min_coarse : 4;
    s->h = d->cell_size;
    s->t_amb0 = d->t_ambient;
    s->ncell = (size_t)s->nx * s->ny * s->nz;
    // SMOKESIM_TMA=0 keeps the coarse-level tiled sweeps on per-thread loads
    // (the form every grid whose rows TMA cannot tile takes anyway); the
    // default 1 feeds them with TMA.  The results are the same.
    if (const char* e = getenv("SMOKESIM_TMA")) s->use_tma = atoi(e) ? 1 : 0;
    if (const char* e = getenv("SMOKESIM_COARSE_SWEEPS")) s->coarse_matrix = atoi(e) ? 0 : 1;
    // SMOKESIM_PDL=0 launches the solve's kernels without programmatic
    // dependent launch (each waits for the previous one to finish before it
    // is scheduled); the results are the same.
    if (const char* e = getenv("SMOKESIM_PDL")) s->pdl = atoi(e) ? 1 : 0;
    // SMOKESIM_CLUSTER=0 runs the mixed solve's small coarse levels as one
    // launch per level operation instead of one thread-block cluster launch;
    // the results are the same.
    if (const char* e = getenv("SMOKESIM_CLUSTER")) s->use_cluster = atoi(e) ? 1 : 0;
    // SMOKESIM_DEVICE_LOOP=0 runs the mixed solve's tolerance loop on the
    // host, reading the residual back after every refinement step, instead of
    // as conditional graph nodes whose residual kernel tests convergence on
    // the device; the results are the same.
    if (const char* e = getenv("SMOKESIM_DEVICE_LOOP")) s->device_loop = atoi(e) ? 1 : 0;
    s->nv[0] = (size_t)(s->nx + 1) * s->ny * s->nz;
    s->nv[1] = (size_t)s->nx * (s->ny + 1) * s->nz;
    s->nv[2] = s->dim == 3 ? (size_t)s->nx * s->ny * (s->nz + 1) : 0;

    // pyramid: reference gen_grid_pressure_solve_textures3d (3d/grid3d.c:45-68)
    // with the smallest level dimension as a parameter
    int dims[3] = {s->nx, s->ny, s->nz};
    int lv = 0;
    while (lv < SS_MAX_LEVELS) {
        bool ok = dims[0] >= s->min_coarse && dims[1] >= s->min_coarse && (s->dim == 2 || dims[2] >= s->min_coarse);
        if (!ok) break;
        s->lv[lv].n[0] = dims[0]; s->lv[lv].n[1] = dims[1]; s->lv[lv].n[2] = s->dim == 2 ? 1 : dims[2];
        dims[0] /= 2; dims[1] /= 2; if (s->dim == 3) dims[2] /= 2;
        ++lv;
    }
    if (lv == 0) {
        s->lv[0].n[0] = s->nx; s->lv[0].n[1] = s->ny; s->lv[0].n[2] = s->nz;
        lv = 1;
    }
    s->levels = lv;
    for (int l = 0; l < lv; ++l) {
        s->lv[l].h = s->h * (float)(1 << l);
        s->lv[l].hh = s->lv[l].h * s->lv[l].h;
    }
    s->bottom = bottom_start(s);
    s->cluster_from = coarse_cluster_from(s);

    int rc = SS_OK;
    auto A = [&](void** p, size_t bytes) { if (rc == SS_OK) rc = dalloc(p, bytes); };
    for (int dd = 0; dd < s->dim; ++dd)
        for (int b = 0; b < 2; ++b) A((void**)&s->vel[dd][b], s->nv[dd] * sizeof(float));
    for (int b = 0; b < 2; ++b) {
        A((void**)&s->dens[b], s->ncell * s->nch * sizeof(float));
        A((void**)&s->temp[b], s->ncell * sizeof(float));
    }
    A((void**)&s->solid, s->ncell);
    A((void**)&s->flags, s->ncell);
    for (int l = 0; l < lv; ++l) {
        const size_t n = (size_t)s->lv[l].n[0] * s->lv[l].n[1] * s->lv[l].n[2];
        A((void**)&s->p[l], n * sizeof(float));
        A((void**)&s->r[l], n * sizeof(float));
        if (l < s->bottom || l == 0) A((void**)&s->p_alt[l], n * sizeof(float));
        if (l > 0) A((void**)&s->alpha[l], n * sizeof(float));
        if (l > 0 && l < s->bottom) A((void**)&s->r_alt[l], n * sizeof(float));
    }
    A((void**)&s->div0, s->ncell * sizeof(float));
    if (s->enclosed) s->div0r = s->div0;
    else A((void**)&s->div0r, s->ncell * sizeof(float));
    // 2D: w between its two kernels (3D computes w in shared memory)
    if (s->dim == 2) A((void**)&s->vort, s->ncell * sizeof(float));
    A((void**)&s->fmask, s->ncell);   // level-0 fluid mask (k_rb.cu, k_mixed.cu, k_adjoint.cu)
    if (s->nx % 2 == 0 && s->levels > 1) {   // colour-split level 0 (k_rb.cu)
        A((void**)&s->rhs_s, s->ncell * sizeof(float));
        A((void**)&s->rhs_r, s->ncell * sizeof(float));
        A((void**)&s->rb_mask, s->ncell);
    }
    s->red.max_blocks = (int)(((s->nx + 32) / 32 + 1) * ((s->ny + 8) / 8 + 1) * (size_t)(s->nz + 1));
    A((void**)&s->red.partial, (size_t)s->red.max_blocks * sizeof(double));
    s->red.stage2 = s->red.max_blocks / 1024 + 2;
    A((void**)&s->red.partial2, (size_t)2 * s->red.stage2 * sizeof(double));
    A((void**)&s->red.out, SLOT_COUNT * sizeof(double));
    if (rc == SS_OK) s->d_err = reinterpret_cast<int*>(s->red.out + SLOT_ERR);
    A((void**)&s->red.ticket, sizeof(unsigned int));
    if (rc == SS_OK) {
        cudaError_t e = cudaMallocHost((void**)&s->red.host, SLOT_COUNT * sizeof(double));
        if (e != cudaSuccess) rc = check_cuda(e, "cudaMallocHost");
    }
    if (rc != SS_OK) {
        free_sim(s);
        return rc;
    }
    // initial state: velocities and pressure 0, smoke (0, 0, 0, t_ambient)
    for (int dd = 0; dd < s->dim; ++dd)
        for (int b = 0; b < 2; ++b) rc = rc ? rc : check_cuda(cudaMemsetAsync(s->vel[dd][b], 0, s->nv[dd] * 4, st), "memset");
    for (int b = 0; b < 2; ++b) {
        if (!rc) rc = check_cuda(cudaMemsetAsync(s->dens[b], 0, s->ncell * s->nch * 4, st), "memset");
        if (!rc) rc = launch_fill(s->temp[b], s->ncell, s->t_amb0, st);
    }
    for (int l = 0; l < lv && !rc; ++l) {
        const size_t n = (size_t)s->lv[l].n[0] * s->lv[l].n[1] * s->lv[l].n[2];
        rc = check_cuda(cudaMemsetAsync(s->p[l], 0, n * 4, st), "memset");
        if (!rc) rc = check_cuda(cudaMemsetAsync(s->r[l], 0, n * 4, st), "memset");
    }
    if (!rc) rc = check_cuda(cudaMemsetAsync(s->red.out, 0, SLOT_COUNT * sizeof(double), st), "memset");
    if (!rc) rc = check_cuda(cudaMemsetAsync(s->red.ticket, 0, sizeof(unsigned int), st), "memset");
    if (!rc) rc = check_cuda(cudaMemsetAsync(s->div0, 0, s->ncell * 4, st), "memset");
    if (!rc && s->div0r != s->div0) rc = check_cuda(cudaMemsetAsync(s->div0r, 0, s->ncell * 4, st), "memset");
    if (!rc && s->rb_mask) rc = rb_init_vector_paths(s, st);
    if (!rc) rc = ss_set_scene(s, nullptr, 0, nullptr, 0, nullptr, 0, stream);
    if (!rc) rc = check_cuda(cudaStreamSynchronize(st), "create sync");
    if (rc) {
        free_sim(s);
        return rc;
    }
    *out = s;
    return SS_OK;
}

int ss_destroy(ss_sim* s) {
    if (!s) return set_error(SS_E_INVALID, "NULL handle");
    cudaDeviceSynchronize();
    free_sim(s);
    return SS_OK;
}

int ss_get_desc(const ss_sim* s, ss_desc* out, int* levels, int level_sizes[][3]) {
    if (!s) return set_error(SS_E_INVALID, "NULL handle");
    if (out) {
        out->dim = s->dim;
        out->n[0] = s->nx; out->n[1] = s->ny; out->n[2] = s->nz;
        out->cell_size = s->h;
        out->density_channels = s->nch;
        out->enclosed = s->enclosed;
        out->min_coarse = s->min_coarse;
        out->t_ambient = s->t_amb0;
    }
    if (levels) *levels = s->levels;
    if (level_sizes)
        for (int l = 0; l < s->levels; ++l)
            for (int d = 0; d < 3; ++d) level_sizes[l][d] = s->lv[l].n[d];
    return SS_OK;
}

// ------------------------------------------------------------------- scene
static int upload_array(void** dptr, int* cap, const void* host, size_t elem, int n, cudaStream_t st) {
    if (n > *cap) {
        cudaFree(*dptr);
        *dptr = nullptr;
        TRY(dalloc(dptr, elem * (size_t)n));
        *cap = n;
    }
    if (n > 0) CU(cudaMemcpyAsync(*dptr, host, elem * (size_t)n, cudaMemcpyHostToDevice, st), "scene upload");
    return SS_OK;
}

static bool scene_moving(const ss_sim* s) {
    for (const ss_obstacle& o : s->ob)
        if (o.anchored != 1.f) return true;
    return false;
}

static int rasterize_solid(ss_sim* s, cudaStream_t st) {
    // solid velocity channels only when some obstacle or box can carry one
    bool need = false;
    for (const ss_obstacle& o : s->ob)
        if ((o.velocity[0] != 0.f || o.velocity[1] != 0.f || o.velocity[2] != 0.f) && o.anchored != 1.f) need = true;
    for (const ss_box& b : s->bx)
        if ((b.velocity[0] != 0.f || b.velocity[1] != 0.f || b.velocity[2] != 0.f) && b.anchored != 1.f) need = true;
    if (scene_moving(s)) need = true;
    if (need && !s->svel[0]) {
        for (int d = 0; d < s->dim; ++d) TRY(dalloc((void**)&s->svel[d], s->ncell * sizeof(float)));
    }
    s->svel_active = need ? 1 : 0;
    TRY(upload_array((void**)&s->d_ob, &s->cap_ob, s->ob.data(), sizeof(ss_obstacle), (int)s->ob.size(), st));
    TRY(upload_array((void**)&s->d_bx, &s->cap_bx, s->bx.data(), sizeof(ss_box), (int)s->bx.size(), st));
    TRY(launch_rasterize(s, st));
    TRY(launch_flags(s, st));
    if (s->rb_mask) TRY(launch_rb_split_mask(s, st));
    TRY(launch_solid_pyramid(s, st));
    return SS_OK;
}

int ss_set_scene(ss_sim* s, const ss_emitter* em, int ne, const ss_obstacle* ob, int no, const ss_box* bx, int nb,
                 void* stream) {
    if (!s) return set_error(SS_E_INVALID, "NULL handle");
    if (ne < 0 || no < 0 || nb < 0 || ne > SS_MAX_EMITTERS || no > SS_MAX_OBSTACLES || nb > SS_MAX_BOXES)
        return set_error(SS_E_INVALID, "scene object count out of range");
    if ((ne && !em) || (no && !ob) || (nb && !bx)) return set_error(SS_E_INVALID, "NULL scene array");
    for (int i = 0; i < ne; ++i) {
        const ss_emitter& e = em[i];
        const float v[] = {e.pos[0], e.pos[1], e.pos[2], e.radius, e.density[0], e.density[1], e.density[2],
                           e.temperature, e.velocity[0], e.velocity[1], e.velocity[2]};
        for (float x : v)
            if (!isfinite(x)) return set_error(SS_E_NONFINITE, "non-finite emitter field");
    }
    for (int i = 0; i < no; ++i) {
        const ss_obstacle& o = ob[i];
        const float v[] = {o.pos[0], o.pos[1], o.pos[2], o.radius, o.velocity[0], o.velocity[1], o.velocity[2], o.anchored};
        for (float x : v)
            if (!isfinite(x)) return set_error(SS_E_NONFINITE, "non-finite obstacle field");
    }
    for (int i = 0; i < nb; ++i) {
        const ss_box& b = bx[i];
        const float v[] = {b.lo[0], b.lo[1], b.lo[2], b.hi[0], b.hi[1], b.hi[2], b.velocity[0], b.velocity[1], b.velocity[2], b.anchored};
        for (float x : v)
            if (!isfinite(x)) return set_error(SS_E_NONFINITE, "non-finite box field");
    }
    cudaStream_t st = as_stream(stream);
    s->em.assign(em, em + ne);
    s->ob.assign(ob, ob + no);
    s->bx.assign(bx, bx + nb);
    TRY(upload_array((void**)&s->d_em, &s->cap_em, s->em.data(), sizeof(ss_emitter), ne, st));
    TRY(rasterize_solid(s, st));
    CU(cudaStreamSynchronize(st), "set_scene sync");
    return SS_OK;
}

int ss_get_scene(ss_sim* s, ss_emitter* em, int ne, ss_obstacle* ob, int no) {
    if (!s) return set_error(SS_E_INVALID, "NULL handle");
    if (em) std::copy_n(s->em.begin(), std::min<size_t>((size_t)std::max(ne, 0), s->em.size()), em);
    if (ob) std::copy_n(s->ob.begin(), std::min<size_t>((size_t)std::max(no, 0), s->ob.size()), ob);
    return SS_OK;
}

// reference update_emitters_status (shaders3d/compute/update_emitters_status.comp:49-59)
static void emitters_status(ss_sim* s, float current_time) {
    for (ss_emitter& e : s->em) {
        if (e.emit == 1 && e.delay != 0) {
            e.emit = 0;
            e.last_emit = (int)current_time;
            continue;
        }
        if (current_time - (float)e.last_emit >= (float)e.delay) e.emit = 1;
    }
}

// reference obstacle_update (shaders3d/compute/obstacle_update.comp:51-135):
// gravity, wall bounce 0.999, push-out against the input positions, damping.
static void obstacles_update(ss_sim* s, float dt) {
    const int n = (int)s->ob.size();
    if (n == 0) return;
    const std::vector<ss_obstacle> in = s->ob;
    const bool d3 = s->dim == 3;
    const int nd = d3 ? 3 : 2;
    const float maxb[3] = {(float)s->nx, (float)s->ny, (float)s->nz};
    for (int i = 0; i < n; ++i) {
        float pos[3] = {in[i].pos[0], in[i].pos[1], d3 ? in[i].pos[2] : 0.f};
        float vel[3] = {in[i].velocity[0], in[i].velocity[1], d3 ? in[i].velocity[2] : 0.f};
        const float r = in[i].radius, anchored = in[i].anchored, movable = 1.f - anchored;
        if (!(anchored == 1.f)) {
            vel[1] = vel[1] + -9.81f * dt * movable;
            vel[0] = vel[0] + 0.f * dt * movable;
            if (d3) vel[2] = vel[2] + 0.f * dt * movable;
            for (int c = 0; c < nd; ++c) pos[c] = pos[c] + vel[c] * dt * movable;
            const float B = 0.999f;
            for (int c = 0; c < nd; ++c) {
                if (pos[c] - r < 0.f) { pos[c] = 0.f + r; vel[c] *= -B; }
                if (pos[c] + r > maxb[c]) { pos[c] = maxb[c] - r; vel[c] *= -B; }
            }
            for (int j = 0; j < n; ++j) {
                if (j == i) continue;
                const float dd[3] = {pos[0] - in[j].pos[0], pos[1] - in[j].pos[1], d3 ? pos[2] - in[j].pos[2] : 0.f};
                const float dist = d3 ? sqrtf(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]) : sqrtf(dd[0] * dd[0] + dd[1] * dd[1]);
                const float min_dist = r + in[j].radius;
                if (dist < min_dist && dist > 0.0001f) {
                    const float nn[3] = {dd[0] / dist, dd[1] / dist, dd[2] / dist};
                    for (int c = 0; c < nd; ++c) pos[c] += nn[c] * (min_dist - dist) * 0.5f * movable;
                    const float rv[3] = {vel[0] - in[j].velocity[0], vel[1] - in[j].velocity[1],
                                         d3 ? vel[2] - in[j].velocity[2] : 0.f};
                    const float vn = d3 ? rv[0] * nn[0] + rv[1] * nn[1] + rv[2] * nn[2] : rv[0] * nn[0] + rv[1] * nn[1];
                    if (vn < 0.f)
                        for (int c = 0; c < nd; ++c) vel[c] -= vn * nn[c] * movable;
                }
            }
        }
        s->ob[i].pos[0] = pos[0]; s->ob[i].pos[1] = pos[1];
        if (d3) s->ob[i].pos[2] = pos[2];
        s->ob[i].velocity[0] = vel[0] * 0.999f;
        s->ob[i].velocity[1] = vel[1] * 0.999f;
        if (d3) s->ob[i].velocity[2] = vel[2] * 0.999f;
    }
}

// ------------------------------------------------------------------- fields
static int field_buffer(ss_sim* s, int f, float** ptr, size_t* count) {
    switch (f) {
    case SS_FIELD_VX: *ptr = s->vel[0][s->vi[0]]; *count = s->nv[0]; return SS_OK;
    case SS_FIELD_VY: *ptr = s->vel[1][s->vi[1]]; *count = s->nv[1]; return SS_OK;
    case SS_FIELD_VZ:
        if (s->dim != 3) return set_error(SS_E_INVALID, "2D grid has no w");
        *ptr = s->vel[2][s->vi[2]]; *count = s->nv[2]; return SS_OK;
    case SS_FIELD_DENSITY: *ptr = s->dens[s->si]; *count = s->ncell * s->nch; return SS_OK;
    case SS_FIELD_TEMPERATURE: *ptr = s->temp[s->si]; *count = s->ncell; return SS_OK;
    case SS_FIELD_PRESSURE: *ptr = s->p[0]; *count = s->ncell; return SS_OK;
    case SS_FIELD_DIVERGENCE: *ptr = s->div0; *count = s->ncell; return SS_OK;
    default: return set_error(SS_E_INVALID, "unknown field");
    }
}

int ss_set_field(ss_sim* s, int f, const float* host, size_t count, void* stream) {
    if (!s || !host) return set_error(SS_E_INVALID, "NULL argument");
    if (f == SS_FIELD_SOLID || f == SS_FIELD_DIVERGENCE) return set_error(SS_E_INVALID, "field is read only (use ss_set_scene)");
    float* d;
    size_t n;
    TRY(field_buffer(s, f, &d, &n));
    if (count != n) return set_error(SS_E_INVALID, "element count does not match the field");
    for (size_t i = 0; i < n; ++i)
        if (!isfinite(host[i])) return set_error(SS_E_NONFINITE, "non-finite value in field data");
    cudaStream_t st = as_stream(stream);
    if (f == SS_FIELD_PRESSURE) s->p64_valid = 0;
    CU(cudaMemcpyAsync(d, host, n * sizeof(float), cudaMemcpyHostToDevice, st), "set_field");
    CU(cudaStreamSynchronize(st), "set_field sync");
    return SS_OK;
}

int ss_set_field_device(ss_sim* s, int f, const float* dev, size_t count, void* stream) {
    if (!s || !dev) return set_error(SS_E_INVALID, "NULL argument");
    if (f == SS_FIELD_SOLID || f == SS_FIELD_DIVERGENCE) return set_error(SS_E_INVALID, "field is read only (use ss_set_scene)");
    float* d;
    size_t n;
    TRY(field_buffer(s, f, &d, &n));
    if (count != n) return set_error(SS_E_INVALID, "element count does not match the field");
    if (f == SS_FIELD_PRESSURE) s->p64_valid = 0;
    CU(cudaMemcpyAsync(d, dev, n * sizeof(float), cudaMemcpyDeviceToDevice, as_stream(stream)), "set_field_device");
    return SS_OK;
}

int ss_get_field_device(ss_sim* s, int f, float* dev, size_t count, void* stream) {
    if (!s || !dev) return set_error(SS_E_INVALID, "NULL argument");
    if (f == SS_FIELD_SOLID || f == SS_FIELD_DIVERGENCE) return set_error(SS_E_INVALID, "use ss_get_field for this field");
    float* d;
    size_t n;
    TRY(field_buffer(s, f, &d, &n));
    if (count != n) return set_error(SS_E_INVALID, "element count does not match the field");
    CU(cudaMemcpyAsync(dev, d, n * sizeof(float), cudaMemcpyDeviceToDevice, as_stream(stream)), "get_field_device");
    return SS_OK;
}

int ss_get_field(ss_sim* s, int f, float* host, size_t count, void* stream) {
    if (!s || !host) return set_error(SS_E_INVALID, "NULL argument");
    cudaStream_t st = as_stream(stream);
    if (f == SS_FIELD_SOLID) {
        if (count != s->ncell) return set_error(SS_E_INVALID, "element count does not match the field");
        std::vector<uint8_t> tmp(s->ncell);
        CU(cudaMemcpyAsync(tmp.data(), s->solid, s->ncell, cudaMemcpyDeviceToHost, st), "get_field");
        CU(cudaStreamSynchronize(st), "get_field sync");
        for (size_t i = 0; i < s->ncell; ++i) host[i] = tmp[i] ? 1.f : 0.f;
        return SS_OK;
    }
    if (f == SS_FIELD_DIVERGENCE) {
        CU(cudaMemsetAsync(s->div0, 0, s->ncell * sizeof(float), st), "memset");
        TRY(launch_divergence(s, true, -1, st));
    }
    float* d;
    size_t n;
    TRY(field_buffer(s, f, &d, &n));
    if (count != n) return set_error(SS_E_INVALID, "element count does not match the field");
    CU(cudaMemcpyAsync(host, d, n * sizeof(float), cudaMemcpyDeviceToHost, st), "get_field");
    CU(cudaStreamSynchronize(st), "get_field sync");
    return check_device_error(s, st);
}

int ss_field_device_ptr(ss_sim* s, int f, void** dptr, size_t* count) {
    if (!s || !dptr) return set_error(SS_E_INVALID, "NULL argument");
    if (f == SS_FIELD_SOLID) {
        *dptr = s->solid;
        if (count) *count = s->ncell;
        return SS_OK;
    }
    float* d;
    size_t n;
    TRY(field_buffer(s, f, &d, &n));
    *dptr = d;
    if (count) *count = n;
    return SS_OK;
}

int ss_clear_grid(ss_sim* s, float t_ambient, void* stream) {
    if (!s) return set_error(SS_E_INVALID, "NULL handle");
    if (!isfinite(t_ambient)) return set_error(SS_E_NONFINITE, "t_ambient");
    cudaStream_t st = as_stream(stream);
    // reference clear_grid3d (3d/grid3d.c:164-183)
    for (int d = 0; d < s->dim; ++d)
        for (int b = 0; b < 2; ++b) CU(cudaMemsetAsync(s->vel[d][b], 0, s->nv[d] * 4, st), "memset");
    for (int b = 0; b < 2; ++b) {
        CU(cudaMemsetAsync(s->dens[b], 0, s->ncell * s->nch * 4, st), "memset");
        TRY(launch_fill(s->temp[b], s->ncell, t_ambient, st));
    }
    for (int l = 0; l < s->levels; ++l) {
        const size_t n = (size_t)s->lv[l].n[0] * s->lv[l].n[1] * s->lv[l].n[2];
        CU(cudaMemsetAsync(s->p[l], 0, n * 4, st), "memset");
    }
    s->p64_valid = 0;
    CU(cudaStreamSynchronize(st), "clear sync");
    return SS_OK;
}

int ss_get_level(ss_sim* s, int L, int what, float* host, size_t count, void* stream) {
    if (!s || !host) return set_error(SS_E_INVALID, "NULL argument");
    if (L < 0 || L >= s->levels) return set_error(SS_E_INVALID, "level out of range");
    const size_t n = (size_t)s->lv[L].n[0] * s->lv[L].n[1] * s->lv[L].n[2];
    if (count != n) return set_error(SS_E_INVALID, "element count does not match the level");
    cudaStream_t st = as_stream(stream);
    if (what == SS_LEVEL_FLUID_WEIGHT) {
        std::vector<float> tmp(n);
        if (L == 0) {
            std::vector<uint8_t> sb(n);
            CU(cudaMemcpyAsync(sb.data(), s->solid, n, cudaMemcpyDeviceToHost, st), "get_level");
            CU(cudaStreamSynchronize(st), "sync");
            for (size_t i = 0; i < n; ++i) host[i] = sb[i] ? 0.f : 1.f;
        } else {
            CU(cudaMemcpyAsync(tmp.data(), s->alpha[L], n * 4, cudaMemcpyDeviceToHost, st), "get_level");
            CU(cudaStreamSynchronize(st), "sync");
            for (size_t i = 0; i < n; ++i) host[i] = 1.f - tmp[i];
        }
        return SS_OK;
    }
    float* d = what == SS_LEVEL_PRESSURE ? s->p[L] : what == SS_LEVEL_RESIDUAL ? s->r[L] : nullptr;
    if (!d) return set_error(SS_E_INVALID, "unknown level array");
    CU(cudaMemcpyAsync(host, d, n * 4, cudaMemcpyDeviceToHost, st), "get_level");
    CU(cudaStreamSynchronize(st), "sync");
    return SS_OK;
}

int ss_set_level(ss_sim* s, int L, int what, const float* host, size_t count, void* stream) {
    if (!s || !host) return set_error(SS_E_INVALID, "NULL argument");
    if (L < 0 || L >= s->levels) return set_error(SS_E_INVALID, "level out of range");
    const size_t n = (size_t)s->lv[L].n[0] * s->lv[L].n[1] * s->lv[L].n[2];
    if (count != n) return set_error(SS_E_INVALID, "element count does not match the level");
    float* d = what == SS_LEVEL_PRESSURE ? s->p[L] : what == SS_LEVEL_RESIDUAL ? s->r[L] : nullptr;
    if (!d) return set_error(SS_E_INVALID, "level array is read only");
    cudaStream_t st = as_stream(stream);
    if (L == 0 && what == SS_LEVEL_PRESSURE) s->p64_valid = 0;
    CU(cudaMemcpyAsync(d, host, n * 4, cudaMemcpyHostToDevice, st), "set_level");
    CU(cudaStreamSynchronize(st), "sync");
    return SS_OK;
}

// ------------------------------------------------------------------ solver
// v_cycle (common/physics/grid.c:177-209).  Levels from s->bottom down run in
// one single-block launch; above it every red-black sweep is one tiled launch,
// the last pre-smoothing sweep carrying the residual + restriction and the
// first post-smoothing sweep the prolongation.
static int v_cycle_rec(ss_sim* s, const StepConsts& c, const ss_mg_schedule& mg, int L, cudaStream_t st) {
    const int q = mg.ref_quirks;
    if (L == 0 && s->rb_active) {
        // level 0 on the colour-split arrays; residual + restriction fused
        TRY(launch_rb_sweep(s, mg.n_pre, st));
        TRY(launch_rb_residual_restrict(s, st));
        const size_t nc = (size_t)s->lv[1].n[0] * s->lv[1].n[1] * s->lv[1].n[2];
        CU(cudaMemsetAsync(s->p[1], 0, nc * sizeof(float), st), "clear coarse p");
        TRY(v_cycle_rec(s, c, mg, 1, st));
        TRY(launch_rb_prolong(s, st));
        return launch_rb_sweep(s, mg.n_post, st);
    }
    if (L >= 1 && L >= s->bottom && L < s->levels) return launch_bottom(s, mg, L, st);
    if (L == s->levels - 1) return launch_smooth(s, c, L, mg.n_coarse, q, st);
    for (int i = 0; i < mg.n_pre; ++i) TRY(launch_rbgs_sweep(s, c, L, q, false, i == mg.n_pre - 1, st));
    // residual written in place only where the reference's post-smoother reads it
    if (mg.n_pre == 0) TRY(launch_residual(s, c, L, q && L > 0, true, q, st));
    const size_t nc = (size_t)s->lv[L + 1].n[0] * s->lv[L + 1].n[1] * s->lv[L + 1].n[2];
    CU(cudaMemsetAsync(s->p[L + 1], 0, nc * sizeof(float), st), "clear coarse p");
    TRY(v_cycle_rec(s, c, mg, L + 1, st));
    if (mg.n_post == 0) return launch_prolong(s, L, st);
    for (int i = 0; i < mg.n_post; ++i) TRY(launch_rbgs_sweep(s, c, L, q, i == 0, false, st));
    return SS_OK;
}

// The device error word collects the bounded waits that gave up (bit 0: a
// coarse-level sweep's TMA tile load did not arrive in time, so that sweep
// skipped its cells).  Only those sweeps (the FP32 solve's coarse levels) set
// it; a solve that may run them arms s->err_armed.  It is read - with the
// statistics slots of a step, which hold it, and by ss_get_stats and
// ss_get_field while armed - reported once and cleared, so the next report
// concerns later launches only.
static int report_device_error(ss_sim* s, int err, cudaStream_t st) {
    s->err_armed = 0;
    if (err) {
        CU(cudaMemsetAsync(s->d_err, 0, sizeof(int), st), "error word clear");
        CU(cudaStreamSynchronize(st), "error word clear");
        if (err & 1)
            return set_error(SS_E_CUDA, "a coarse-level sweep gave up waiting for its TMA tile loads (bounded wait); "
                                        "the pressure of that solve is not valid");
        return set_error(SS_E_CUDA, "unknown bit set in the device error word");
    }
    return SS_OK;
}

static int check_device_error(ss_sim* s, cudaStream_t st) {
    int err = 0;
    CU(cudaMemcpyAsync(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "error word");
    CU(cudaStreamSynchronize(st), "error word sync");
    return report_device_error(s, err, st);
}

// the statistics slots and the error word, in one copy and one synchronisation
static int read_slots(ss_sim* s, cudaStream_t st) {
    CU(cudaMemcpyAsync(s->red.host, s->red.out, SLOT_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st), "slots");
    CU(cudaStreamSynchronize(st), "slots sync");
    int err = 0;
    memcpy(&err, &s->red.host[SLOT_ERR], sizeof(int));
    return report_device_error(s, err, st);
}

static int ensure_pyramid(ss_sim* s, cudaStream_t st) {
    if (s->pyramid_dirty) TRY(launch_solid_pyramid(s, st));
    return SS_OK;
}

}  // extern "C"

// ------------------------------------------------------- solve graphs
// The multigrid part of a solve is the same sequence of launches every step
// (same pointers, schedule and constants): it is recorded once as a CUDA
// graph and replayed, which removes the per-launch CPU and GPU gaps of its
// many small coarse-level kernels.  The key holds everything the recorded
// launches bake in besides the simulation's own (stable) buffers.  Runs the
// body directly on the legacy stream or when the caller is capturing.
struct GraphKey {
    int kind, parity, slot, rb, bottom;
    ss_mg_schedule mg;
    float dt, rho;
};

template <typename F>
static int run_graph(ss_sim* s, int which, const GraphKey& key, cudaStream_t st, F body) {
    if (!s->use_graphs || st == nullptr) return body();
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CU(cudaStreamIsCapturing(st, &cs), "cudaStreamIsCapturing");
    if (cs != cudaStreamCaptureStatusNone) return body();
    static_assert(sizeof(GraphKey) <= sizeof(s->graphs[0].key), "graph key size");
    unsigned char kb[sizeof(s->graphs[0].key)] = {};
    memcpy(kb, &key, sizeof(GraphKey));
    ss_sim::SolveGraph& g = s->graphs[which];
    if (g.exec && memcmp(g.key, kb, sizeof kb) == 0) {
        CU(cudaGraphLaunch(g.exec, st), "cudaGraphLaunch");
        s->nlaunch += g.launches;
        return SS_OK;
    }
    if (g.exec) {
        cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    const long long before = s->nlaunch;
    CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
    const int rc = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc != SS_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    CU(e, "cudaStreamEndCapture");
    const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        g.exec = nullptr;
        return check_cuda(ei, "cudaGraphInstantiate");
    }
    memcpy(g.key, kb, sizeof kb);
    g.launches = s->nlaunch - before;
    CU(cudaGraphLaunch(g.exec, st), "cudaGraphLaunch");
    return SS_OK;
}

static GraphKey graph_key(const ss_sim* s, int kind, int parity, int slot, int rb, const ss_params* p) {
    GraphKey k;
    memset(&k, 0, sizeof k);
    k.kind = kind; k.parity = parity; k.slot = slot; k.rb = rb; k.bottom = s->bottom;
    k.mg = p->mg;
    k.dt = p->time_step; k.rho = p->density;
    return k;
}

extern "C" {

// ------------------------------------------------------- mixed precision
// Buffers of the mixed-precision solve, made on its first use: the FP64
// level-0 pressure and 2-byte coarse levels.
static int ensure_mixed(ss_sim* s, int prec, cudaStream_t st) {
    if (!rb_supported(s, 0))
        return set_error(SS_E_UNSUPPORTED, "the mixed-precision solve needs an even nx and at least two levels");
    if (!s->p64) {
        CU(cudaMalloc((void**)&s->p64, s->ncell * sizeof(double)), "cudaMalloc(p64)");
        CU(cudaMalloc((void**)&s->p64b, s->ncell * sizeof(double)), "cudaMalloc(p64)");
        s->p64_valid = 0;
    }
    if (!s->red.partial_max)
        CU(cudaMalloc((void**)&s->red.partial_max, (size_t)s->red.max_blocks * sizeof(double)), "cudaMalloc");

    if (!s->d_scale) {
        CU(cudaMalloc((void**)&s->d_scale, 2 * sizeof(float)), "cudaMalloc");
        const float one[2] = {1.f, 1.f};
        CU(cudaMemcpyAsync(s->d_scale, one, sizeof(one), cudaMemcpyHostToDevice, st), "scale init");
        CU(cudaStreamSynchronize(st), "scale init");
    }
    for (int l = 1; l < s->levels; ++l) {
        const size_t n = (size_t)s->lv[l].n[0] * s->lv[l].n[1] * s->lv[l].n[2];
        if (!s->cp[l]) {
            CU(cudaMalloc(&s->cp[l], n * 2), "cudaMalloc(coarse p)");
            CU(cudaMemsetAsync(s->cp[l], 0, n * 2, st), "memset");
        }
        if (!s->cr[l]) {
            CU(cudaMalloc(&s->cr[l], n * 2), "cudaMalloc(coarse r)");
            CU(cudaMemsetAsync(s->cr[l], 0, n * 2, st), "memset");
        }
    }
    if (s->coarse_matrix && !s->cmat && s->bottom <= s->levels - 1) {
        const ss::Level& lc = s->lv[s->levels - 1];
        const long long nc = (long long)lc.n[0] * lc.n[1] * lc.n[2];
        if (nc <= kCoarseResponseMax) {
            CU(cudaMalloc((void**)&s->cmat, (size_t)(nc * nc) * sizeof(float)), "cudaMalloc(coarse matrix)");
            CU(cudaMalloc((void**)&s->cmat_alpha, (size_t)nc * sizeof(float)), "cudaMalloc(coarse matrix)");
            CU(cudaMalloc((void**)&s->cmat_state, 2 * sizeof(int)), "cudaMalloc(coarse matrix)");
            CU(cudaMalloc((void**)&s->cmat_part, kProductLanes * sizeof(float)), "cudaMalloc(coarse matrix)");
            CU(cudaMemsetAsync(s->cmat_state, 0xff, 2 * sizeof(int), st), "memset");
            s->cmat_n = (int)nc;
            s->cmat_dirty = 1;
            s->cmat_iters = -1;
        }
    }
    TRY(coarse_cluster_setup(s));
    s->cstore = prec;
    return SS_OK;
}

// One V-cycle on the correction e (colour-split FP32 level 0 in p_alt[0],
// coarse levels FP16/BF16), corrected operators (ref_quirks = 0).
static int v_cycle_mixed(ss_sim* s, const StepConsts& c, const ss_mg_schedule& mg, int L, int prec, cudaStream_t st) {
    if (L == 0) {
        // e starts at 0 and the prolongation zeroes non-fluid cells: the
        // half-sweeps may take the select-free form where that prolongation runs
        const bool z = rb_zero_form(s);
        TRY(launch_rb_sweep(s, mg.n_pre, st, z, true));   // e starts at 0
        TRY(launch_rb_residual_restrict_mixed(s, prec, st));   // also clears level 1's p
        TRY(v_cycle_mixed(s, c, mg, 1, prec, st));
        TRY(launch_rb_prolong_mixed(s, prec, st));
        return launch_rb_sweep(s, mg.n_post, st, z);
    }
    if (L == s->cluster_from && s->cluster_ctas > 0) return coarse_cluster(s, mg, L, prec, st);
    if (L >= s->bottom) return coarse_bottom(s, mg, L, prec, st);
    if (L == s->levels - 1) return coarse_smooth(s, c, L, mg.n_coarse, prec, st);
    TRY(coarse_smooth(s, c, L, mg.n_pre, prec, st));
    TRY(coarse_residual_restrict(s, c, L, prec, st));   // also clears level L+1's p
    TRY(v_cycle_mixed(s, c, mg, L + 1, prec, st));
    TRY(coarse_prolong(s, L, prec, st));
    return coarse_smooth(s, c, L, mg.n_post, prec, st);
}

// Warm start of the mixed solve.  p64 holds the previous step's pressure
// p(n-1).  With warm_start 1 and p64c holding p(n-2) - the solved pressure the
// previous mixed solve started from - the solve starts from the linear
// extrapolation 2 p(n-1) - p(n-2) and p64c takes p(n-1): the pre-solve
// divergence pass does that in place (extrapolates(), k_divergence's ep/eq).
// Otherwise p64c just takes p(n-1) (warm_start_p64), so that the next solve
// can extrapolate.  A fresh p64 (made from the FP32 pressure, not solved by
// this path) starts no history.
static bool extrapolates(const ss_sim* s, int mode, bool fresh) {
    return mode == 1 && !fresh && s->prev_ok && s->p64c;
}

static int warm_start_p64(ss_sim* s, int mode, bool fresh, cudaStream_t st) {
    if (mode != 1 || fresh) {
        s->prev_ok = 0;
        return SS_OK;
    }
    if (!s->p64c) CU(cudaMalloc((void**)&s->p64c, s->ncell * sizeof(double)), "cudaMalloc(p64c)");
    CU(cudaMemcpyAsync(s->p64c, s->p64, s->ncell * sizeof(double), cudaMemcpyDeviceToDevice, st), "warm start copy");
    s->prev_ok = 1;
    return SS_OK;
}

// ------------------------------------------------ device-side tolerance loop
// The mixed solve's tolerance loop as one graph: the first residual, then
// refinement step 1 as the body of a conditional (IF) graph node, step 2 as an
// IF node inside step 1's body, and so on, depth steps deep.  The last block
// of each residual launch applies the host loop's test (k_ir_residual,
// IrDecide) and sets the condition of the next step, so the steps run back to
// back with no host round trip between them.  A condition nobody set stays 0
// (the default, restored at every launch of the graph) and ends the chain:
// nothing in it can loop.  The steps alternate the FP64 buffers, so the chain
// is recorded once per starting parity (graphs 4 and 5).
constexpr int kChainDepth = 8;

static int build_solve_chain(ss_sim* s, const StepConsts& c, const ss_mg_schedule& mg, int depth,
                             ss_sim::SolveGraph& g) {
    if (!s->chain_stream)
        CU(cudaStreamCreateWithFlags(&s->chain_stream, cudaStreamNonBlocking), "cudaStreamCreate(chain)");
    cudaStream_t cs = s->chain_stream;
    double* const pa = s->p64;
    double* const pb = s->p64b;
    const int pdl = s->pdl;
    s->pdl = 0;   // plain stream order inside the conditional bodies
    cudaGraph_t top = nullptr;
    int rc = check_cuda(cudaGraphCreate(&top, 0), "cudaGraphCreate(solve chain)");
    cudaGraph_t cur = top;   // the graph that receives step k
    for (int k = 0; k <= depth && rc == SS_OK; ++k) {
        IrDecide d;
        d.tol = mg.tol;
        d.k = k;
        d.more = k < depth ? 1 : 0;
        d.active = 1;
        if (d.more)
            rc = check_cuda(cudaGraphConditionalHandleCreate(&d.next, cur, 0, cudaGraphCondAssignDefault),
                            "cudaGraphConditionalHandleCreate");
        if (rc == SS_OK)
            rc = check_cuda(cudaStreamBeginCaptureToGraph(cs, cur, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
                            "cudaStreamBeginCaptureToGraph");
        if (rc != SS_OK) break;
        const long long before = s->nlaunch;
        if (k > 0) rc = v_cycle_mixed(s, c, mg, 0, mg.precision, cs);
        if (rc == SS_OK) rc = launch_ir_residual(s, c, SLOT_RESIDUAL, k > 0, cs, &d);
        (k == 0 ? g.launches : g.step_launches) = s->nlaunch - before;
        cudaGraph_t next = nullptr;
        if (rc == SS_OK && d.more) {
            cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            rc = check_cuda(cudaStreamGetCaptureInfo(cs, &cst, nullptr, nullptr, &deps, &nd), "cudaStreamGetCaptureInfo");
            if (rc == SS_OK) {
                cudaGraphNodeParams np{};
                np.type = cudaGraphNodeTypeConditional;
                np.conditional.handle = d.next;
                np.conditional.type = cudaGraphCondTypeIf;
                np.conditional.size = 1;
                cudaGraphNode_t node = nullptr;
                rc = check_cuda(cudaGraphAddNode(&node, cur, deps, nd, &np), "cudaGraphAddNode(conditional)");
                if (rc == SS_OK) next = np.conditional.phGraph_out[0];
            }
        }
        cudaGraph_t captured = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(cs, &captured);
        if (rc == SS_OK) rc = check_cuda(ee, "cudaStreamEndCapture(solve chain)");
        if (k > 0) std::swap(s->p64, s->p64b);
        cur = next;
    }
    s->p64 = pa;
    s->p64b = pb;
    s->pdl = pdl;
    if (rc == SS_OK) {
        const cudaError_t ei = cudaGraphInstantiate(&g.exec, top, 0);
        if (ei != cudaSuccess) g.exec = nullptr;
        rc = check_cuda(ei, "cudaGraphInstantiate(solve chain)");
    }
    if (top) cudaGraphDestroy(top);
    if (rc != SS_OK) {
        cudaGetLastError();
        return set_error(rc, g_err +
                                 " (recording the device-side tolerance loop; SMOKESIM_DEVICE_LOOP=0 runs it on the host)");
    }
    return SS_OK;
}

// The device-side loop needs a stream that graphs can be launched on and that
// is not being recorded by the caller.
static bool chain_ok(ss_sim* s, cudaStream_t st) {
    if (!s->device_loop || !s->use_graphs || st == nullptr) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return false;
    return cs == cudaStreamCaptureStatusNone;
}

// Runs up to depth refinement steps of the tolerance loop on the device and
// reads the statistics slots once; *k = the steps it took.  The FP64 buffers
// end swapped after an odd number of steps.
static int run_solve_chain(ss_sim* s, const ss_params* p, const StepConsts& c, int depth, cudaStream_t st,
                           int* k_out) {
    const GraphKey key = graph_key(s, 4, s->p64_parity, SLOT_RESIDUAL, depth, p);
    unsigned char kb[sizeof(s->graphs[0].key)] = {};
    memcpy(kb, &key, sizeof(GraphKey));
    ss_sim::SolveGraph& g = s->graphs[4 + s->p64_parity];
    if (!g.exec || memcmp(g.key, kb, sizeof kb) != 0) {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
        const long long n0 = s->nlaunch;
        const int rc = build_solve_chain(s, c, p->mg, depth, g);
        s->nlaunch = n0;
        if (rc != SS_OK) return rc;
        memcpy(g.key, kb, sizeof kb);
    }
    CU(cudaGraphLaunch(g.exec, st), "cudaGraphLaunch(solve chain)");
    TRY(read_slots(s, st));
    const double kd = s->red.host[SLOT_STEPS];
    if (!(kd >= 0.0 && kd <= (double)depth))
        return set_error(SS_E_CUDA, "the device-side tolerance loop reported an impossible step count");
    const int k = (int)kd;
    s->nlaunch += g.launches + (long long)k * g.step_launches;
    if (k & 1) {
        std::swap(s->p64, s->p64b);
        s->p64_parity ^= 1;
    }
    *k_out = k;
    return SS_OK;
}

// Mixed-precision projection: iterative refinement of the FP64 pressure with
// FP32 V-cycles on the FP64 residual (k_mixed.cu).  Each refinement step
// counts as one V-cycle in the statistics.
// defer_p0: the caller's FP64 velocity update writes the FP32 pressure copy
static int pressure_solve_mixed(ss_sim* s, const ss_params* p, const StepConsts& c, cudaStream_t st,
                                bool defer_p0 = false) {
    const ss_mg_schedule& mg = p->mg;
    if (mg.ref_quirks) return set_error(SS_E_INVALID, "the mixed-precision solve runs the corrected operators (ref_quirks = 0)");
    TRY(ensure_mixed(s, mg.precision, st));
    TRY(ensure_pyramid(s, st));
    TRY(update_coarse_matrix(s, mg, st));
    const bool tol_mode = mg.tol > 0.0;
    const bool stats = p->collect_stats || tol_mode;
    const bool fresh = !s->p64_valid;
    const bool extrap = extrapolates(s, mg.warm_start, fresh);
    TRY(launch_divergence(s, true, stats ? SLOT_DIV_BEFORE : -1, st, nullptr, -1, extrap ? s->p64 : nullptr,
                          extrap ? s->p64c : nullptr));
    if (fresh) TRY(launch_p64_from_p0(s, st));
    if (!extrap) TRY(warm_start_p64(s, mg.warm_start, fresh, st));
    const int cap = mg.n_vcycles > 0 ? mg.n_vcycles : 1;
    int done = 0;
    double db = 0.0, res = 0.0;
    bool conv = true;
    bool pending = false;   // the last V-cycle's correction is not in p64 yet
    bool finished = false;
    if (tol_mode && chain_ok(s, st)) {
        // the first steps (all of them, as a rule) on the device; where the
        // chain ends unconverged below the cap, the host loop carries on
        TRY(run_solve_chain(s, p, c, std::min(cap, kChainDepth), st, &done));
        db = sqrt(s->red.host[SLOT_DIV_BEFORE]);
        res = sqrt(s->red.host[SLOT_RESIDUAL]);
        if (res <= mg.tol * db) {
            finished = true;
        } else if (done == cap) {
            conv = false;
            finished = true;
        } else {
            pending = true;
            ++done;
        }
    }
    while (!finished) {
        const bool last = !tol_mode && done == cap;
        if (last && !stats) break;
        if (pending) {
            // the last V-cycle + adding its correction and evaluating the
            // residual in one pass, recorded as one graph per buffer parity
            const int slot = stats ? SLOT_RESIDUAL : -1;
            TRY(run_graph(s, 2 + s->p64_parity, graph_key(s, 2, s->p64_parity, slot, 1, p), st, [&]() -> int {
                TRY(v_cycle_mixed(s, c, mg, 0, mg.precision, st));
                return launch_ir_residual(s, c, slot, true, st);
            }));
            std::swap(s->p64, s->p64b);
            s->p64_parity ^= 1;
        } else {
            TRY(launch_ir_residual(s, c, stats ? SLOT_RESIDUAL : -1, false, st));
        }
        pending = false;
        if (tol_mode || last) {
            TRY(read_slots(s, st));
            db = sqrt(s->red.host[SLOT_DIV_BEFORE]);
            res = sqrt(s->red.host[SLOT_RESIDUAL]);
            if (last) break;
            if (res <= mg.tol * db) break;
            if (done == cap) { conv = false; break; }
        }
        pending = true;   // the V-cycle runs at the top of the next pass
        ++done;
        if (!tol_mode && done == cap && !stats) {
            TRY(v_cycle_mixed(s, c, mg, 0, mg.precision, st));
            TRY(launch_ir_accumulate(s, st));
            pending = false;
            break;
        }
    }
    if (!defer_p0) TRY(launch_p0_from_p64(s, st));
    if (stats) {
        s->st.div_before = db;
        s->st.residual = res;
    }
    s->st.vcycles = done;
    s->st.converged = conv ? 1 : 0;
    return SS_OK;
}

// multigrid_pressure_solve (common/physics/grid.c:173-175)
static int pressure_solve(ss_sim* s, const ss_params* p, const StepConsts& c, cudaStream_t st,
                          bool defer_p0 = false) {
    const ss_mg_schedule& mg = p->mg;
    if (mg.precision != SS_PREC_FP32) return pressure_solve_mixed(s, p, c, st, defer_p0);
    s->p64_valid = 0;
    s->err_armed = 1;   // its coarse-level sweeps may take the bounded-wait TMA form
    const bool tol_mode = mg.tol > 0.0;
    const bool stats = p->collect_stats || tol_mode;
    TRY(ensure_pyramid(s, st));
    TRY(launch_divergence(s, true, stats ? SLOT_DIV_BEFORE : -1, st, &c, mg.ref_quirks));
    const int cap = mg.n_vcycles > 0 ? mg.n_vcycles : 1;
    int done = 0;
    bool conv = true;
    const bool rb = rb_supported(s, mg.ref_quirks);
    auto cycle = [&]() -> int {
        if (rb) TRY(launch_rb_convert(s, true, st));
        s->rb_active = rb ? 1 : 0;
        int rc = v_cycle_rec(s, c, mg, 0, st);
        s->rb_active = 0;
        if (rc) return rc;
        if (rb) TRY(launch_rb_convert(s, false, st));
        return SS_OK;
    };
    if (!tol_mode) {
        TRY(run_graph(s, 0, graph_key(s, 0, 0, stats ? SLOT_RESIDUAL : -1, rb, p), st, [&]() -> int {
            if (rb) TRY(launch_rb_convert(s, true, st));
            s->rb_active = rb ? 1 : 0;
            for (int i = 0; i < cap; ++i) {
                int rc = v_cycle_rec(s, c, mg, 0, st);
                if (rc) { s->rb_active = 0; return rc; }
            }
            s->rb_active = 0;
            if (rb) TRY(launch_rb_convert(s, false, st));
            if (stats) TRY(launch_projected_residual_norm(s, c, SLOT_RESIDUAL, st));
            return SS_OK;
        }));
        done = cap;
        if (stats) {
            TRY(read_slots(s, st));
            s->st.div_before = sqrt(s->red.host[SLOT_DIV_BEFORE]);
            s->st.residual = sqrt(s->red.host[SLOT_RESIDUAL]);
        }
    } else {
        TRY(launch_projected_residual_norm(s, c, SLOT_RESIDUAL, st));
        TRY(read_slots(s, st));
        const double db = sqrt(s->red.host[SLOT_DIV_BEFORE]);
        double res = sqrt(s->red.host[SLOT_RESIDUAL]);
        while (done < cap && !(res <= mg.tol * db)) {
            TRY(run_graph(s, 1, graph_key(s, 1, 0, SLOT_RESIDUAL, rb, p), st, [&]() -> int {
                TRY(cycle());
                return launch_projected_residual_norm(s, c, SLOT_RESIDUAL, st);
            }));
            ++done;
            TRY(read_slots(s, st));
            res = sqrt(s->red.host[SLOT_RESIDUAL]);
        }
        conv = res <= mg.tol * db;
        s->st.div_before = db;
        s->st.residual = res;
    }
    s->st.vcycles = done;
    s->st.converged = conv ? 1 : 0;
    return SS_OK;
}

static int save_vel(ss_sim* s, float* const dst[3], cudaStream_t st) {
    for (int d = 0; d < s->dim; ++d)
        if (dst[d]) CU(cudaMemcpyAsync(dst[d], s->vel[d][s->vi[d]], s->nv[d] * sizeof(float), cudaMemcpyDeviceToDevice, st),
                       "save velocity");
    return SS_OK;
}

static int do_step(ss_sim* s, const ss_params* p, cudaStream_t st, StepSaves* sv = nullptr) {
    const StepConsts c = make_consts(s, p);
    const int m = p->stage_mask;
    if (m & SS_STAGE_HANDLE_EMITTERS) {
        emitters_status(s, p->current_time);
        TRY(upload_array((void**)&s->d_em, &s->cap_em, s->em.data(), sizeof(ss_emitter), (int)s->em.size(), st));
        TRY(launch_emitters(s, c, st));
        TRY(launch_force_field(s, c, st));
    }
    if (sv) {
        TRY(save_vel(s, sv->emit_vel, st));
        if (sv->emit_dens)
            CU(cudaMemcpyAsync(sv->emit_dens, s->dens[s->si], s->ncell * s->nch * sizeof(float), cudaMemcpyDeviceToDevice, st), "save");
        if (sv->emit_temp)
            CU(cudaMemcpyAsync(sv->emit_temp, s->temp[s->si], s->ncell * sizeof(float), cudaMemcpyDeviceToDevice, st), "save");
    }
    if (m & SS_STAGE_ADVECT_VELOCITIES) {
        TRY(launch_advect_velocities(s, c, (m & SS_STAGE_APPLY_BUOYANCY) != 0, st));
    } else if (m & SS_STAGE_APPLY_BUOYANCY) {
        TRY(launch_buoyancy(s, c, st));
    }
    if (sv) TRY(save_vel(s, sv->force_vel, st));
    if (m & SS_STAGE_APPLY_VORTICITY) TRY(launch_vorticity(s, c, st));
    // a mixed solve followed by the update leaves the FP32 pressure copy to
    // the update kernel, which reads the FP64 pressure anyway
    const bool defer_p0 = (m & SS_STAGE_RESOLVE_PRESSURE) && (m & SS_STAGE_UPDATE_VELOCITIES) &&
                          p->mg.precision != SS_PREC_FP32;
    if (m & SS_STAGE_RESOLVE_PRESSURE) {
        const bool f64 = p->mg.precision != SS_PREC_FP32;
        if (sv && sv->pres_restore) {
            // the pressure this step's solve produced in an earlier run
            if (f64) {
                TRY(ensure_mixed(s, p->mg.precision, st));
                s->prev_ok = 0;
                CU(cudaMemcpyAsync(s->p64, sv->pres_restore, s->ncell * sizeof(double), cudaMemcpyDeviceToDevice, st),
                   "pressure restore");
                s->p64_valid = 1;
                if (!defer_p0) TRY(launch_p0_from_p64(s, st));
            } else {
                CU(cudaMemcpyAsync(s->p[0], sv->pres_restore, s->ncell * sizeof(float), cudaMemcpyDeviceToDevice, st),
                   "pressure restore");
                s->p64_valid = 0;
            }
            s->st.vcycles = sv->vcycles_restore;
            s->st.converged = 1;
            sv->vcycles = sv->vcycles_restore;
        } else {
            TRY(pressure_solve(s, p, c, st, defer_p0));
            if (sv) sv->vcycles = s->st.vcycles;
            if (sv && sv->pres_save) {
                if (f64) CU(cudaMemcpyAsync(sv->pres_save, s->p64, s->ncell * sizeof(double), cudaMemcpyDeviceToDevice, st),
                            "pressure save");
                else CU(cudaMemcpyAsync(sv->pres_save, s->p[0], s->ncell * sizeof(float), cudaMemcpyDeviceToDevice, st),
                        "pressure save");
            }
        }
    }
    if (m & SS_STAGE_UPDATE_VELOCITIES) {
        if (p->mg.precision != SS_PREC_FP32 && s->p64_valid) {
            TRY(launch_update_velocities_p64(s, c, st, defer_p0 ? s->p[0] : nullptr));
        } else {
            if (defer_p0) TRY(launch_p0_from_p64(s, st));
            TRY(launch_update_velocities(s, c, st));
        }
    }
    // divergence left by the projection (statistics): folded into the smoke
    // advection, which loads the same faces, when that stage runs next
    const bool div_after = (m & SS_STAGE_UPDATE_VELOCITIES) && (m & SS_STAGE_RESOLVE_PRESSURE) &&
                           (p->collect_stats || p->mg.tol > 0.0);
    const bool div_in_smoke = div_after && (m & SS_STAGE_ADVECT_SMOKE);
    if (div_after && !div_in_smoke) TRY(launch_divergence(s, false, SLOT_DIV_AFTER, st));
    if (sv) TRY(save_vel(s, sv->proj_vel, st));
    if (m & SS_STAGE_ADVECT_SMOKE) TRY(launch_advect_smoke(s, c, st, div_in_smoke ? SLOT_DIV_AFTER : -1));
    if (div_after) {
        TRY(read_slots(s, st));
        s->st.div_after = sqrt(s->red.host[SLOT_DIV_AFTER]);
        s->st.rel_div = s->st.div_before > 0 ? s->st.div_after / s->st.div_before : 0.0;
    }
    if (m & SS_STAGE_OBSTACLES) {
        if (scene_moving(s)) {
            obstacles_update(s, p->time_step);
            TRY(rasterize_solid(s, st));
        } else {
            obstacles_update(s, p->time_step);  // anchored: only the stored velocity decays
        }
    }
    s->st.steps += 1;
    return SS_OK;
}

int ss_run_physics_step(ss_sim* s, const ss_params* p, int nsteps, void* stream) {
    TRY(check_params(s, p));
    if (nsteps < 0) return set_error(SS_E_INVALID, "nsteps < 0");
    cudaStream_t st = as_stream(stream);
    s->st.steps = 0;
    s->nlaunch = 0;
    for (int i = 0; i < nsteps; ++i) TRY(do_step(s, p, st));
    s->st.kernel_launches = s->nlaunch;
    CU(cudaGetLastError(), "step");
    if (p->mg.tol > 0.0 && (p->stage_mask & SS_STAGE_RESOLVE_PRESSURE) && !s->st.converged)
        return set_error(SS_E_NOT_CONVERGED, "V-cycle cap reached before the divergence tolerance");
    return SS_OK;
}

int ss_set_force_field(ss_sim* s, int n, const float* field, void* stream) {
    if (!s) return set_error(SS_E_INVALID, "NULL handle");
    if (n < 0 || n > 256) return set_error(SS_E_INVALID, "force field size out of range (0..256)");
    if (n > 0 && s->dim != 3) return set_error(SS_E_UNSUPPORTED, "the force field is 3D only");
    if (n > 0 && !field) return set_error(SS_E_INVALID, "NULL field");
    cudaStream_t st = as_stream(stream);
    const size_t count = (size_t)3 * n * n * n;
    for (size_t i = 0; i < count; ++i)
        if (!std::isfinite(field[i])) return set_error(SS_E_NONFINITE, "force field");
    if (n != s->ff_n) {
        if (s->ffield) CU(cudaStreamSynchronize(st), "force field sync");
        cudaFree(s->ffield);
        s->ffield = nullptr;
        s->ff_n = 0;
        if (n > 0) CU(cudaMalloc((void**)&s->ffield, count * sizeof(float)), "cudaMalloc(force field)");
    }
    if (n > 0) {
        CU(cudaMemcpyAsync(s->ffield, field, count * sizeof(float), cudaMemcpyHostToDevice, st), "force field");
        CU(cudaStreamSynchronize(st), "force field sync");
    }
    s->ff_n = n;
    return SS_OK;
}

int ss_get_stats(ss_sim* s, ss_stats* out) {
    if (!s || !out) return set_error(SS_E_INVALID, "NULL argument");
    *out = s->st;
    return s->err_armed ? check_device_error(s, nullptr) : SS_OK;
}

// ------------------------------------------------------------ single stages
int ss_update_emitters_status(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    emitters_status(s, p->current_time);
    return upload_array((void**)&s->d_em, &s->cap_em, s->em.data(), sizeof(ss_emitter), (int)s->em.size(), as_stream(stream));
}

int ss_handle_emitters(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    cudaStream_t st = as_stream(stream);
    TRY(upload_array((void**)&s->d_em, &s->cap_em, s->em.data(), sizeof(ss_emitter), (int)s->em.size(), st));
    TRY(launch_emitters(s, make_consts(s, p), st));
    return launch_force_field(s, make_consts(s, p), st);
}

int ss_advect_velocities(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    return launch_advect_velocities(s, make_consts(s, p), false, as_stream(stream));
}

int ss_apply_buoyancy(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    return launch_buoyancy(s, make_consts(s, p), as_stream(stream));
}

int ss_apply_vorticity(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    return launch_vorticity(s, make_consts(s, p), as_stream(stream));
}

int ss_multigrid_pressure_solve(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    cudaStream_t st = as_stream(stream);
    TRY(pressure_solve(s, p, make_consts(s, p), st));
    if (p->mg.tol > 0.0 && !s->st.converged)
        return set_error(SS_E_NOT_CONVERGED, "V-cycle cap reached before the divergence tolerance");
    return SS_OK;
}

int ss_v_cycle(ss_sim* s, const ss_params* p, int level, void* stream) {
    TRY(check_params(s, p));
    if (level == 0) s->p64_valid = 0;
    if (level < 0 || level >= s->levels) return set_error(SS_E_INVALID, "level out of range");
    cudaStream_t st = as_stream(stream);
    TRY(ensure_pyramid(s, st));
    const StepConsts c = make_consts(s, p);
    if (level != 0) return v_cycle_rec(s, c, p->mg, level, st);
    TRY(launch_divergence(s, true, -1, st, &c, p->mg.ref_quirks));
    const bool rb = rb_supported(s, p->mg.ref_quirks);
    if (rb) TRY(launch_rb_convert(s, true, st));
    s->rb_active = rb ? 1 : 0;
    const int rc = v_cycle_rec(s, c, p->mg, 0, st);
    s->rb_active = 0;
    if (rc) return rc;
    if (rb) TRY(launch_rb_convert(s, false, st));
    return SS_OK;
}

int ss_smooth(ss_sim* s, const ss_params* p, int level, int iterations, void* stream) {
    TRY(check_params(s, p));
    if (level == 0) s->p64_valid = 0;
    if (level < 0 || level >= s->levels || iterations < 0) return set_error(SS_E_INVALID, "level/iterations out of range");
    cudaStream_t st = as_stream(stream);
    TRY(ensure_pyramid(s, st));
    const StepConsts c = make_consts(s, p);
    if (level == 0 && rb_supported(s, p->mg.ref_quirks)) {
        // the colour-split sweeps the V-cycle uses (same values)
        TRY(launch_divergence(s, true, -1, st, &c, p->mg.ref_quirks));
        TRY(launch_rb_convert(s, true, st));
        TRY(launch_rb_sweep(s, iterations, st));
        return launch_rb_convert(s, false, st);
    }
    if (level == 0) TRY(launch_divergence(s, true, -1, st));
    return launch_smooth(s, c, level, iterations, p->mg.ref_quirks, st);
}

int ss_compute_residual(ss_sim* s, const ss_params* p, int level, void* stream) {
    TRY(check_params(s, p));
    if (level < 0 || level >= s->levels) return set_error(SS_E_INVALID, "level out of range");
    cudaStream_t st = as_stream(stream);
    TRY(ensure_pyramid(s, st));
    if (level == 0) TRY(launch_divergence(s, true, -1, st));
    return launch_residual(s, make_consts(s, p), level, true, false, p->mg.ref_quirks, st);
}

int ss_compute_restrict(ss_sim* s, const ss_params* p, int level, void* stream) {
    TRY(check_params(s, p));
    if (level < 0 || level + 1 >= s->levels) return set_error(SS_E_INVALID, "level out of range");
    cudaStream_t st = as_stream(stream);
    TRY(ensure_pyramid(s, st));
    return launch_restrict(s, level, st);
}

int ss_prolong_and_add(ss_sim* s, const ss_params* p, int level, void* stream) {
    TRY(check_params(s, p));
    if (level == 0) s->p64_valid = 0;
    if (level < 0 || level >= s->levels) return set_error(SS_E_INVALID, "level out of range");
    return launch_prolong(s, level, as_stream(stream));
}

int ss_update_velocities(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    if (p->mg.precision != SS_PREC_FP32 && s->p64_valid)
        return launch_update_velocities_p64(s, make_consts(s, p), as_stream(stream));
    return launch_update_velocities(s, make_consts(s, p), as_stream(stream));
}

int ss_advect_smoke(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    return launch_advect_smoke(s, make_consts(s, p), as_stream(stream));
}

int ss_obstacle_update_step(ss_sim* s, const ss_params* p, void* stream) {
    TRY(check_params(s, p));
    obstacles_update(s, p->time_step);
    if (scene_moving(s)) TRY(rasterize_solid(s, as_stream(stream)));
    return SS_OK;
}

int ss_update_solid_map(ss_sim* s, void* stream) {
    if (!s) return set_error(SS_E_INVALID, "NULL handle");
    return rasterize_solid(s, as_stream(stream));
}

int ss_init_solid_map(ss_sim* s, void* stream) {
    if (!s) return set_error(SS_E_INVALID, "NULL handle");
    return rasterize_solid(s, as_stream(stream));
}

}  // extern "C"

int ss::run_step(ss_sim* s, const ss_params* p, cudaStream_t st, StepSaves* saves) { return do_step(s, p, st, saves); }
