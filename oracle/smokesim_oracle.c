/*
 * smokesim_oracle.c -- TEST INFRASTRUCTURE, not product code.
 *
 * A CPU restatement (C11 + OpenMP) of SmokeSim's per-frame smoke step, used
 * only as the checker of the CUDA path (tests, __graft_entry__.smoke and the
 * CPU-baseline leg of bench.py).  Built twice: `real` = float (parity oracle
 * and timed CPU baseline) and `real` = double (accuracy oracle).
 *
 * Parity unpinned: the reference is GLSL 4.60 compute run by an OpenGL driver
 * that neither this machine nor the GPU machine has, and it ships no tests,
 * golden vectors or fixtures.  Each function below restates one compute shader
 * (or one host routine) and cites the reference file:line it follows; it keeps
 * the reference's ping-pong buffers, red-black ordering, in-place residual,
 * V-cycle recursion and GL border/clamp semantics.  Texture filtering is
 * written out as explicit nested linear interpolation in `real` arithmetic
 * (GL hardware uses fixed-point weights, so no CPU restatement can match a
 * GPU's texture unit bit for bit).  Where the reference reads a texel outside
 * its texture (calculate_vorticity's off-by-one bound) the fetch returns 0.
 *
 * Deliberate, documented choices where the reference leaves freedom:
 *  - back-trace in grid units: p - v*(dt/h) instead of (p*h - v*dt)/h;
 *  - texel coordinates are formed directly (texel centre at integer index)
 *    instead of through normalised uv;
 *  - lerp(a,b,t) = a*(1-t) + b*t, applied x, then y, then z;
 *  - texel coordinates are clamped to [-2, size+1] before floor (values out
 *    there sample only border texels).
 * Extensions (parameters, absent from the reference): emitter face-velocity
 * injection, box obstacles, multiple V-cycles / tolerance solves, the
 * post-smoothing right-hand-side fix (ref_quirks = 0) and divergence norms.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/smokesim.h"

#ifdef OG_DOUBLE
typedef double real;
#else
typedef float real;
#endif

#define OMP_FOR _Pragma("omp parallel for collapse(2) schedule(static)")

typedef struct og_sim {
    int dim, nx, ny, nz, nch, enclosed, min_coarse;
    real h;
    float t_ambient0;
    size_t ncell, nvx, nvy, nvz;
    real *vx[2], *vy[2], *vz[2];
    int vxi, vyi, vzi;
    real *smoke[2][4];        /* r, g, b, a(temperature) */
    int si;
    real *vort[3];
    int levels;
    int ls[SS_MAX_LEVELS][3];
    real *p[SS_MAX_LEVELS], *r[SS_MAX_LEVELS], *solid[SS_MAX_LEVELS][4];
    ss_emitter* em; int ne;
    ss_obstacle* ob; int no;
    ss_box* bx; int nb;
    int fp16_smoke, fp16_vort;  /* optional reference storage rounding (RGBA16F textures) */
    ss_stats st;
    /* mixed-precision projection: FP64 level-0 pressure and the rounding
     * (0 none, SS_PREC_MIXED FP16, SS_PREC_MIXED_BF16) of every coarse-level
     * store of the correction V-cycle */
    double* p64;
    int p64_valid;
    double* p64_prev;   /* the extrapolated warm start's p(n-2) */
    int prev_ok;        /* p64_prev holds the pressure the current p64 was solved from */
    int cround;
    real force[3];   /* control force on the faces inside active emitters */
    real* ff;        /* coarse control force field, 3 * ffn^3 (none: ffn == 0) */
    int ffn;
    /* mixed solve: response matrix of the coarsest level's sweeps,
     * cm[i * cm_n + j] = dp_j / dr_i, with the solid fractions and iteration
     * count it was built for */
    real* cm;
    real* cm_alpha;
    size_t cm_n;
    int cm_iters;
    int cm_off;      /* 1: sweep the coarsest level (the CUDA path's SMOKESIM_COARSE_SWEEPS=1) */
} og_sim;

/* ---------------------------------------------------------------- helpers */
static inline real f16(real x) { return (real)(_Float16)x; }
/* float -> bfloat16 -> float, round to nearest even (finite values) */
static inline real bf16(real x) {
    float f = (float)x;
    uint32_t u;
    memcpy(&u, &f, 4);
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    memcpy(&f, &u, 4);
    return (real)f;
}
static inline real lerp_(real a, real b, real t) { return a * ((real)1 - t) + b * t; }
static inline real clampt(real t, real lo, real hi) { return fmin(fmax(t, lo), hi); }

static inline size_t I3(int x, int y, int z, int ax, int ay) { return ((size_t)z * ay + y) * ax + x; }

static inline real fetch(const real* a, int ax, int ay, int az, int x, int y, int z, real border) {
    if (x < 0 || y < 0 || z < 0 || x >= ax || y >= ay || z >= az) return border;
    return a[I3(x, y, z, ax, ay)];
}

/* GL_LINEAR + CLAMP_TO_BORDER sample at texel-space coordinate (tx,ty,tz). */
static real sample_border(const real* a, int dim, int ax, int ay, int az,
                          real tx, real ty, real tz, real border) {
    tx = clampt(tx, (real)-2, (real)(ax + 1));
    ty = clampt(ty, (real)-2, (real)(ay + 1));
    real fx = floor(tx), fy = floor(ty);
    int x0 = (int)fx, y0 = (int)fy;
    real wx = tx - fx, wy = ty - fy;
    if (dim == 2) {
        real c00 = fetch(a, ax, ay, 1, x0, y0, 0, border), c10 = fetch(a, ax, ay, 1, x0 + 1, y0, 0, border);
        real c01 = fetch(a, ax, ay, 1, x0, y0 + 1, 0, border), c11 = fetch(a, ax, ay, 1, x0 + 1, y0 + 1, 0, border);
        return lerp_(lerp_(c00, c10, wx), lerp_(c01, c11, wx), wy);
    }
    tz = clampt(tz, (real)-2, (real)(az + 1));
    real fz = floor(tz);
    int z0 = (int)fz;
    real wz = tz - fz;
    real c000 = fetch(a, ax, ay, az, x0, y0, z0, border), c100 = fetch(a, ax, ay, az, x0 + 1, y0, z0, border);
    real c010 = fetch(a, ax, ay, az, x0, y0 + 1, z0, border), c110 = fetch(a, ax, ay, az, x0 + 1, y0 + 1, z0, border);
    real c001 = fetch(a, ax, ay, az, x0, y0, z0 + 1, border), c101 = fetch(a, ax, ay, az, x0 + 1, y0, z0 + 1, border);
    real c011 = fetch(a, ax, ay, az, x0, y0 + 1, z0 + 1, border), c111 = fetch(a, ax, ay, az, x0 + 1, y0 + 1, z0 + 1, border);
    real c0 = lerp_(lerp_(c000, c100, wx), lerp_(c010, c110, wx), wy);
    real c1 = lerp_(lerp_(c001, c101, wx), lerp_(c011, c111, wx), wy);
    return lerp_(c0, c1, wz);
}

/* GL_LINEAR + CLAMP_TO_EDGE sample (pressure pyramid, 3d/grid3d.c:63). */
static inline int clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }
static real sample_edge(const real* a, int dim, int ax, int ay, int az, real tx, real ty, real tz) {
    real fx = floor(tx), fy = floor(ty);
    int x0 = (int)fx, y0 = (int)fy;
    real wx = tx - fx, wy = ty - fy;
    int xa = clampi(x0, ax), xb = clampi(x0 + 1, ax), ya = clampi(y0, ay), yb = clampi(y0 + 1, ay);
    if (dim == 2) {
        real c00 = a[I3(xa, ya, 0, ax, ay)], c10 = a[I3(xb, ya, 0, ax, ay)];
        real c01 = a[I3(xa, yb, 0, ax, ay)], c11 = a[I3(xb, yb, 0, ax, ay)];
        return lerp_(lerp_(c00, c10, wx), lerp_(c01, c11, wx), wy);
    }
    real fz = floor(tz);
    int z0 = (int)fz;
    real wz = tz - fz;
    int za = clampi(z0, az), zb = clampi(z0 + 1, az);
    real c0 = lerp_(lerp_(a[I3(xa, ya, za, ax, ay)], a[I3(xb, ya, za, ax, ay)], wx),
                    lerp_(a[I3(xa, yb, za, ax, ay)], a[I3(xb, yb, za, ax, ay)], wx), wy);
    real c1 = lerp_(lerp_(a[I3(xa, ya, zb, ax, ay)], a[I3(xb, ya, zb, ax, ay)], wx),
                    lerp_(a[I3(xa, yb, zb, ax, ay)], a[I3(xb, yb, zb, ax, ay)], wx), wy);
    return lerp_(c0, c1, wz);
}

#define NX s->nx
#define NY s->ny
#define NZ s->nz
#define VX(b) s->vx[b]
#define CUR_VX s->vx[s->vxi]
#define CUR_VY s->vy[s->vyi]
#define CUR_VZ s->vz[s->vzi]
#define OTH_VX s->vx[1 - s->vxi]
#define OTH_VY s->vy[1 - s->vyi]
#define OTH_VZ s->vz[1 - s->vzi]

static inline real alpha0(const og_sim* s, int x, int y, int z) { return s->solid[0][3][I3(x, y, z, NX, NY)]; }

/* velocity at grid-space point g (reference get_interpolated_velocity,
 * shaders3d/compute/advect_vx.comp:33-46; 2D advect_vx.comp:31-42). */
static void interp_velocity(const og_sim* s, real gx, real gy, real gz, real v[3]) {
    const real hf = (real)0.5;
    if (s->dim == 2) {
        v[0] = sample_border(CUR_VX, 2, NX + 1, NY, 1, gx, gy - hf, 0, 0);
        v[1] = sample_border(CUR_VY, 2, NX, NY + 1, 1, gx - hf, gy, 0, 0);
        v[2] = 0;
        return;
    }
    v[0] = sample_border(CUR_VX, 3, NX + 1, NY, NZ, gx, gy - hf, gz - hf, 0);
    v[1] = sample_border(CUR_VY, 3, NX, NY + 1, NZ, gx - hf, gy, gz - hf, 0);
    v[2] = sample_border(CUR_VZ, 3, NX, NY, NZ + 1, gx - hf, gy - hf, gz, 0);
}

void og_set_scene(struct og_sim* s, const ss_emitter* em, int ne, const ss_obstacle* ob, int no, const ss_box* bx, int nb);

/* ---------------------------------------------------------------- lifetime */
og_sim* og_create(const ss_desc* d) {
    if (!d || (d->dim != 2 && d->dim != 3)) return NULL;
    og_sim* s = (og_sim*)calloc(1, sizeof(og_sim));
    s->dim = d->dim; s->nx = d->n[0]; s->ny = d->n[1]; s->nz = d->dim == 2 ? 1 : d->n[2];
    s->nch = d->density_channels == 3 ? 3 : 1;
    s->enclosed = d->enclosed;
    s->min_coarse = d->min_coarse > 0 ? d->min_coarse : 4;
    s->h = (real)d->cell_size;
    s->t_ambient0 = d->t_ambient;
    s->ncell = (size_t)NX * NY * NZ;
    s->nvx = (size_t)(NX + 1) * NY * NZ;
    s->nvy = (size_t)NX * (NY + 1) * NZ;
    s->nvz = s->dim == 3 ? (size_t)NX * NY * (NZ + 1) : 0;
    for (int b = 0; b < 2; ++b) {
        s->vx[b] = (real*)calloc(s->nvx, sizeof(real));
        s->vy[b] = (real*)calloc(s->nvy, sizeof(real));
        s->vz[b] = (real*)calloc(s->nvz ? s->nvz : 1, sizeof(real));
        for (int c = 0; c < 4; ++c) {
            s->smoke[b][c] = (real*)calloc(s->ncell, sizeof(real));
        }
        for (size_t i = 0; i < s->ncell; ++i) s->smoke[b][3][i] = (real)d->t_ambient;
    }
    for (int c = 0; c < 3; ++c) s->vort[c] = (real*)calloc(s->ncell, sizeof(real));
    /* pyramid: reference gen_grid_pressure_solve_textures3d (3d/grid3d.c:45-68),
     * generalised to stop at min_coarse instead of 4. */
    int dims[3] = {NX, NY, NZ};
    int lv = 0;
    while (lv < SS_MAX_LEVELS) {
        int ok = dims[0] >= s->min_coarse && dims[1] >= s->min_coarse && (s->dim == 2 || dims[2] >= s->min_coarse);
        if (!ok) break;
        s->ls[lv][0] = dims[0]; s->ls[lv][1] = dims[1]; s->ls[lv][2] = s->dim == 2 ? 1 : dims[2];
        size_t n = (size_t)s->ls[lv][0] * s->ls[lv][1] * s->ls[lv][2];
        s->p[lv] = (real*)calloc(n, sizeof(real));
        s->r[lv] = (real*)calloc(n, sizeof(real));
        for (int c = 0; c < 4; ++c) s->solid[lv][c] = (real*)calloc(n, sizeof(real));
        dims[0] /= 2; dims[1] /= 2; if (s->dim == 3) dims[2] /= 2;
        ++lv;
    }
    s->levels = lv;
    if (lv == 0) {  /* grid smaller than min_coarse: single level */
        s->ls[0][0] = NX; s->ls[0][1] = NY; s->ls[0][2] = NZ;
        s->p[0] = (real*)calloc(s->ncell, sizeof(real));
        s->r[0] = (real*)calloc(s->ncell, sizeof(real));
        for (int c = 0; c < 4; ++c) s->solid[0][c] = (real*)calloc(s->ncell, sizeof(real));
        s->levels = 1;
    }
    s->em = (ss_emitter*)calloc(SS_MAX_EMITTERS, sizeof(ss_emitter));
    s->ob = (ss_obstacle*)calloc(SS_MAX_OBSTACLES, sizeof(ss_obstacle));
    s->bx = (ss_box*)calloc(SS_MAX_BOXES, sizeof(ss_box));
    og_set_scene(s, NULL, 0, NULL, 0, NULL, 0);  /* wall shell of an enclosed grid */
    return s;
}

void og_destroy(og_sim* s) {
    if (!s) return;
    for (int b = 0; b < 2; ++b) {
        free(s->vx[b]); free(s->vy[b]); free(s->vz[b]);
        for (int c = 0; c < 4; ++c) free(s->smoke[b][c]);
    }
    for (int c = 0; c < 3; ++c) free(s->vort[c]);
    for (int l = 0; l < s->levels; ++l) {
        free(s->p[l]); free(s->r[l]);
        for (int c = 0; c < 4; ++c) free(s->solid[l][c]);
    }
    free(s->em); free(s->ob); free(s->bx);
    free(s->p64);
    free(s->p64_prev);
    free(s->cm);
    free(s->cm_alpha);
    free(s->ff);
    free(s);
}

int og_levels(const og_sim* s, int sizes[][3]) {
    for (int l = 0; l < s->levels; ++l) { sizes[l][0] = s->ls[l][0]; sizes[l][1] = s->ls[l][1]; sizes[l][2] = s->ls[l][2]; }
    return s->levels;
}

void og_set_fp16_storage(og_sim* s, int smoke, int vort) { s->fp16_smoke = smoke; s->fp16_vort = vort; }

/* ------------------------------------------------------------ solid map */
/* init_solid_map (shaders3d/compute/init_solid_map.comp:34-48; 2D :32-45) */
void og_init_solid_map(og_sim* s) {
    OMP_FOR
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                int shell = x == 0 || x == NX - 1 || y == 0 || y == NY - 1 ||
                            (s->dim == 3 && (z == 0 || z == NZ - 1));
                if (shell) {
                    size_t i = I3(x, y, z, NX, NY);
                    s->solid[0][0][i] = 0; s->solid[0][1][i] = 0; s->solid[0][2][i] = 0; s->solid[0][3][i] = 1;
                }
            }
}

/* update_solid_map (shaders3d/compute/update_solid_map.comp:46-83; 2D :44-81):
 * cells with 2 <= idx <= n-2 on every axis; last obstacle wins.  Boxes are an
 * extension rasterised after the spheres with the same valid range. */
void og_update_solid_map(og_sim* s) {
    OMP_FOR
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                int invalid = x <= 1 || y <= 1 || x >= NX - 1 || y >= NY - 1 ||
                              (s->dim == 3 && (z <= 1 || z >= NZ - 1));
                if (invalid) continue;
                real nv[4] = {0, 0, 0, 0};
                for (int i = 0; i < s->no; ++i) {
                    const ss_obstacle* o = &s->ob[i];
                    real dx = (real)x - (real)o->pos[0], dy = (real)y - (real)o->pos[1];
                    real d2 = dx * dx + dy * dy;
                    if (s->dim == 3) { real dz = (real)z - (real)o->pos[2]; d2 = d2 + dz * dz; }
                    real dist = sqrt(d2);
                    if (dist < (real)o->radius) {
                        real m = (real)1 - (real)o->anchored;
                        nv[0] = (real)o->velocity[0] * m; nv[1] = (real)o->velocity[1] * m;
                        nv[2] = s->dim == 3 ? (real)o->velocity[2] * m : 0; nv[3] = 1;
                    }
                }
                for (int i = 0; i < s->nb; ++i) {
                    const ss_box* b = &s->bx[i];
                    int in = (real)x >= (real)b->lo[0] && (real)x < (real)b->hi[0] &&
                             (real)y >= (real)b->lo[1] && (real)y < (real)b->hi[1] &&
                             (s->dim == 2 || ((real)z >= (real)b->lo[2] && (real)z < (real)b->hi[2]));
                    if (in) {
                        real m = (real)1 - (real)b->anchored;
                        nv[0] = (real)b->velocity[0] * m; nv[1] = (real)b->velocity[1] * m;
                        nv[2] = s->dim == 3 ? (real)b->velocity[2] * m : 0; nv[3] = 1;
                    }
                }
                size_t i = I3(x, y, z, NX, NY);
                for (int c = 0; c < 4; ++c) s->solid[0][c][i] = f16(nv[c]);
            }
}

/* obstacle_update (shaders3d/compute/obstacle_update.comp:51-135; 2D
 * obstacle_update.comp:49-131): gravity, wall bounce 0.999, pairwise push-out
 * against the INPUT positions, damping 0.999.  The 2D shader is dispatched with
 * an 8x8 local size as if it were 128 wide (common/physics/grid.c:156-162), so
 * the reference updates only the first 8 of every 128 obstacles and reads
 * unwritten shared memory; here every obstacle is updated as in 3D. */
void og_obstacle_update(og_sim* s, real dt) {
    int n = s->no;
    if (n == 0) return;
    ss_obstacle* in = (ss_obstacle*)malloc(sizeof(ss_obstacle) * n);
    memcpy(in, s->ob, sizeof(ss_obstacle) * n);
    const int d3 = s->dim == 3;
    for (int i = 0; i < n; ++i) {
        real pos[3] = {in[i].pos[0], in[i].pos[1], d3 ? in[i].pos[2] : 0};
        real vel[3] = {in[i].velocity[0], in[i].velocity[1], d3 ? in[i].velocity[2] : 0};
        real r = in[i].radius, anchored = in[i].anchored, movable = (real)1 - anchored;
        int anchored_flag = anchored == 1;
        if (!anchored_flag) {
            vel[1] = vel[1] + (real)-9.81f * dt * movable;
            vel[0] = vel[0] + (real)0 * dt * movable;
            if (d3) vel[2] = vel[2] + (real)0 * dt * movable;
            for (int c = 0; c < (d3 ? 3 : 2); ++c) pos[c] = pos[c] + vel[c] * dt * movable;
            real maxb[3] = {(real)s->nx, (real)s->ny, (real)s->nz};
            const real B = (real)0.999f;
            for (int c = 0; c < (d3 ? 3 : 2); ++c) {
                if (pos[c] - r < 0) { pos[c] = 0 + r; vel[c] *= -B; }
                if (pos[c] + r > maxb[c]) { pos[c] = maxb[c] - r; vel[c] *= -B; }
            }
            for (int j = 0; j < n; ++j) {
                if (j == i) continue;
                real d[3] = {pos[0] - in[j].pos[0], pos[1] - in[j].pos[1], d3 ? pos[2] - in[j].pos[2] : 0};
                real dist = d3 ? sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) : sqrt(d[0] * d[0] + d[1] * d[1]);
                real min_dist = r + in[j].radius;
                if (dist < min_dist && dist > (real)0.0001f) {
                    real nn[3] = {d[0] / dist, d[1] / dist, d[2] / dist};
                    for (int c = 0; c < (d3 ? 3 : 2); ++c) pos[c] += nn[c] * (min_dist - dist) * (real)0.5f * movable;
                    real rv[3] = {vel[0] - in[j].velocity[0], vel[1] - in[j].velocity[1], d3 ? vel[2] - in[j].velocity[2] : 0};
                    real vn = d3 ? rv[0] * nn[0] + rv[1] * nn[1] + rv[2] * nn[2] : rv[0] * nn[0] + rv[1] * nn[1];
                    if (vn < 0) for (int c = 0; c < (d3 ? 3 : 2); ++c) vel[c] -= vn * nn[c] * movable;
                }
            }
        }
        s->ob[i].pos[0] = (float)pos[0]; s->ob[i].pos[1] = (float)pos[1]; if (d3) s->ob[i].pos[2] = (float)pos[2];
        s->ob[i].velocity[0] = (float)(vel[0] * (real)0.999f);
        s->ob[i].velocity[1] = (float)(vel[1] * (real)0.999f);
        if (d3) s->ob[i].velocity[2] = (float)(vel[2] * (real)0.999f);
    }
    free(in);
}

void og_set_scene(og_sim* s, const ss_emitter* em, int ne, const ss_obstacle* ob, int no, const ss_box* bx, int nb) {
    s->ne = ne; s->no = no; s->nb = nb;
    if (ne) memcpy(s->em, em, sizeof(ss_emitter) * ne);
    if (no) memcpy(s->ob, ob, sizeof(ss_obstacle) * no);
    if (nb) memcpy(s->bx, bx, sizeof(ss_box) * nb);
    for (int c = 0; c < 4; ++c) memset(s->solid[0][c], 0, sizeof(real) * s->ncell);
    if (s->enclosed) og_init_solid_map(s);
    og_update_solid_map(s);
}

void og_get_scene(const og_sim* s, ss_emitter* em, int ne, ss_obstacle* ob, int no) {
    if (em) memcpy(em, s->em, sizeof(ss_emitter) * (ne < s->ne ? ne : s->ne));
    if (ob) memcpy(ob, s->ob, sizeof(ss_obstacle) * (no < s->no ? no : s->no));
}

/* ------------------------------------------------------------- emitters */
/* update_emitters_status (shaders3d/compute/update_emitters_status.comp:49-59).
 * The 2D shader has the same body but the 8x8 local size / 128-wide dispatch
 * mismatch (common/physics/grid.c:89-93); here every emitter is updated. */
void og_update_emitters_status(og_sim* s, float current_time) {
    for (int i = 0; i < s->ne; ++i) {
        ss_emitter* e = &s->em[i];
        if (e->emit == 1 && e->delay != 0) { e->emit = 0; e->last_emit = (int)current_time; continue; }
        if (current_time - (float)e->last_emit >= (float)e->delay) e->emit = 1;
    }
}

static inline real emitter_dist(const og_sim* s, const ss_emitter* e, int x, int y, int z) {
    real dx = (real)x - (real)e->pos[0], dy = (real)y - (real)e->pos[1];
    real d2 = dx * dx + dy * dy;
    if (s->dim == 3) { real dz = (real)z - (real)e->pos[2]; d2 = d2 + dz * dz; }
    return sqrt(d2);
}

/* handle_emitters (shaders3d/compute/handle_emitters.comp:49-76; 2D :47-74):
 * smoke.rgb += rho_e*falloff*dt, smoke.a += T_e*falloff*dt inside the radius;
 * falloff = smoothstep(r, 0, dist) (literal edge order) or 1. */
void og_handle_emitters(og_sim* s, real dt) {
    int cur = s->si, oth = 1 - s->si;
    OMP_FOR
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                size_t i = I3(x, y, z, NX, NY);
                real sm[4] = {s->smoke[cur][0][i], s->smoke[cur][1][i], s->smoke[cur][2][i], s->smoke[cur][3][i]};
                for (int k = 0; k < s->ne; ++k) {
                    const ss_emitter* e = &s->em[k];
                    if (!(e->emit > 0)) continue;
                    real dist = emitter_dist(s, e, x, y, z);
                    real rad = (real)e->radius;
                    if (dist < rad) {
                        real falloff;
                        if (e->falloff > 0) {
                            real t = (dist - rad) / ((real)0 - rad);
                            t = clampt(t, 0, 1);
                            falloff = t * t * ((real)3 - (real)2 * t);
                        } else {
                            falloff = 1;
                        }
                        for (int c = 0; c < s->nch; ++c) sm[c] = sm[c] + (real)e->density[c] * falloff * dt;
                        sm[3] = sm[3] + (real)e->temperature * falloff * dt;
                    }
                }
                for (int c = 0; c < 4; ++c) s->smoke[oth][c][i] = s->fp16_smoke ? f16(sm[c]) : sm[c];
            }
    s->si = oth;
}

/* Extension: emitter face-velocity injection (in place on the current buffers).
 * A face whose integer index lies inside an active emitter with set_velocity
 * takes that emitter's velocity component (last emitter wins). */
/* Extension: set_velocity emitters overwrite the face velocities inside
 * them; a control force adds dt * force to every face inside an active
 * emitter afterwards. */
void og_emitter_velocity(og_sim* s, real dt) {
    const int forced = s->force[0] != 0 || s->force[1] != 0 || s->force[2] != 0;
    int any = forced;
    for (int k = 0; k < s->ne; ++k) any |= (s->em[k].emit > 0 && s->em[k].set_velocity);
    if (!any) return;
    for (int comp = 0; comp < s->dim; ++comp) {
        int ax = NX + (comp == 0), ay = NY + (comp == 1), az = NZ + (comp == 2);
        real* a = comp == 0 ? CUR_VX : comp == 1 ? CUR_VY : CUR_VZ;
        OMP_FOR
        for (int z = 0; z < az; ++z)
            for (int y = 0; y < ay; ++y)
                for (int x = 0; x < ax; ++x) {
                    int inside = 0;
                    for (int k = 0; k < s->ne; ++k) {
                        const ss_emitter* e = &s->em[k];
                        if (!(e->emit > 0)) continue;
                        if (emitter_dist(s, e, x, y, z) < (real)e->radius) {
                            inside = 1;
                            if (e->set_velocity) a[I3(x, y, z, ax, ay)] = (real)e->velocity[comp];
                        }
                    }
                    if (forced && inside) a[I3(x, y, z, ax, ay)] = a[I3(x, y, z, ax, ay)] + dt * s->force[comp];
                }
    }
}

/* Extension: coarse control force field.  Three components on n^3
 * cell-centred samples over the domain; each face takes dt times the
 * GL_LINEAR + CLAMP_TO_EDGE sample of its component at the face position
 * (texel coordinate (pos / N) * n - 1/2), after the emitters.  3D only. */
static void og_apply_force_field(og_sim* s, real dt) {
    if (s->ffn <= 0 || s->dim != 3) return;
    const int n = s->ffn;
    const size_t nn = (size_t)n * n * n;
    for (int comp = 0; comp < 3; ++comp) {
        int ax = NX + (comp == 0), ay = NY + (comp == 1), az = NZ + (comp == 2);
        real* a = comp == 0 ? CUR_VX : comp == 1 ? CUR_VY : CUR_VZ;
        const real* f = s->ff + comp * nn;
        OMP_FOR
        for (int z = 0; z < az; ++z)
            for (int y = 0; y < ay; ++y)
                for (int x = 0; x < ax; ++x) {
                    const real xf = (real)x + (comp == 0 ? (real)0 : (real)0.5);
                    const real yf = (real)y + (comp == 1 ? (real)0 : (real)0.5);
                    const real zf = (real)z + (comp == 2 ? (real)0 : (real)0.5);
                    const real tx = (xf / (real)NX) * (real)n - (real)0.5;
                    const real ty = (yf / (real)NY) * (real)n - (real)0.5;
                    const real tz = (zf / (real)NZ) * (real)n - (real)0.5;
                    const real val = sample_edge(f, 3, n, n, n, tx, ty, tz);
                    a[I3(x, y, z, ax, ay)] = a[I3(x, y, z, ax, ay)] + dt * val;
                }
    }
}

void og_set_force_field(og_sim* s, int n, const float* f) {
    free(s->ff);
    s->ff = NULL;
    s->ffn = 0;
    if (n <= 0 || !f) return;
    const size_t cnt = (size_t)3 * n * n * n;
    s->ff = (real*)malloc(cnt * sizeof(real));
    for (size_t i = 0; i < cnt; ++i) s->ff[i] = (real)f[i];
    s->ffn = n;
}
void og_set_force_field_f64(og_sim* s, int n, const double* f) {
    free(s->ff);
    s->ff = NULL;
    s->ffn = 0;
    if (n <= 0 || !f) return;
    const size_t cnt = (size_t)3 * n * n * n;
    s->ff = (real*)malloc(cnt * sizeof(real));
    for (size_t i = 0; i < cnt; ++i) s->ff[i] = (real)f[i];
    s->ffn = n;
}

void og_set_emitter_force(og_sim* s, const float f[3]) {
    for (int d = 0; d < 3; ++d) s->force[d] = d < s->dim ? (real)f[d] : (real)0;
}
void og_set_emitter_force_f64(og_sim* s, const double f[3]) {
    for (int d = 0; d < 3; ++d) s->force[d] = d < s->dim ? (real)f[d] : (real)0;
}

/* ------------------------------------------------------------- advection */
static inline int solid_oob1(const og_sim* s, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ) return 1;
    return alpha0(s, x, y, z) >= 1;
}
static inline int solid_oob0(const og_sim* s, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ) return 0;
    return alpha0(s, x, y, z) >= 1;
}

/* advect_vx/vy/vz (shaders3d/compute/advect_vx.comp:54-77, advect_vy.comp:55-79,
 * advect_vz.comp:55-78; 2D advect_vx.comp:50-73, advect_vy.comp:51-75). */
static void advect_velocities_impl(og_sim* s, real dt, const real wind[3]) {
    const real hf = (real)0.5, cfl = dt / s->h;
    for (int comp = 0; comp < s->dim; ++comp) {
        int ax = NX + (comp == 0), ay = NY + (comp == 1), az = NZ + (comp == 2);
        const real* src = comp == 0 ? CUR_VX : comp == 1 ? CUR_VY : CUR_VZ;
        real* dst = comp == 0 ? OTH_VX : comp == 1 ? OTH_VY : OTH_VZ;
        OMP_FOR
        for (int z = 0; z < az; ++z)
            for (int y = 0; y < ay; ++y)
                for (int x = 0; x < ax; ++x) {
                    size_t i = I3(x, y, z, ax, ay);
                    int id[3] = {x, y, z};
                    if (id[comp] == 0 && wind[comp] != 0) { dst[i] = wind[comp]; continue; }
                    int xm = x - (comp == 0), ym = y - (comp == 1), zm = z - (comp == 2);
                    if (solid_oob1(s, x, y, z) || solid_oob1(s, xm, ym, zm)) { dst[i] = 0; continue; }
                    real g[3] = {(real)x + (comp == 0 ? 0 : hf), (real)y + (comp == 1 ? 0 : hf),
                                 s->dim == 3 ? (real)z + (comp == 2 ? 0 : hf) : 0};
                    real v[3];
                    interp_velocity(s, g[0], g[1], g[2], v);
                    real b[3] = {g[0] - v[0] * cfl, g[1] - v[1] * cfl, g[2] - v[2] * cfl};
                    real t[3] = {b[0] - (comp == 0 ? 0 : hf), b[1] - (comp == 1 ? 0 : hf), b[2] - (comp == 2 ? 0 : hf)};
                    dst[i] = sample_border(src, s->dim, ax, ay, az, t[0], t[1], t[2], 0);
                }
    }
    s->vxi ^= 1; s->vyi ^= 1; if (s->dim == 3) s->vzi ^= 1;
}

/* advect_smoke (shaders3d/compute/advect_smoke.comp:55-72; 2D :51-68) */
static void advect_smoke_impl(og_sim* s, real dt, real t_amb) {
    const real hf = (real)0.5, cfl = dt / s->h;
    int cur = s->si, oth = 1 - s->si;
    OMP_FOR
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                size_t i = I3(x, y, z, NX, NY);
                if (alpha0(s, x, y, z) >= 1) {
                    s->smoke[oth][0][i] = 0; s->smoke[oth][1][i] = 0; s->smoke[oth][2][i] = 0;
                    s->smoke[oth][3][i] = s->fp16_smoke ? f16(t_amb) : t_amb;
                    continue;
                }
                real g[3] = {(real)x + hf, (real)y + hf, s->dim == 3 ? (real)z + hf : 0};
                real v[3];
                interp_velocity(s, g[0], g[1], g[2], v);
                real b[3] = {g[0] - v[0] * cfl, g[1] - v[1] * cfl, g[2] - v[2] * cfl};
                for (int c = 0; c < 4; ++c) {
                    real border = c == 3 ? t_amb : 0;
                    real val = sample_border(s->smoke[cur][c], s->dim, NX, NY, NZ, b[0] - hf, b[1] - hf, b[2] - hf, border);
                    s->smoke[oth][c][i] = s->fp16_smoke ? f16(val) : val;
                }
            }
    s->si = oth;
}

/* ------------------------------------------------------------- buoyancy */
/* apply_buoyancy (shaders3d/compute/apply_buoyancy.comp:39-52; 2D :37-50).
 * Faces touching solid (out of grid = fluid here) are NOT written: the write
 * buffer keeps its previous content. */
static void apply_buoyancy_impl(og_sim* s, real dt, real t_amb, real alpha, real beta) {
    const real hf = (real)0.5;
    int ax = NX, ay = NY + 1, az = NZ;
    const real* src = CUR_VY;
    real* dst = OTH_VY;
    int cur = s->si;
    OMP_FOR
    for (int z = 0; z < az; ++z)
        for (int y = 0; y < ay; ++y)
            for (int x = 0; x < ax; ++x) {
                if (solid_oob0(s, x, y, z) || solid_oob0(s, x, y - 1, z)) continue;
                real sm[4];
                for (int c = 0; c < 4; ++c)
                    sm[c] = sample_border(s->smoke[cur][c], s->dim, NX, NY, NZ, (real)x, (real)y - hf, (real)z,
                                          c == 3 ? t_amb : 0);
                real total = sm[0] + sm[1] + sm[2];
                real buoy = -alpha * total + beta * (sm[3] - t_amb);
                size_t i = I3(x, y, z, ax, ay);
                dst[i] = src[i] + buoy * dt;
            }
    s->vyi ^= 1;
}

/* ------------------------------------------------------------- vorticity */
static inline real getv(const real* a, int ax, int ay, int az, int x, int y, int z) {
    return fetch(a, ax, ay, az, x, y, z, 0);
}
/* calculate_vorticity (shaders3d/compute/calculate_vorticity.comp:59-84; 2D :51-69) */
static void calculate_vorticity_impl(og_sim* s) {
    const real hf = (real)0.5, two_h = (real)2 * s->h;
    const real *u = CUR_VX, *v = CUR_VY, *w = CUR_VZ;
    const int d3 = s->dim == 3;
#define CCX(X, Y, Z) ((getv(u, NX + 1, NY, NZ, X, Y, Z) + getv(u, NX + 1, NY, NZ, (X) + 1, Y, Z)) * hf)
#define CCY(X, Y, Z) ((getv(v, NX, NY + 1, NZ, X, Y, Z) + getv(v, NX, NY + 1, NZ, X, (Y) + 1, Z)) * hf)
#define CCZ(X, Y, Z) ((getv(w, NX, NY, NZ + 1, X, Y, Z) + getv(w, NX, NY, NZ + 1, X, Y, (Z) + 1)) * hf)
    OMP_FOR
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                size_t i = I3(x, y, z, NX, NY);
                if (alpha0(s, x, y, z) >= 1) { s->vort[0][i] = 0; s->vort[1][i] = 0; s->vort[2][i] = 0; continue; }
                if (!d3) {
                    real z1 = CCY(x + 1, y, 0) - CCY(x - 1, y, 0);
                    real z2 = CCX(x, y + 1, 0) - CCX(x, y - 1, 0);
                    s->vort[0][i] = (z1 - z2) / two_h;
                    continue;
                }
                real x1 = CCZ(x, y + 1, z) - CCZ(x, y - 1, z);
                real x2 = CCY(x, y, z + 1) - CCY(x, y, z - 1);
                real ox = (x1 - x2) / two_h;
                real y1 = CCX(x, y, z + 1) - CCX(x, y, z - 1);
                real y2 = CCZ(x + 1, y, z) - CCZ(x - 1, y, z);
                real oy = (y1 - y2) / two_h;
                real z1 = CCY(x + 1, y, z) - CCY(x - 1, y, z);
                real z2 = CCX(x, y + 1, z) - CCX(x, y - 1, z);
                real oz = (z1 - z2) / two_h;
                if (s->fp16_vort) { ox = f16(ox); oy = f16(oy); oz = f16(oz); }
                s->vort[0][i] = ox; s->vort[1][i] = oy; s->vort[2][i] = oz;
            }
#undef CCX
#undef CCY
#undef CCZ
}

static inline void vort_at(const og_sim* s, int x, int y, int z, real o[3]) {
    if (x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ) { o[0] = o[1] = o[2] = 0; return; }
    size_t i = I3(x, y, z, NX, NY);
    o[0] = s->vort[0][i]; o[1] = s->dim == 3 ? s->vort[1][i] : 0; o[2] = s->dim == 3 ? s->vort[2][i] : 0;
}
static inline real vmag(const og_sim* s, int x, int y, int z) {
    real o[3];
    vort_at(s, x, y, z, o);
    if (s->dim == 2) return fabs(o[0]);
    return sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
}

/* apply_vorticity_x/y/z (shaders3d/compute/apply_vorticity_x.comp:43-63 and
 * siblings; 2D apply_vorticity_x.comp:41-60, apply_vorticity_y.comp:41-60).
 * The force of cell idx is applied to face idx; 2D uses f_x = -n_y*w,
 * f_y = -n_x*w. */
static void apply_vorticity_impl(og_sim* s, real dt, real eps_conf, real rho) {
    const real two_h = (real)2 * s->h, eps = (real)1e-20f, hf = (real)0.5;
    const int d3 = s->dim == 3;
    for (int comp = 0; comp < s->dim; ++comp) {
        int ax = NX + (comp == 0), ay = NY + (comp == 1), az = NZ + (comp == 2);
        const real* src = comp == 0 ? CUR_VX : comp == 1 ? CUR_VY : CUR_VZ;
        real* dst = comp == 0 ? OTH_VX : comp == 1 ? OTH_VY : OTH_VZ;
        OMP_FOR
        for (int z = 0; z < az; ++z)
            for (int y = 0; y < ay; ++y)
                for (int x = 0; x < ax; ++x) {
                    real dx = vmag(s, x + 1, y, z) - vmag(s, x - 1, y, z);
                    real dy = vmag(s, x, y + 1, z) - vmag(s, x, y - 1, z);
                    real f;
                    if (d3) {
                        real dz = vmag(s, x, y, z + 1) - vmag(s, x, y, z - 1);
                        real gx = dx / two_h, gy = dy / two_h, gz = dz / two_h;
                        real len = sqrt(gx * gx + gy * gy + gz * gz) + eps;
                        real nx = gx / len, ny = gy / len, nz = gz / len;
                        real o[3];
                        vort_at(s, x, y, z, o);
                        if (comp == 0) f = ny * o[2] - o[1] * nz;
                        else if (comp == 1) f = nz * o[0] - o[2] * nx;
                        else f = nx * o[1] - o[0] * ny;
                    } else {
                        real gx = dx / two_h, gy = dy / two_h;
                        real len = sqrt(gx * gx + gy * gy) + eps;
                        real nx = gx / len, ny = gy / len;
                        real o[3];
                        vort_at(s, x, y, 0, o);
                        f = comp == 0 ? -ny * o[0] : -nx * o[0];
                    }
                    size_t i = I3(x, y, z, ax, ay);
                    dst[i] = src[i] + (f * hf * eps_conf * s->h * dt) / rho;
                }
    }
    s->vxi ^= 1; s->vyi ^= 1; if (d3) s->vzi ^= 1;
}

/* ------------------------------------------------------------- multigrid */
static inline real hL(const og_sim* s, int L) { return s->h * (real)(1 << L); }
/* value kept by a coarse-level store of the mixed-precision correction solve */
static inline real cstore(const og_sim* s, real v) {
    return s->cround == SS_PREC_MIXED ? f16(v) : s->cround == SS_PREC_MIXED_BF16 ? bf16(v) : v;
}

/* level-0 divergence with solid-velocity substitution; `oob_solid` selects the
 * residual kernel's out-of-grid rule (solid, vec4(0,0,0,1)) instead of the
 * smoother's (fluid, vec4(0)).  smooth.comp:105-113, compute_residual.comp:116-124. */
static inline real delta_v0(const og_sim* s, int x, int y, int z, int oob_solid) {
    const real* S[4] = {s->solid[0][0], s->solid[0][1], s->solid[0][2], s->solid[0][3]};
    real sd[6][4];
    const int off[6][3] = {{0, 1, 0}, {0, -1, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 0, 1}, {0, 0, -1}};
    int nn = s->dim == 3 ? 6 : 4;
    for (int k = 0; k < nn; ++k) {
        int X = x + off[k][0], Y = y + off[k][1], Z = z + off[k][2];
        if (X < 0 || Y < 0 || Z < 0 || X >= NX || Y >= NY || Z >= NZ) {
            sd[k][0] = sd[k][1] = sd[k][2] = 0; sd[k][3] = oob_solid ? 1 : 0;
        } else {
            size_t i = I3(X, Y, Z, NX, NY);
            for (int c = 0; c < 4; ++c) sd[k][c] = S[c][i];
        }
    }
    const real *u = CUR_VX, *v = CUR_VY, *w = CUR_VZ;
    real v_top = sd[0][3] >= 1 ? sd[0][1] : v[I3(x, y + 1, z, NX, NY + 1)];
    real v_bottom = sd[1][3] >= 1 ? sd[1][1] : v[I3(x, y, z, NX, NY + 1)];
    real v_right = sd[2][3] >= 1 ? sd[2][0] : u[I3(x + 1, y, z, NX + 1, NY)];
    real v_left = sd[3][3] >= 1 ? sd[3][0] : u[I3(x, y, z, NX + 1, NY)];
    real d = v_right - v_left + v_top - v_bottom;
    if (s->dim == 3) {
        real v_front = sd[4][3] >= 1 ? sd[4][2] : w[I3(x, y, z + 1, NX, NY)];
        real v_back = sd[5][3] >= 1 ? sd[5][2] : w[I3(x, y, z, NX, NY)];
        d = d + v_front - v_back;
    }
    return d;
}

/* smooth (common/physics/grid.c:211-234 + shaders3d/compute/pressure_solve/smooth.comp:79-136;
 * 2D smooth.comp:74-123). */
/* Out-of-grid rule of the pressure operators.  ref_quirks = 1 keeps the
 * reference's mismatch (smoother: fluid with p = 0; residual: solid).  The
 * corrected mode uses one rule in both, the physical one: solid for an
 * enclosed grid, open (p = 0) otherwise; with the wall shell dissolving on
 * coarse levels (restrict_solid zeroes alpha < 0.5) the reference's rule makes
 * the coarse problems Dirichlet and the V-cycle stalls near 1e-3. */
static inline int smooth_oob_solid(const og_sim* s, int quirks) { return quirks ? 0 : s->enclosed; }
static inline int resid_oob_solid(const og_sim* s, int quirks) { return quirks ? 1 : s->enclosed; }

void og_smooth_mode(og_sim* s, int L, int iterations, real dt, real rho, int quirks);
void og_smooth(og_sim* s, int L, int iterations, real dt, real rho) { og_smooth_mode(s, L, iterations, dt, rho, 1); }
void og_smooth_mode(og_sim* s, int L, int iterations, real dt, real rho, int quirks) {
    const real oobA = (real)smooth_oob_solid(s, quirks);
    const int ax = s->ls[L][0], ay = s->ls[L][1], az = s->ls[L][2];
    real* P = s->p[L];
    const real* R = s->r[L];
    real* const* SD = s->solid[L];
    const real h = hL(s, L);
    const int d3 = s->dim == 3;
    int parity = 0;
    for (int it = 0; it < iterations * 2; ++it) {
        OMP_FOR
        for (int z = 0; z < az; ++z)
            for (int y = 0; y < ay; ++y)
                for (int x = 0; x < ax; ++x) {
                    if ((x + y + z) % 2 != parity) continue;
                    size_t ic = I3(x, y, z, ax, ay);
                    if (SD[3][ic] >= 1) continue;
#define A_(X, Y, Z) (((X) < 0 || (Y) < 0 || (Z) < 0 || (X) >= ax || (Y) >= ay || (Z) >= az) ? oobA : SD[3][I3(X, Y, Z, ax, ay)])
#define P_(X, Y, Z) (((X) < 0 || (Y) < 0 || (Z) < 0 || (X) >= ax || (Y) >= ay || (Z) >= az) ? (real)0 : P[I3(X, Y, Z, ax, ay)])
                    real f_top = (real)1 - A_(x, y + 1, z), f_bottom = (real)1 - A_(x, y - 1, z);
                    real f_right = (real)1 - A_(x + 1, y, z), f_left = (real)1 - A_(x - 1, y, z);
                    real f_front = d3 ? (real)1 - A_(x, y, z + 1) : 0, f_back = d3 ? (real)1 - A_(x, y, z - 1) : 0;
                    real f_sum = f_top + f_bottom + f_right + f_left;
                    if (d3) f_sum = f_sum + f_front + f_back;
                    if (f_sum == 0) continue;
                    real delta_v = L == 0 ? delta_v0(s, x, y, z, (int)oobA) : R[ic];
                    real p_sum = P_(x, y + 1, z) * f_top + P_(x, y - 1, z) * f_bottom;
                    p_sum = p_sum + P_(x + 1, y, z) * f_right;
                    p_sum = p_sum + P_(x - 1, y, z) * f_left;
                    if (d3) {
                        p_sum = p_sum + P_(x, y, z + 1) * f_front;
                        p_sum = p_sum + P_(x, y, z - 1) * f_back;
                    }
                    real p;
                    if (L == 0) p = (p_sum - rho * h * delta_v / dt) / f_sum;
                    else p = (p_sum - delta_v * (h * h)) / f_sum;
                    P[ic] = L > 0 ? cstore(s, p) : p;
#undef A_
#undef P_
                }
        parity = 1 - parity;
    }
}

/* compute_residual (shaders3d/compute/pressure_solve/compute_residual.comp:77-130;
 * 2D :72-117): written in place over r[L]; out of grid = solid. */
void og_compute_residual_mode(og_sim* s, int L, real dt, real rho, int quirks);
void og_compute_residual(og_sim* s, int L, real dt, real rho) { og_compute_residual_mode(s, L, dt, rho, 1); }
void og_compute_residual_mode(og_sim* s, int L, real dt, real rho, int quirks) {
    const real oobA = (real)resid_oob_solid(s, quirks);
    const int ax = s->ls[L][0], ay = s->ls[L][1], az = s->ls[L][2];
    const real* P = s->p[L];
    real* R = s->r[L];
    real* const* SD = s->solid[L];
    const real h = hL(s, L);
    const int d3 = s->dim == 3;
    OMP_FOR
    for (int z = 0; z < az; ++z)
        for (int y = 0; y < ay; ++y)
            for (int x = 0; x < ax; ++x) {
                size_t ic = I3(x, y, z, ax, ay);
                if (SD[3][ic] >= 1) { R[ic] = 0; continue; }
#define A_(X, Y, Z) (((X) < 0 || (Y) < 0 || (Z) < 0 || (X) >= ax || (Y) >= ay || (Z) >= az) ? oobA : SD[3][I3(X, Y, Z, ax, ay)])
#define P_(X, Y, Z) (((X) < 0 || (Y) < 0 || (Z) < 0 || (X) >= ax || (Y) >= ay || (Z) >= az) ? (real)0 : P[I3(X, Y, Z, ax, ay)])
                real f_top = (real)1 - A_(x, y + 1, z), f_bottom = (real)1 - A_(x, y - 1, z);
                real f_right = (real)1 - A_(x + 1, y, z), f_left = (real)1 - A_(x - 1, y, z);
                real f_front = d3 ? (real)1 - A_(x, y, z + 1) : 0, f_back = d3 ? (real)1 - A_(x, y, z - 1) : 0;
                real p_sum = P_(x, y + 1, z) * f_top + P_(x, y - 1, z) * f_bottom;
                p_sum = p_sum + P_(x + 1, y, z) * f_right;
                p_sum = p_sum + P_(x - 1, y, z) * f_left;
                real f_sum = f_top + f_bottom + f_right + f_left;
                if (d3) {
                    p_sum = p_sum + P_(x, y, z + 1) * f_front;
                    p_sum = p_sum + P_(x, y, z - 1) * f_back;
                    f_sum = f_sum + f_front + f_back;
                }
                real old_residual = R[ic];
                if (L == 0) {
                    real delta_v = delta_v0(s, x, y, z, (int)oobA);
                    old_residual = rho * delta_v / (dt * h);
                }
                R[ic] = old_residual - (p_sum - f_sum * P[ic]) / (h * h);
#undef A_
#undef P_
            }
}

/* restrict_residual + restrict_solid (pressure_solve/restrict_residual.comp:40-64,
 * restrict_solid.comp:53-78; 2D :40-59, :53-73). */
void og_compute_restrict(og_sim* s, int L) {
    const int fx = s->ls[L][0], fy = s->ls[L][1];
    const int ax = s->ls[L + 1][0], ay = s->ls[L + 1][1], az = s->ls[L + 1][2];
    const real* R = s->r[L];
    real* RC = s->r[L + 1];
    const int d3 = s->dim == 3;
    OMP_FOR
    for (int z = 0; z < az; ++z)
        for (int y = 0; y < ay; ++y)
            for (int x = 0; x < ax; ++x) {
                int X = 2 * x, Y = 2 * y, Z = 2 * z;
                size_t o = I3(x, y, z, ax, ay);
                if (d3) {
                    real bottom = R[I3(X, Y, Z, fx, fy)] + R[I3(X, Y, Z + 1, fx, fy)] + R[I3(X + 1, Y, Z, fx, fy)] + R[I3(X + 1, Y, Z + 1, fx, fy)];
                    real top = R[I3(X, Y + 1, Z, fx, fy)] + R[I3(X, Y + 1, Z + 1, fx, fy)] + R[I3(X + 1, Y + 1, Z, fx, fy)] + R[I3(X + 1, Y + 1, Z + 1, fx, fy)];
                    RC[o] = cstore(s, (bottom + top) / (real)8);
                    for (int c = 0; c < 4; ++c) {
                        const real* S = s->solid[L][c];
                        real b = S[I3(X, Y, Z, fx, fy)] + S[I3(X, Y, Z + 1, fx, fy)] + S[I3(X + 1, Y, Z, fx, fy)] + S[I3(X + 1, Y, Z + 1, fx, fy)];
                        real t = S[I3(X, Y + 1, Z, fx, fy)] + S[I3(X, Y + 1, Z + 1, fx, fy)] + S[I3(X + 1, Y + 1, Z, fx, fy)] + S[I3(X + 1, Y + 1, Z + 1, fx, fy)];
                        s->solid[L + 1][c][o] = (b + t) / (real)8;
                    }
                } else {
                    real sum = R[I3(X, Y, 0, fx, fy)] + R[I3(X + 1, Y, 0, fx, fy)] + R[I3(X, Y + 1, 0, fx, fy)] + R[I3(X + 1, Y + 1, 0, fx, fy)];
                    RC[o] = cstore(s, sum / (real)4);
                    for (int c = 0; c < 4; ++c) {
                        const real* S = s->solid[L][c];
                        real sm = S[I3(X, Y, 0, fx, fy)] + S[I3(X + 1, Y, 0, fx, fy)] + S[I3(X, Y + 1, 0, fx, fy)] + S[I3(X + 1, Y + 1, 0, fx, fy)];
                        s->solid[L + 1][c][o] = sm / (real)4;
                    }
                }
                real keep = s->solid[L + 1][3][o] >= (real)0.5 ? (real)1 : (real)0;
                for (int c = 0; c < 4; ++c) s->solid[L + 1][c][o] = f16(s->solid[L + 1][c][o] * keep);
            }
}

/* prolong_pressure (pressure_solve/prolong_pressure.comp:39-51): p_L += trilinear
 * (clamp to edge) of p_{L+1} at the fine cell centres, on every cell. */
void og_prolong_and_add(og_sim* s, int L) {
    const int ax = s->ls[L][0], ay = s->ls[L][1], az = s->ls[L][2];
    int next = L + 1 < s->levels ? L + 1 : s->levels - 1;
    const int cx = s->ls[next][0], cy = s->ls[next][1], cz = s->ls[next][2];
    real* P = s->p[L];
    const real* PC = s->p[next];
    const real hf = (real)0.5;
    OMP_FOR
    for (int z = 0; z < az; ++z)
        for (int y = 0; y < ay; ++y)
            for (int x = 0; x < ax; ++x) {
                real tx = (((real)x + hf) / (real)ax) * (real)cx - hf;
                real ty = (((real)y + hf) / (real)ay) * (real)cy - hf;
                real tz = (((real)z + hf) / (real)az) * (real)cz - hf;
                size_t i = I3(x, y, z, ax, ay);
                P[i] = L > 0 ? cstore(s, P[i] + sample_edge(PC, s->dim, cx, cy, cz, tx, ty, tz))
                             : P[i] + sample_edge(PC, s->dim, cx, cy, cz, tx, ty, tz);
            }
}

/* v_cycle (common/physics/grid.c:177-209).  With ref_quirks == 0 the level's
 * right-hand side is kept aside so the post-smoother solves the same system
 * as the pre-smoother, and both operators use one out-of-grid rule. */
/* The mixed solve's coarsest level (levels >= 2, at most 1024 cells) is not
 * swept: its n_coarse red-black iterations from p = 0 are a linear map of the
 * right-hand side, applied as a matrix (k_mg.cu k_bottom / coarse_product).
 * The matrix is the iterations' response to unit right-hand sides in FP32
 * without the coarse-storage rounding, rebuilt when the level's solid
 * fractions or the iteration count change; p_j = cstore(sum_i cm[i n + j] r_i)
 * in the summation order of the CUDA product. */
static int og_coarse_matrix_applies(const og_sim* s, int L) {
    const size_t n = (size_t)s->ls[L][0] * s->ls[L][1] * s->ls[L][2];
    return !s->cm_off && s->cround != 0 && L >= 1 && L == s->levels - 1 && n <= 1024;
}

void og_set_coarse_matrix(og_sim* s, int on) { s->cm_off = on ? 0 : 1; }

static void og_coarse_matrix(og_sim* s, int L, const ss_mg_schedule* mg, real dt, real rho) {
    const size_t n = (size_t)s->ls[L][0] * s->ls[L][1] * s->ls[L][2];
    const real* A = s->solid[L][3];
    real* P = s->p[L];
    real* R = s->r[L];
    if (!s->cm || s->cm_n != n || s->cm_iters != mg->n_coarse || memcmp(s->cm_alpha, A, n * sizeof(real)) != 0) {
        free(s->cm);
        free(s->cm_alpha);
        s->cm = (real*)malloc(n * n * sizeof(real));
        s->cm_alpha = (real*)malloc(n * sizeof(real));
        real* keep_r = (real*)malloc(n * sizeof(real));
        memcpy(keep_r, R, n * sizeof(real));
        const int cr = s->cround;
        s->cround = 0;
        for (size_t i = 0; i < n; ++i) {
            memset(P, 0, n * sizeof(real));
            memset(R, 0, n * sizeof(real));
            R[i] = (real)1;
            og_smooth_mode(s, L, mg->n_coarse, dt, rho, mg->ref_quirks);
            memcpy(s->cm + i * n, P, n * sizeof(real));
        }
        s->cround = cr;
        memcpy(R, keep_r, n * sizeof(real));
        free(keep_r);
        memcpy(s->cm_alpha, A, n * sizeof(real));
        s->cm_n = n;
        s->cm_iters = mg->n_coarse;
    }
    /* `parts` slices of i per value (the largest power of two <= 32 with
     * parts * n <= 16384, the lanes of the GPU's 16-block cluster), each with
     * eight round-robin partial sums added pairwise, the slices folded as a
     * tree: v[q] += v[q + o], o = parts/2 .. 1 */
    size_t parts = 1;
    while (parts < 32 && parts * 2 * n <= 16384) parts *= 2;
    const size_t chunk = (n + parts - 1) / parts;
    for (size_t j = 0; j < n; ++j) {
        real v[32];
        for (size_t q = 0; q < parts; ++q) {
            real a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            const size_t i0 = q * chunk, i1 = i0 + chunk < n ? i0 + chunk : n;
            for (size_t i = i0; i < i1; ++i) a[(i - i0) & 7] = a[(i - i0) & 7] + s->cm[i * n + j] * R[i];
            v[q] = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
        }
        for (size_t o = parts / 2; o >= 1; o /= 2)
            for (size_t q = 0; q < o; ++q) v[q] = v[q] + v[q + o];
        P[j] = cstore(s, v[0]);
    }
}

void og_v_cycle(og_sim* s, int L, const ss_mg_schedule* mg, real dt, real rho) {
    const int q = mg->ref_quirks;
    if (L == s->levels - 1) {
        if (og_coarse_matrix_applies(s, L)) og_coarse_matrix(s, L, mg, dt, rho);
        else og_smooth_mode(s, L, mg->n_coarse, dt, rho, q);
        return;
    }
    og_smooth_mode(s, L, mg->n_pre, dt, rho, q);
    size_t n = (size_t)s->ls[L][0] * s->ls[L][1] * s->ls[L][2];
    real* keep = NULL;
    if (!mg->ref_quirks && L > 0) {
        keep = (real*)malloc(sizeof(real) * n);
        memcpy(keep, s->r[L], sizeof(real) * n);
    }
    og_compute_residual_mode(s, L, dt, rho, q);
    og_compute_restrict(s, L);
    size_t nc = (size_t)s->ls[L + 1][0] * s->ls[L + 1][1] * s->ls[L + 1][2];
    memset(s->p[L + 1], 0, sizeof(real) * nc);
    og_v_cycle(s, L + 1, mg, dt, rho);
    if (keep) { memcpy(s->r[L], keep, sizeof(real) * n); free(keep); }
    og_prolong_and_add(s, L);
    og_smooth_mode(s, L, mg->n_post, dt, rho, q);
}

/* ||div||_2 over fluid cells (smoother semantics), FP64 accumulation. */
double og_divergence_norm(og_sim* s) {
    double acc = 0;
#pragma omp parallel for collapse(2) reduction(+ : acc) schedule(static)
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                if (alpha0(s, x, y, z) >= 1) continue;
                double d = (double)delta_v0(s, x, y, z, 0);
                acc += d * d;
            }
    return sqrt(acc);
}

/* FP64 evaluation of the divergence left after projecting with the current p:
 * R = div - (dt/(rho h)) * (sum_f p_nb - f_sum p), smoother boundary rules. */
double og_projected_residual_norm(og_sim* s, real dt, real rho) {
    const double k = (double)dt / ((double)rho * (double)s->h);
    const real* P = s->p[0];
    const int d3 = s->dim == 3;
    double acc = 0;
#pragma omp parallel for collapse(2) reduction(+ : acc) schedule(static)
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                if (alpha0(s, x, y, z) >= 1) continue;
                const int off[6][3] = {{0, 1, 0}, {0, -1, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 0, 1}, {0, 0, -1}};
                double psum = 0, fsum = 0;
                for (int q = 0; q < (d3 ? 6 : 4); ++q) {
                    int X = x + off[q][0], Y = y + off[q][1], Z = z + off[q][2];
                    int oob = X < 0 || Y < 0 || Z < 0 || X >= NX || Y >= NY || Z >= NZ;
                    double f = oob ? 1.0 : 1.0 - (double)alpha0(s, X, Y, Z);
                    double pn = oob ? 0.0 : (double)P[I3(X, Y, Z, NX, NY)];
                    psum += f * pn;
                    fsum += f;
                }
                double r = (double)delta_v0(s, x, y, z, 0) - k * (psum - fsum * (double)P[I3(x, y, z, NX, NY)]);
                acc += r * r;
            }
    return sqrt(acc);
}

/* ------------------------------------------- mixed-precision projection
 * Extension (no counterpart in the reference).  Iterative refinement of an
 * FP64 level-0 pressure: the FP64 residual of the projection
 *   rho_i = div_i - k (sum_{fluid nb} p_j - n_i p_i),  k = dt/(rho h),
 * is the right-hand side of one correction V-cycle (level 0 in `real`,
 * coarse levels rounded to FP16/BF16 on every store, the restricted residual
 * scaled by a power of two first), and the correction is added in FP64.
 * Level-0 operators use the corrected out-of-grid rule (solid if enclosed). */
static inline int fluid0(const og_sim* s, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ) return !s->enclosed;
    return alpha0(s, x, y, z) < 1;
}
static inline int ingrid(const og_sim* s, int x, int y, int z) {
    return !(x < 0 || y < 0 || z < 0 || x >= NX || y >= NY || z >= NZ);
}
static const int OFF6[6][3] = {{0, 1, 0}, {0, -1, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 0, 1}, {0, 0, -1}};

/* red-black sweeps on e with the level-0 right-hand side rhs_s */
static void mx_smooth0(og_sim* s, real* e, const real* rhs_s, int iterations) {
    const int nn = s->dim == 3 ? 6 : 4;
    for (int it = 0; it < 2 * iterations; ++it) {
        const int parity = it & 1;
        OMP_FOR
        for (int z = 0; z < NZ; ++z)
            for (int y = 0; y < NY; ++y)
                for (int x = 0; x < NX; ++x) {
                    if (((x + y + z) & 1) != parity || !fluid0(s, x, y, z)) continue;
                    real sum = 0;
                    int fs = 0;
                    for (int q = 0; q < nn; ++q) {
                        int X = x + OFF6[q][0], Y = y + OFF6[q][1], Z = z + OFF6[q][2];
                        if (!fluid0(s, X, Y, Z)) continue;
                        ++fs;
                        real v = ingrid(s, X, Y, Z) ? e[I3(X, Y, Z, NX, NY)] : (real)0;
                        sum = q == 0 ? v : sum + v;
                    }
                    if (fs == 0) continue;
                    e[I3(x, y, z, NX, NY)] = (sum - rhs_s[I3(x, y, z, NX, NY)]) / (real)fs;
                }
    }
}

/* residual of the correction equation at level 0, restricted into r[1]
 * (scaled, rounded to the coarse storage) */
static void mx_residual_restrict0(og_sim* s, const real* e, const real* rhs_r, real scale) {
    const int nn = s->dim == 3 ? 6 : 4;
    const real hh = hL(s, 0) * hL(s, 0);
    const int cx = s->ls[1][0], cy = s->ls[1][1], cz = s->ls[1][2];
    real* RC = s->r[1];
    OMP_FOR
    for (int Z = 0; Z < cz; ++Z)
        for (int Y = 0; Y < cy; ++Y)
            for (int X = 0; X < cx; ++X) {
                real v[2][2][2];
                for (int dz = 0; dz < (s->dim == 3 ? 2 : 1); ++dz)
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx) {
                            int x = 2 * X + dx, y = 2 * Y + dy, z = s->dim == 3 ? 2 * Z + dz : 0;
                            real res = 0;
                            if (fluid0(s, x, y, z)) {
                                real sum = 0;
                                int fs = 0;
                                for (int q = 0; q < nn; ++q) {
                                    int XX = x + OFF6[q][0], YY = y + OFF6[q][1], ZZ = z + OFF6[q][2];
                                    real w = 0;
                                    if (fluid0(s, XX, YY, ZZ)) {
                                        ++fs;
                                        if (ingrid(s, XX, YY, ZZ)) w = e[I3(XX, YY, ZZ, NX, NY)];
                                    }
                                    sum = q == 0 ? w : sum + w;
                                }
                                const size_t c = I3(x, y, z, NX, NY);
                                real lap = sum - (real)fs * e[c];
                                res = rhs_r[c] - lap / hh;
                            }
                            v[dz][dy][dx] = res;
                        }
                real out;
                if (s->dim == 3) {
                    real bottom = v[0][0][0] + v[1][0][0] + v[0][0][1] + v[1][0][1];
                    real top = v[0][1][0] + v[1][1][0] + v[0][1][1] + v[1][1][1];
                    out = (bottom + top) / (real)8;
                } else {
                    out = (v[0][0][0] + v[0][0][1] + v[0][1][0] + v[0][1][1]) / (real)4;
                }
                RC[I3(X, Y, Z, cx, cy)] = cstore(s, out * scale);
            }
}

/* e += (trilinear of p[1]) / scale on every level-0 cell */
static void mx_prolong0(og_sim* s, real* e, real inv_scale) {
    const int cx = s->ls[1][0], cy = s->ls[1][1], cz = s->ls[1][2];
    const real* PC = s->p[1];
    const real hf = (real)0.5;
    OMP_FOR
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                real tx = (((real)x + hf) / (real)NX) * (real)cx - hf;
                real ty = (((real)y + hf) / (real)NY) * (real)cy - hf;
                real tz = (((real)z + hf) / (real)NZ) * (real)cz - hf;
                size_t i = I3(x, y, z, NX, NY);
                real sv = sample_edge(PC, s->dim, cx, cy, cz, tx, ty, tz) * inv_scale;
                e[i] = e[i] + sv;
            }
}

/* FP64 residual of the projection; right-hand sides of the correction
 * equation; returns sum of squares and stores max|rho| */
static double mx_ir_residual(og_sim* s, real dt, real rho, real* rhs_s, real* rhs_r, double* amax_out) {
    const int nn = s->dim == 3 ? 6 : 4;
    const double k = (double)dt / ((double)rho * (double)s->h);
    const double inv_k = 1.0 / k;
    const real hh = hL(s, 0) * hL(s, 0);
    const double inv_khh = 1.0 / (k * (double)hh);
    double acc = 0, amax = 0;
#pragma omp parallel for collapse(2) reduction(+ : acc) reduction(max : amax) schedule(static)
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                const size_t c = I3(x, y, z, NX, NY);
                rhs_s[c] = 0;
                rhs_r[c] = 0;
                if (!fluid0(s, x, y, z)) continue;
                double sum = 0;
                int cnt = 0;
                for (int q = 0; q < nn; ++q) {
                    int X = x + OFF6[q][0], Y = y + OFF6[q][1], Z = z + OFF6[q][2];
                    double w = 0;
                    if (fluid0(s, X, Y, Z)) {
                        ++cnt;
                        if (ingrid(s, X, Y, Z)) w = s->p64[I3(X, Y, Z, NX, NY)];
                    }
                    sum = q == 0 ? w : sum + w;
                }
                const double d = (double)delta_v0(s, x, y, z, 0);
                const double r = d - k * (sum - (double)cnt * s->p64[c]);
                acc += r * r;
                if (fabs(r) > amax) amax = fabs(r);
                rhs_s[c] = (real)(r * inv_k);
                rhs_r[c] = (real)(r * inv_khh);
            }
    *amax_out = amax * inv_khh;
    return acc;
}

static int og_mixed_pressure_solve(og_sim* s, const ss_mg_schedule* mg, real dt, real rho) {
    if (s->levels < 2 || NX % 2 != 0 || mg->ref_quirks) return 0;
    ss_mg_schedule m2 = *mg;
    m2.ref_quirks = 0;
    if (!s->p64) s->p64 = (double*)calloc(s->ncell, sizeof(double));
    int fresh = 0;
    if (!s->p64_valid) {
        for (size_t i = 0; i < s->ncell; ++i) s->p64[i] = (double)s->p[0][i];
        s->p64_valid = 1;
        fresh = 1;
    }
    /* warm start: with warm_start 1 and the previous solve's starting (solved)
     * pressure p(n-2) kept, start from 2 p(n-1) - p(n-2); keep p(n-1) either
     * way.  A fresh p64, not solved by this path, starts no history. */
    if (mg->warm_start == 1 && !fresh) {
        if (!s->p64_prev) s->p64_prev = (double*)calloc(s->ncell, sizeof(double));
        if (s->prev_ok) {
            for (size_t i = 0; i < s->ncell; ++i) {
                const double a = s->p64[i], c = s->p64_prev[i];
                s->p64[i] = 2.0 * a - c;
                s->p64_prev[i] = a;
            }
        } else {
            memcpy(s->p64_prev, s->p64, s->ncell * sizeof(double));
            s->prev_ok = 1;
        }
    } else {
        s->prev_ok = 0;
    }
    real* e = (real*)malloc(sizeof(real) * s->ncell);
    real* rhs_s = (real*)malloc(sizeof(real) * s->ncell);
    real* rhs_r = (real*)malloc(sizeof(real) * s->ncell);
    const double db = og_divergence_norm(s);
    const int tol_mode = mg->tol > 0;
    const int cap = mg->n_vcycles > 0 ? mg->n_vcycles : 1;
    int done = 0, conv = 1;
    double res = 0;
    for (;;) {
        double amax = 0;
        res = sqrt(mx_ir_residual(s, dt, rho, rhs_s, rhs_r, &amax));
        if (!tol_mode && done == cap) break;
        if (tol_mode && res <= mg->tol * db) break;
        if (done == cap) { conv = 0; break; }
        int ex = 0;
        frexp(amax, &ex);
        ex = ex < -100 ? -100 : ex > 100 ? 100 : ex;
        const real scale = (real)(float)ldexp(1.0, -ex), inv_scale = (real)(float)ldexp(1.0, ex);
        memset(e, 0, sizeof(real) * s->ncell);
        /* one V-cycle on e */
        s->cround = mg->precision;
        mx_smooth0(s, e, rhs_s, m2.n_pre);
        og_compute_restrict(s, 0);          /* coarse solid pyramid (r[1] overwritten next) */
        mx_residual_restrict0(s, e, rhs_r, scale);
        memset(s->p[1], 0, sizeof(real) * (size_t)s->ls[1][0] * s->ls[1][1] * s->ls[1][2]);
        og_v_cycle(s, 1, &m2, dt, rho);
        mx_prolong0(s, e, inv_scale);
        mx_smooth0(s, e, rhs_s, m2.n_post);
        s->cround = 0;
        for (size_t c = 0; c < s->ncell; ++c)
            if (alpha0(s, (int)(c % NX), (int)((c / NX) % NY), (int)(c / ((size_t)NX * NY))) < 1) s->p64[c] += (double)e[c];
        ++done;
    }
    for (size_t i = 0; i < s->ncell; ++i) s->p[0][i] = (real)s->p64[i];
    free(e); free(rhs_s); free(rhs_r);
    s->st.div_before = db;
    s->st.residual = res;
    s->st.vcycles = done;
    s->st.converged = conv;
    return conv;
}

/* multigrid_pressure_solve (common/physics/grid.c:173-175): n_vcycles V-cycles,
 * or (tol > 0) V-cycles until the projected residual <= tol * div_before. */
int og_multigrid_pressure_solve(og_sim* s, const ss_mg_schedule* mg, real dt, real rho) {
    if (mg->precision != SS_PREC_FP32) return og_mixed_pressure_solve(s, mg, dt, rho);
    s->p64_valid = 0;
    double db = og_divergence_norm(s);
    s->st.div_before = db;
    int ncyc = mg->n_vcycles > 0 ? mg->n_vcycles : 1;
    int done = 0, conv = 0;
    if (mg->tol > 0) {
        double res = og_projected_residual_norm(s, dt, rho);
        while (done < ncyc && !(res <= mg->tol * db)) {
            og_v_cycle(s, 0, mg, dt, rho);
            ++done;
            res = og_projected_residual_norm(s, dt, rho);
        }
        conv = res <= mg->tol * db;
        s->st.residual = res;
    } else {
        for (; done < ncyc; ++done) og_v_cycle(s, 0, mg, dt, rho);
        s->st.residual = og_projected_residual_norm(s, dt, rho);
        conv = 1;
    }
    s->st.vcycles = done;
    s->st.converged = conv;
    return conv;
}

/* update_vx/vy/vz (shaders3d/compute/update_vx.comp:45-62 and siblings; 2D :43-60). */
static void update_velocities_impl(og_sim* s, real dt, real rho, int use_p64) {
    const real k = -dt / (rho * s->h);
    const double k64 = -(double)dt / ((double)rho * (double)s->h);
    const real* P = s->p[0];
    const double* P64 = use_p64 ? s->p64 : NULL;
    for (int comp = 0; comp < s->dim; ++comp) {
        int ax = NX + (comp == 0), ay = NY + (comp == 1), az = NZ + (comp == 2);
        const real* src = comp == 0 ? CUR_VX : comp == 1 ? CUR_VY : CUR_VZ;
        real* dst = comp == 0 ? OTH_VX : comp == 1 ? OTH_VY : OTH_VZ;
        OMP_FOR
        for (int z = 0; z < az; ++z)
            for (int y = 0; y < ay; ++y)
                for (int x = 0; x < ax; ++x) {
                    int xm = x - (comp == 0), ym = y - (comp == 1), zm = z - (comp == 2);
                    size_t i = I3(x, y, z, ax, ay);
                    if (solid_oob0(s, x, y, z) || solid_oob0(s, xm, ym, zm)) {
                        int oob = x >= NX || y >= NY || z >= NZ;
                        dst[i] = oob ? 0 : s->solid[0][comp][I3(x, y, z, NX, NY)];
                        continue;
                    }
                    if (P64) {
                        double q_hi = (x >= NX || y >= NY || z >= NZ) ? 0 : P64[I3(x, y, z, NX, NY)];
                        double q_lo = (xm < 0 || ym < 0 || zm < 0) ? 0 : P64[I3(xm, ym, zm, NX, NY)];
                        dst[i] = (real)((double)src[i] + k64 * (q_hi - q_lo));
                        continue;
                    }
                    real p_hi = (x >= NX || y >= NY || z >= NZ) ? 0 : P[I3(x, y, z, NX, NY)];
                    real p_lo = (xm < 0 || ym < 0 || zm < 0) ? 0 : P[I3(xm, ym, zm, NX, NY)];
                    dst[i] = src[i] + k * (p_hi - p_lo);
                }
    }
    s->vxi ^= 1; s->vyi ^= 1; if (s->dim == 3) s->vzi ^= 1;
}

/* -------------------------------------------------------------- renderer
 * Restatement of the reference's smoke fragment shaders for the headless
 * image the CUDA renderer writes: shaders3d/graphics/ray_march_smoke.frag:
 * 80-175 (AABB entry/exit, per-pixel sine-hash jitter, front-to-back
 * compositing, shadow march, Henyey-Greenstein phase with the shader's
 * PI = 3.14 and factor 3) and shaders2d/graphics/draw_smoke.frag:43-58.
 * Pinhole camera in box space [0, n/min(n)]; no scene depth buffer;
 * single-channel density is grey (r = g = b). */
static void rn_normalize(float v[3]) {
    float l = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int k = 0; k < 3; ++k) v[k] = v[k] / l;
}
static void rn_cross(const float a[3], const float b[3], float o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static unsigned char rn_unorm8(float v) {
    v = fminf(fmaxf(v, 0.f), 1.f);
    return (unsigned char)(v * 255.f + 0.5f);
}
static void rn_rgb(const og_sim* s, const float box[3], float px, float py, float pz, float rgb[3]) {
    const real* const* sm = (const real* const*)s->smoke[s->si];
    float tx = (px / box[0]) * (float)NX - 0.5f;
    float ty = (py / box[1]) * (float)NY - 0.5f;
    float tz = (pz / box[2]) * (float)NZ - 0.5f;
    rgb[0] = (float)sample_border(sm[0], 3, NX, NY, NZ, tx, ty, tz, 0);
    if (s->nch == 3) {
        rgb[1] = (float)sample_border(sm[1], 3, NX, NY, NZ, tx, ty, tz, 0);
        rgb[2] = (float)sample_border(sm[2], 3, NX, NY, NZ, tx, ty, tz, 0);
    } else {
        rgb[1] = rgb[0];
        rgb[2] = rgb[0];
    }
}

void og_render(const og_sim* s, const ss_render_desc* d, unsigned char* rgba) {
    const int W = d->width, H = d->height;
    int mn = NX < NY ? NX : NY;
    if (s->dim == 3 && NZ < mn) mn = NZ;
    const float m = (float)mn;
    const float box[3] = {(float)NX / m, (float)NY / m, s->dim == 3 ? (float)NZ / m : 1.f};
    float fwd[3], right[3], up[3], light[3];
    for (int k = 0; k < 3; ++k) { fwd[k] = d->camera_target[k] - d->camera_pos[k]; light[k] = d->light_direction[k]; }
    rn_normalize(fwd);
    rn_cross(fwd, d->camera_up, right);
    rn_normalize(right);
    rn_cross(right, fwd, up);
    rn_normalize(light);
    const float tan_half = tanf(0.5f * d->fov_y), aspect = (float)W / (float)H;
    const float step = d->step_size, shadow_step = d->step_size * d->shadow_step_factor;
#pragma omp parallel for schedule(dynamic, 4)
    for (int row = 0; row < H; ++row)
        for (int px = 0; px < W; ++px) {
            unsigned char* out = rgba + 4 * ((size_t)row * W + px);
            const int py = H - 1 - row;
            const float u = ((float)px + 0.5f) / (float)W, v = ((float)py + 0.5f) / (float)H;
            if (s->dim == 2) {
                const real* const* sm = (const real* const*)s->smoke[s->si];
                float tx = u * (float)NX - 0.5f, ty = v * (float)NY - 0.5f;
                float rgb[3];
                rgb[0] = (float)sample_border(sm[0], 2, NX, NY, 1, tx, ty, 0, 0);
                if (s->nch == 3) {
                    rgb[1] = (float)sample_border(sm[1], 2, NX, NY, 1, tx, ty, 0, 0);
                    rgb[2] = (float)sample_border(sm[2], 2, NX, NY, 1, tx, ty, 0, 0);
                } else {
                    rgb[1] = rgb[0];
                    rgb[2] = rgb[0];
                }
                const float raw = fmaxf(rgb[0], fmaxf(rgb[1], rgb[2]));
                const float alpha = 1.f - expf(-raw * d->smoke_density_factor);
                for (int k = 0; k < 3; ++k) {
                    const float sc = raw > 0.001f ? rgb[k] / raw : 0.f;
                    out[k] = rn_unorm8(d->ambient_color[k] * (1.f - alpha) + sc * alpha);
                }
                out[3] = 255;
                continue;
            }
            const float ndx = 2.f * u - 1.f, ndy = 2.f * v - 1.f;
            const float sx = ndx * tan_half * aspect, sy = ndy * tan_half;
            float dv[3], dir[3];
            for (int k = 0; k < 3; ++k) dv[k] = fwd[k] + right[k] * sx + up[k] * sy;
            const float dl = sqrtf(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            for (int k = 0; k < 3; ++k) dir[k] = dv[k] / dl;
            float enter = -INFINITY, exit_ = INFINITY;
            for (int k = 0; k < 3; ++k) {
                const float inv = 1.f / dir[k];
                const float t0 = (0.f - d->camera_pos[k]) * inv, t1 = (box[k] - d->camera_pos[k]) * inv;
                enter = fmaxf(enter, fminf(t0, t1));
                exit_ = fminf(exit_, fmaxf(t0, t1));
            }
            if (exit_ < fmaxf(enter, 0.f)) {
                out[0] = out[1] = out[2] = out[3] = 0;
                continue;
            }
            const int steps = (int)((exit_ - enter) / step) + 1;
            const float sn = sinf(u * 12.9898f + v * 78.233f) * 43758.5453f;
            const float noise = sn - floorf(sn);
            float t = enter + noise * step;
            const float cos_t = (-dir[0]) * light[0] + (-dir[1]) * light[1] + (-dir[2]) * light[2];
            const float g = d->phase_g;
            float phase;
            if (g == 0.f) {
                phase = 1.f / 3.14f;
            } else {
                const float den = 1.f + g * g - 2.f * g * cos_t;
                phase = 1.f / (4.f * 3.14f) * (1.f - g * g) / (den * sqrtf(den));
            }
            phase = phase * 3.f;
            float T = 1.f, col[3] = {0.f, 0.f, 0.f};
            for (int i = 0; i < steps; ++i) {
                if (t > exit_) break;
                const float pos[3] = {d->camera_pos[0] + dir[0] * t, d->camera_pos[1] + dir[1] * t, d->camera_pos[2] + dir[2] * t};
                float rgb[3];
                rn_rgb(s, box, pos[0], pos[1], pos[2], rgb);
                const float total = rgb[0] + rgb[1] + rgb[2];
                if (total > 0.001f) {
                    float ld = 0.f, lp[3] = {pos[0], pos[1], pos[2]};
                    for (int j = 0; j < d->shadow_steps; ++j) {
                        for (int k = 0; k < 3; ++k) lp[k] = lp[k] + light[k] * shadow_step;
                        float sh[3];
                        rn_rgb(s, box, lp[0], lp[1], lp[2], sh);
                        ld = ld + (sh[0] + sh[1] + sh[2]);
                    }
                    const float atten = expf(-ld * d->shadow_density_factor * shadow_step);
                    const float alpha = 1.f - expf(-total * d->smoke_density_factor * step);
                    const float ta = T * alpha;
                    for (int k = 0; k < 3; ++k) {
                        const float lc = d->ambient_color[k] + (d->light_color[k] * atten) * phase;
                        col[k] = col[k] + ta * ((rgb[k] / total) * lc);
                    }
                    T = T * (1.f - alpha);
                    if (T < 0.001f) break;
                }
                t = t + step;
            }
            out[0] = rn_unorm8(col[0]);
            out[1] = rn_unorm8(col[1]);
            out[2] = rn_unorm8(col[2]);
            out[3] = rn_unorm8(1.f - T);
        }
}

/* ------------------------------------------------------------- the step */
/* run_physics_step (common/physics/physics.c:72-101). */
void og_run_physics_step(og_sim* s, const ss_params* prm) {
    const real dt = prm->time_step, rho = prm->density, tamb = prm->t_ambient;
    const real wind[3] = {prm->wind[0], prm->wind[1], prm->wind[2]};
    const int m = prm->stage_mask;
    if (m & SS_STAGE_HANDLE_EMITTERS) {
        og_update_emitters_status(s, prm->current_time);
        og_handle_emitters(s, dt);
        og_emitter_velocity(s, dt);
        og_apply_force_field(s, dt);
    }
    if (m & SS_STAGE_ADVECT_VELOCITIES) advect_velocities_impl(s, dt, wind);
    if (m & SS_STAGE_APPLY_BUOYANCY) apply_buoyancy_impl(s, dt, tamb, prm->t_weight_coeff, prm->t_temp_coeff);
    if (m & SS_STAGE_APPLY_VORTICITY) {
        calculate_vorticity_impl(s);
        apply_vorticity_impl(s, dt, prm->vorticity_confinement, rho);
    }
    if (m & SS_STAGE_RESOLVE_PRESSURE) og_multigrid_pressure_solve(s, &prm->mg, dt, rho);
    if (m & SS_STAGE_UPDATE_VELOCITIES) {
        update_velocities_impl(s, dt, rho, prm->mg.precision != SS_PREC_FP32 && s->p64_valid);
        if (m & SS_STAGE_RESOLVE_PRESSURE) {
            s->st.div_after = og_divergence_norm(s);
            s->st.rel_div = s->st.div_before > 0 ? s->st.div_after / s->st.div_before : 0;
        }
    }
    if (m & SS_STAGE_ADVECT_SMOKE) advect_smoke_impl(s, dt, tamb);
    if (m & SS_STAGE_OBSTACLES) {
        og_obstacle_update(s, dt);
        og_update_solid_map(s);
    }
    s->st.steps += 1;
}

/* single-stage entry points for the parity tests */
void og_stage_advect_velocities(og_sim* s, const ss_params* p) {
    const real w[3] = {p->wind[0], p->wind[1], p->wind[2]};
    advect_velocities_impl(s, p->time_step, w);
}
void og_stage_apply_buoyancy(og_sim* s, const ss_params* p) {
    apply_buoyancy_impl(s, p->time_step, p->t_ambient, p->t_weight_coeff, p->t_temp_coeff);
}
void og_stage_apply_vorticity(og_sim* s, const ss_params* p) {
    calculate_vorticity_impl(s);
    apply_vorticity_impl(s, p->time_step, p->vorticity_confinement, p->density);
}
void og_stage_update_velocities(og_sim* s, const ss_params* p) {
    update_velocities_impl(s, p->time_step, p->density, p->mg.precision != SS_PREC_FP32 && s->p64_valid);
}
void og_stage_advect_smoke(og_sim* s, const ss_params* p) { advect_smoke_impl(s, p->time_step, p->t_ambient); }
void og_stage_handle_emitters(og_sim* s, const ss_params* p) {
    og_update_emitters_status(s, p->current_time);
    og_handle_emitters(s, p->time_step);
    og_emitter_velocity(s, p->time_step);
    og_apply_force_field(s, p->time_step);
}
void og_stage_multigrid(og_sim* s, const ss_params* p) { og_multigrid_pressure_solve(s, &p->mg, p->time_step, p->density); }
void og_stage_obstacles(og_sim* s, const ss_params* p) { og_obstacle_update(s, p->time_step); og_update_solid_map(s); }
void og_get_stats(const og_sim* s, ss_stats* out) { *out = s->st; }

/* ------------------------------------------------------------- field I/O */
static real* field_ptr(og_sim* s, int f, int ch, size_t* n) {
    switch (f) {
    case SS_FIELD_VX: *n = s->nvx; return CUR_VX;
    case SS_FIELD_VY: *n = s->nvy; return CUR_VY;
    case SS_FIELD_VZ: *n = s->nvz; return s->dim == 3 ? CUR_VZ : NULL;
    case SS_FIELD_DENSITY: *n = s->ncell; return ch < 3 ? s->smoke[s->si][ch] : NULL;
    case SS_FIELD_TEMPERATURE: *n = s->ncell; return s->smoke[s->si][3];
    case SS_FIELD_PRESSURE: *n = s->ncell; return s->p[0];
    case SS_FIELD_SOLID: *n = s->ncell; return s->solid[0][3];
    default: *n = 0; return NULL;
    }
}

/* density is channel-major: channel c occupies [c*ncell, (c+1)*ncell) */
int og_set_field(og_sim* s, int f, const float* src, size_t count) {
    int nch = f == SS_FIELD_DENSITY ? s->nch : 1;
    size_t n;
    if (!field_ptr(s, f, 0, &n) || count != n * nch) return SS_E_INVALID;
    for (int c = 0; c < nch; ++c) {
        real* d = field_ptr(s, f, c, &n);
        for (size_t i = 0; i < n; ++i) d[i] = (real)src[c * n + i];
    }
    /* a new pressure is the mixed solve's next warm start (its FP64 copy and
     * history are dropped), as the GPU path's ss_set_field does */
    if (f == SS_FIELD_PRESSURE) s->p64_valid = 0;
    return 0;
}
int og_set_field_f64(og_sim* s, int f, const double* src, size_t count) {
    int nch = f == SS_FIELD_DENSITY ? s->nch : 1;
    size_t n;
    if (!field_ptr(s, f, 0, &n) || count != n * nch) return SS_E_INVALID;
    for (int c = 0; c < nch; ++c) {
        real* d = field_ptr(s, f, c, &n);
        for (size_t i = 0; i < n; ++i) d[i] = (real)src[c * n + i];
    }
    /* a new pressure is the mixed solve's next warm start (its FP64 copy and
     * history are dropped), as the GPU path's ss_set_field does */
    if (f == SS_FIELD_PRESSURE) s->p64_valid = 0;
    return 0;
}
int og_get_field(og_sim* s, int f, float* dst, size_t count) {
    int nch = f == SS_FIELD_DENSITY ? s->nch : 1;
    size_t n;
    if (!field_ptr(s, f, 0, &n) || count != n * nch) return SS_E_INVALID;
    for (int c = 0; c < nch; ++c) {
        const real* d = field_ptr(s, f, c, &n);
        for (size_t i = 0; i < n; ++i) dst[c * n + i] = (float)d[i];
    }
    return 0;
}
int og_get_field_f64(og_sim* s, int f, double* dst, size_t count) {
    int nch = f == SS_FIELD_DENSITY ? s->nch : 1;
    size_t n;
    if (!field_ptr(s, f, 0, &n) || count != n * nch) return SS_E_INVALID;
    for (int c = 0; c < nch; ++c) {
        const real* d = field_ptr(s, f, c, &n);
        for (size_t i = 0; i < n; ++i) dst[c * n + i] = (double)d[i];
    }
    return 0;
}
/* both ping-pong buffers of the velocities (the stale-buffer quirk reads the other one) */
int og_set_velocity_other(og_sim* s, int comp, const float* src, size_t count) {
    real* d = comp == 0 ? OTH_VX : comp == 1 ? OTH_VY : OTH_VZ;
    size_t n = comp == 0 ? s->nvx : comp == 1 ? s->nvy : s->nvz;
    if (count != n) return SS_E_INVALID;
    for (size_t i = 0; i < n; ++i) d[i] = (real)src[i];
    return 0;
}

/* level arrays: 0 pressure, 1 residual, 2 fluid weight (1 - alpha) */
int og_get_level(og_sim* s, int L, int what, float* dst, size_t count) {
    if (L < 0 || L >= s->levels) return SS_E_INVALID;
    size_t n = (size_t)s->ls[L][0] * s->ls[L][1] * s->ls[L][2];
    if (count != n) return SS_E_INVALID;
    for (size_t i = 0; i < n; ++i) {
        real v = what == 0 ? s->p[L][i] : what == 1 ? s->r[L][i] : (real)1 - s->solid[L][3][i];
        dst[i] = (float)v;
    }
    return 0;
}
int og_set_level(og_sim* s, int L, int what, const float* src, size_t count) {
    if (L < 0 || L >= s->levels || what > 1) return SS_E_INVALID;
    size_t n = (size_t)s->ls[L][0] * s->ls[L][1] * s->ls[L][2];
    if (count != n) return SS_E_INVALID;
    real* d = what == 0 ? s->p[L] : s->r[L];
    for (size_t i = 0; i < n; ++i) d[i] = (real)src[i];
    if (L == 0 && what == 0) s->p64_valid = 0;
    return 0;
}
/* Compute the coarse solid maps of every level (restrict_solid chain), as the
 * first V-cycle would. */
void og_restrict_solid_all(og_sim* s) {
    for (int L = 0; L + 1 < s->levels; ++L) {
        /* restrict only the solid part: save r, restrict, restore */
        size_t nc = (size_t)s->ls[L + 1][0] * s->ls[L + 1][1] * s->ls[L + 1][2];
        real* keep = (real*)malloc(sizeof(real) * nc);
        memcpy(keep, s->r[L + 1], sizeof(real) * nc);
        og_compute_restrict(s, L);
        memcpy(s->r[L + 1], keep, sizeof(real) * nc);
        free(keep);
    }
}

int og_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void og_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
