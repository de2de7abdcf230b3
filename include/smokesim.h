/*
 * smokesim.h - C ABI of the B200 smoke-step library (libsmokesim.so).
 *
 * This library replaces the OpenGL compute dispatches of SmokeSim's per-frame
 * smoke step.  In the reference the step is driven by
 *   run_physics_step(grid*, physics_info*)            common/physics/physics.c:72-101
 * which calls one host function per stage (common/physics/grid.h:37-68), each a
 * glUseProgram + glDispatchCompute over GL textures bound to fixed slots
 * (common/graphics/opengl_bindings.h:8-42) with parameters in std140 UBOs
 * (common/physics/physics.c:142-180).  Here the grid, its MAC velocity arrays,
 * the smoke fields and the multigrid pyramid live in device memory owned by an
 * opaque ss_sim handle; every stage is a hand-written sm_100a CUDA kernel.
 *
 * Conventions
 *  - Every entry point returns SS_OK (0) or a negative SS_E* code; nothing
 *    calls exit().  ss_strerror() names the code, ss_last_error_message()
 *    gives the detail of the last failure on the calling thread.
 *  - The caller owns host buffers, the library owns device buffers.
 *  - `stream` arguments are cudaStream_t passed as void* (NULL = the legacy
 *    default stream).  Calls on one handle are not thread-safe.
 *  - Arrays are x-fastest: index (z*ny + y)*nx + x, with the MAC face arrays
 *    one longer on their own axis (u: (nx+1)*ny*nz, v: nx*(ny+1)*nz,
 *    w: nx*ny*(nz+1)).  A 2D grid has nz = 1 and no w array.
 */
#ifndef SMOKESIM_B200_H
#define SMOKESIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SS_ABI_VERSION 1

typedef struct ss_sim ss_sim;   /* opaque handle; owns all device memory of one grid */
#define SS_MAX_LEVELS 16           /* reference MAX_GRID_SIZE_ARRAY, common/physics/grid.h:17 */
#define SS_MAX_EMITTERS 256
#define SS_MAX_OBSTACLES 4096
#define SS_MAX_BOXES 256

/* ---- status codes ------------------------------------------------------ */
enum ss_status {
    SS_OK = 0,
    SS_E_INVALID = -1,          /* bad argument, size or NULL handle */
    SS_E_CUDA = -2,             /* a CUDA runtime call failed */
    SS_E_OOM = -3,              /* device or host allocation failed */
    SS_E_NOT_CONVERGED = -4,    /* tolerance solve hit its V-cycle cap */
    SS_E_NONFINITE = -5,        /* NaN/Inf found in a host input */
    SS_E_UNSUPPORTED = -6       /* feature not available for this grid */
};

/* ---- grid description (reference grid3d/grid2d + cell_size) ------------ */
typedef struct ss_desc {
    int dim;                /* 2 or 3 (reference grid.is_2d, common/physics/grid.h:20-29) */
    int n[3];               /* cells per axis; n[2] must be 1 when dim == 2 */
    float cell_size;        /* h (reference grid.cell_size) */
    int density_channels;   /* 1 (r only) or 3 (reference RGB smoke.rgb) */
    int enclosed;           /* 1: solid wall shell, reference init_solid_map (common/gui/gui.c:121-123) */
    int min_coarse;         /* smallest multigrid level dimension; reference pyramid stops at 4 (3d/grid3d.c:48) */
    float t_ambient;        /* initial smoke temperature, reference gen_grid_textures(grid, t_ambient) (3d/grid3d.c:35-38) */
} ss_desc;

/* ---- scene objects ------------------------------------------------------ */
/* Emitter: reference `emitter` (common/physics/emitters.h:10-14) holds ivec4
 * pos_radius, ivec4 density_temp and ivec4 emitter_settings {delay, last_emit,
 * emit, falloff}; the same values are carried here as floats/ints.  The
 * velocity fields are an extension: when set_velocity != 0, every MAC face
 * whose index lies inside the sphere gets that velocity in the emitter stage. */
typedef struct ss_emitter {
    float pos[3];
    float radius;
    float density[3];       /* RGB density per second (channel 0 only when density_channels == 1) */
    float temperature;      /* temperature per second */
    int delay;              /* emitter_settings.x */
    int last_emit;          /* emitter_settings.y */
    int emit;               /* emitter_settings.z (state, updated by the status stage) */
    int falloff;            /* emitter_settings.w: smoothstep falloff when > 0 */
    int set_velocity;       /* extension: drive face velocities inside the sphere */
    float velocity[3];
} ss_emitter;

/* Sphere (3D) / disc (2D) obstacle: reference `obstacle`
 * (common/physics/obstacles.h:10-13): vec4 pos_radius, vec4 velocities_anchored. */
typedef struct ss_obstacle {
    float pos[3];
    float radius;
    float velocity[3];
    float anchored;         /* 1 = static; 0 = rigid body moved by the obstacle stage */
} ss_obstacle;

/* Axis-aligned box (extension, not in the reference): cells with
 * lo <= index < hi on every axis become solid, rasterised after the spheres. */
typedef struct ss_box {
    float lo[3];
    float hi[3];
    float velocity[3];
    float anchored;
} ss_box;

/* ---- per-step parameters ------------------------------------------------ */
/* Stage toggles: reference physics_step_settings (common/physics/physics.h:10-18). */
enum ss_stage_bits {
    SS_STAGE_HANDLE_EMITTERS   = 1 << 0,
    SS_STAGE_ADVECT_VELOCITIES = 1 << 1,
    SS_STAGE_APPLY_BUOYANCY    = 1 << 2,
    SS_STAGE_APPLY_VORTICITY   = 1 << 3,
    SS_STAGE_RESOLVE_PRESSURE  = 1 << 4,
    SS_STAGE_UPDATE_VELOCITIES = 1 << 5,
    SS_STAGE_ADVECT_SMOKE      = 1 << 6,
    SS_STAGE_OBSTACLES         = 1 << 7,   /* obstacle_update_step + update_solid_map */
    SS_STAGE_ALL               = 0xff
};

enum ss_precision {
    SS_PREC_FP32 = 0,       /* FP32 V-cycles on the pressure itself */
    SS_PREC_MIXED = 1,      /* FP64 fine residual + refinement, FP32 smoothing, FP16 coarse corrections */
    SS_PREC_MIXED_BF16 = 2  /* the same with BF16 coarse corrections */
};

/* Multigrid schedule.  Reference: 1 V-cycle per frame, 16 pre- and 16
 * post-smoothing red-black sweeps, 80 at the coarsest level
 * (common/physics/grid.c:259-295). */
typedef struct ss_mg_schedule {
    int n_pre;              /* red-black sweeps before restriction */
    int n_post;             /* red-black sweeps after prolongation */
    int n_coarse;           /* sweeps on the coarsest level */
    int n_vcycles;          /* V-cycles per frame (tol == 0) or the cap (tol > 0) */
    double tol;             /* > 0: iterate until relative divergence <= tol (mixed-precision solve on a
                               caller's stream: the first 8 refinement steps run as conditional graph
                               nodes with the test on the device; SMOKESIM_DEVICE_LOOP=0 tests on the host) */
    int ref_quirks;         /* 1: post-smoothing at level > 0 reads the in-place residual (reference) */
    int precision;          /* ss_precision */
    int warm_start;         /* mixed-precision solve: 0 starts from the previous step's pressure (as the
                               reference does); 1 from its linear extrapolation 2 p(n-1) - p(n-2) once two
                               consecutive mixed solves exist (fewer refinement steps; forward runs only:
                               ss_adjoint_forward rejects it) */
} ss_mg_schedule;

/* Physics constants: reference physics_settings (common/physics/physics.h:22-32). */
typedef struct ss_params {
    float time_step;            /* dt */
    float density;              /* rho */
    float t_ambient;
    float t_weight_coeff;       /* alpha in  dt*(-alpha*(r+g+b) + beta*(T - T_amb)) */
    float t_temp_coeff;         /* beta */
    float vorticity_confinement;/* epsilon */
    float wind[3];
    float current_time;         /* emitter clock (reference time UBO, main.c:133-135) */
    int stage_mask;             /* ss_stage_bits */
    int collect_stats;          /* 1: measure div_before / div_after of every solve (two extra reductions) */
    ss_mg_schedule mg;
} ss_params;

/* ---- fields ---------------------------------------------------------------- */
enum ss_field {
    SS_FIELD_VX = 0,            /* (nx+1)*ny*nz floats */
    SS_FIELD_VY = 1,            /* nx*(ny+1)*nz */
    SS_FIELD_VZ = 2,            /* nx*ny*(nz+1), 3D only */
    SS_FIELD_DENSITY = 3,       /* density_channels planes of nx*ny*nz, channel-major */
    SS_FIELD_TEMPERATURE = 4,   /* nx*ny*nz */
    SS_FIELD_PRESSURE = 5,      /* nx*ny*nz, level 0 (warm start of the next solve) */
    SS_FIELD_SOLID = 6,         /* nx*ny*nz floats: 1 solid, 0 fluid (alpha channel of the solid map) */
    SS_FIELD_DIVERGENCE = 7     /* nx*ny*nz, discrete divergence of the current velocities (read only) */
};

/* ---- statistics of the last step / solve ----------------------------------- */
typedef struct ss_stats {
    int vcycles;                /* V-cycles (or refinement iterations) of the last solve */
    int converged;              /* 1 when tol > 0 was met */
    double div_before;          /* ||div u||_2 over fluid cells entering the solve */
    double residual;            /* ||div u - (dt/(rho h)) L p||_2 at exit of the solve */
    double div_after;           /* ||div u||_2 after update_velocities (FP64 evaluation) */
    double rel_div;             /* div_after / div_before */
    int steps;                  /* steps run by the last ss_run_physics_step */
    int fluid_cells;
    long long kernel_launches;  /* CUDA kernels launched by the last ss_run_physics_step */
} ss_stats;

/* ---- lifetime --------------------------------------------------------------- */
int ss_create(const ss_desc* desc, void* stream, ss_sim** out);
int ss_destroy(ss_sim* sim);
int ss_get_desc(const ss_sim* sim, ss_desc* out, int* levels, int level_sizes[][3]);
const char* ss_strerror(int status);
const char* ss_last_error_message(void);
int ss_abi_version(void);

/* Default parameters = reference get_default_p_settings / get_default_p_s_settings
 * (common/physics/physics.c:7-33) and the reference solver schedule. */
void ss_default_params(ss_params* out);

/* ---- scene (reference upload_emitters / upload_obstacles) ------------------- */
/* Copies the scene to the device and rasterises the solid map now (the
 * reference does this at the end of every frame, common/physics/physics.c:99-100). */
int ss_set_scene(ss_sim* sim, const ss_emitter* emitters, int n_emitters,
                 const ss_obstacle* obstacles, int n_obstacles,
                 const ss_box* boxes, int n_boxes, void* stream);
/* Current emitter / obstacle state (reference extract_obstacles_data, obstacles.c). */
int ss_get_scene(ss_sim* sim, ss_emitter* emitters, int n_emitters,
                 ss_obstacle* obstacles, int n_obstacles);

/* ---- state I/O ----------------------------------------------------------------- */
int ss_set_field(ss_sim* sim, int field, const float* host, size_t count, void* stream);
int ss_get_field(ss_sim* sim, int field, float* host, size_t count, void* stream);
/* Device pointer of the current buffer of a field (for a renderer).  Valid until
 * the next call that swaps buffers. */
int ss_field_device_ptr(ss_sim* sim, int field, void** dptr, size_t* count);
/* Device-to-device copies of a field (stream-ordered, no synchronisation):
 * for renderers and autograd bindings that hold the data on the GPU. */
int ss_set_field_device(ss_sim* sim, int field, const float* dev, size_t count, void* stream);
int ss_get_field_device(ss_sim* sim, int field, float* dev, size_t count, void* stream);
/* Reference clear_grid (3d/grid3d.c:164-183): zero velocities and pressure,
 * smoke = (0, 0, 0, t_ambient). */
int ss_clear_grid(ss_sim* sim, float t_ambient, void* stream);

/* ---- the step ------------------------------------------------------------------ */
/* Reference run_physics_step (common/physics/physics.c:72-101), nsteps times. */
int ss_run_physics_step(ss_sim* sim, const ss_params* params, int nsteps, void* stream);
/* Statistics of the last ss_run_physics_step call.  Every bounded wait inside
 * a kernel that gave up (bit 0 of the simulation's device error word: a
 * coarse-level sweep whose TMA tile loads did not arrive in time) is reported
 * as SS_E_CUDA by the next call that reads the device back - ss_get_stats,
 * ss_get_field with a host destination, or the step itself when it collects
 * statistics or solves to a tolerance - and then cleared.  A step that neither
 * collects statistics nor solves to a tolerance returns SS_OK before its
 * kernels ran, so check one of those calls before trusting its fields. */
int ss_get_stats(ss_sim* sim, ss_stats* out);

/* ---- individual stages (reference common/physics/grid.h:37-68) -------------- */
int ss_update_emitters_status(ss_sim* sim, const ss_params* params, void* stream);   /* grid.c:89-93 */
int ss_handle_emitters(ss_sim* sim, const ss_params* params, void* stream);          /* grid.c:78-87 */
int ss_advect_velocities(ss_sim* sim, const ss_params* params, void* stream);        /* grid.c:57-76 */
int ss_apply_buoyancy(ss_sim* sim, const ss_params* params, void* stream);           /* grid.c:106-115 */
int ss_apply_vorticity(ss_sim* sim, const ss_params* params, void* stream);          /* grid.c:117-145 (calculate + apply) */
int ss_multigrid_pressure_solve(ss_sim* sim, const ss_params* params, void* stream); /* grid.c:173-175 */
int ss_v_cycle(ss_sim* sim, const ss_params* params, int level, void* stream);       /* grid.c:177-209 */
int ss_smooth(ss_sim* sim, const ss_params* params, int level, int iterations, void* stream); /* grid.c:211-234 */
int ss_compute_residual(ss_sim* sim, const ss_params* params, int level, void* stream);       /* grid.c:235-242 */
int ss_compute_restrict(ss_sim* sim, const ss_params* params, int level, void* stream);       /* grid.c:243-257 */
int ss_prolong_and_add(ss_sim* sim, const ss_params* params, int level, void* stream);        /* grid.c:259-266 */
int ss_update_velocities(ss_sim* sim, const ss_params* params, void* stream);        /* grid.c:36-55 */
int ss_advect_smoke(ss_sim* sim, const ss_params* params, void* stream);             /* grid.c:95-104 */
int ss_obstacle_update_step(ss_sim* sim, const ss_params* params, void* stream);     /* grid.c:156-162 */
int ss_update_solid_map(ss_sim* sim, void* stream);                                  /* grid.c:164-171 */
int ss_init_solid_map(ss_sim* sim, void* stream);                                    /* grid.c:147-154 */

/* ---- allocation-free divergence norm ---------------------------------------- */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc -
 * a host application that hands out all device memory from its own fixed
 * budget (a game engine or renderer with a VRAM cap), or a per-frame callback
 * where an allocation would stall the frame - and that therefore cannot create
 * an ss_sim.  Writes to *out_norm (device memory, one double) the L2 norm over
 * fluid cells of the discrete divergence of the caller's MAC velocities u, v,
 * w (device arrays in the layout above; w unused when dim == 2), where
 * solid[c] != 0 marks solid cells (device, one byte per cell), solid
 * neighbours' faces count as velocity 0 and out-of-grid neighbours as fluid:
 * the quantity ss_stats.div_before reports when every obstacle is at rest.
 * Allocates nothing: its scratch (16384 FP64 partial sums, 128 KiB) is a
 * static device array that every GPU loading this library holds until exit.
 * At most 67,108,864 cells; larger grids return SS_E_INVALID.  The first call
 * on each device looks up that array's address (a one-time set-up, repeated
 * only when the device's CUDA context changed, e.g. after cudaDeviceReset);
 * make that first call before any stream capture begins.  All calls share the
 * scratch, so calls that overlap on the GPU (different streams, no ordering)
 * race. */
int ss_divergence_norm_noalloc(int dim, const int n[3], const float* u, const float* v, const float* w,
                               const uint8_t* solid, double* out_norm, void* stream);

/* ---- adjoint (reverse-mode derivatives of a rollout) ------------------------ */
/* No counterpart in the reference.  Hand-written transposes of every stage:
 * semi-Lagrangian advection as a scatter-add plus the chain rule through the
 * back-traced point, buoyancy, vorticity confinement, the projection update,
 * each V-cycle of the multigrid schedule (red-black sweeps in reverse colour
 * order, residual + restriction, prolongation) and the divergence.  The
 * projection must run the corrected operators (ref_quirks = 0); with the
 * mixed-precision solve the forward's recorded refinement steps are
 * transposed as FP32 V-cycles (the same linear map in exact arithmetic);
 * obstacles are treated as fixed geometry.
 *
 * Control force: every step adds dt * force to the face velocities inside
 * the active emitters (after their velocity injection); ss_set_emitter_force
 * sets it for plain steps, the rollout below takes one per step. */
int ss_set_emitter_force(ss_sim* sim, const float force[3]);

/* Coarse control force field (an extension for inverse control; no
 * counterpart in the reference): three components on n^3 cell-centred samples
 * spanning the whole domain, upsampled trilinearly (clamp to edge) to every
 * face position and added as dt * F to the face velocities after the
 * emitters, every step.  field: host array of 3*n*n*n floats, component-major
 * (F_x, then F_y, then F_z), x fastest; n = 0 removes the field.  3D only. */
int ss_set_force_field(ss_sim* sim, int n, const float* field, void* stream);

typedef struct ss_adjoint ss_adjoint;
/* A rollout of nsteps steps from the simulation's current state, with the
 * state checkpointed every checkpoint_every steps (0: every step) so the
 * reverse pass recomputes at most checkpoint_every steps per segment. */
int ss_adjoint_create(ss_sim* sim, int nsteps, int checkpoint_every, ss_adjoint** out);
int ss_adjoint_destroy(ss_adjoint* adj);
/* Forward pass: nsteps steps with params, forces[k*3 + d] (host, NULL = no
 * force) on step k.  Leaves the simulation in the final state. */
int ss_adjoint_forward(ss_adjoint* adj, const ss_params* params, const float* forces, void* stream);
/* Reverse pass for a loss of the final state: grad_density (nch*nx*ny*nz),
 * grad_temperature and grad_velocity[d] are device arrays of dL/d(final
 * field), any of them NULL for zero.  Writes dL/d(force) per step to
 * grad_forces (host, nsteps*3, may be NULL); the derivatives with respect to
 * the initial state are then read with ss_adjoint_field_device_ptr.  The
 * simulation is left in the rollout's initial state. */
int ss_adjoint_backward(ss_adjoint* adj, const ss_params* params, const float* grad_density,
                        const float* grad_temperature, const float* const grad_velocity[3], float* grad_forces,
                        void* stream);
/* dL/d(initial field) after ss_adjoint_backward: SS_FIELD_VX/VY/VZ/DENSITY/
 * TEMPERATURE/PRESSURE (the pressure that warm-starts the first solve). */
int ss_adjoint_field_device_ptr(ss_adjoint* adj, int field, void** dptr, size_t* count);
/* the same copied to dst (device memory when dst_on_device, else host) */
int ss_adjoint_get_field(ss_adjoint* adj, int field, float* dst, size_t count, int dst_on_device, void* stream);
/* Scatter-adds of the reverse pass: on = 0 (default) sums with atomicAdd, so
 * two reverse passes agree only to rounding; on = 1 switches to the
 * owner-computes variant (each destination enumerates the sources whose
 * trilinear taps cover it and sums them in a fixed order), which gives
 * bitwise-identical gradients run to run at a higher cost.  Allocates its
 * scratch (32 bytes per face) on first use. */
int ss_adjoint_set_deterministic(ss_adjoint* adj, int on);
/* Statistics of the last reverse pass: kernel launches and device bytes held
 * by checkpoints and recomputation buffers. */
/* Pressure store (off by default): with on != 0 the next ss_adjoint_forward
 * also keeps every step's solved pressure (nsteps fields, FP64 with the
 * mixed-precision solve, FP32 otherwise), and ss_adjoint_backward's
 * recomputation of a segment takes the stored pressure instead of running the
 * pressure solve again.  The recomputed states - and so the gradients - are
 * the same; the reverse pass saves one pressure solve per recomputed step for
 * nsteps * ncell * 8 bytes of device memory (counted in checkpoint_bytes). */
int ss_adjoint_set_pressure_store(ss_adjoint* adj, int on);
int ss_adjoint_info(ss_adjoint* adj, long long* kernel_launches, long long* checkpoint_bytes, long long* workspace_bytes);
/* dL/d(force field) after ss_adjoint_backward: 3*n^3 floats (host), the layout
 * of ss_set_force_field; count must match the simulation's field. */
int ss_adjoint_force_field_grad(ss_adjoint* adj, float* dst, size_t count);

/* ---- headless renderer -------------------------------------------------- */
/* Replaces the reference's GL fragment shaders with CUDA kernels writing an
 * RGBA8 image: 3D ray_march_smoke.frag:114-175 (front-to-back compositing
 * with alpha = 1 - exp(-density * k * step), a shadow march towards the light,
 * a Henyey-Greenstein phase of g = 0.5 scaled by 3, a per-pixel hash
 * jitter of the first sample), 2D draw_smoke.frag:43-58 (ambient / smoke
 * colour mix).  The box spans [0, n_d / min(n)] per axis; there is no scene
 * depth buffer headless, so every ray runs to the box exit.  Single-channel
 * density renders as grey smoke (r = g = b = density). */
typedef struct ss_render_desc {
    int width, height;              /* image size; rows are written top row first */
    float camera_pos[3];            /* box space (3D) */
    float camera_target[3];
    float camera_up[3];
    float fov_y;                    /* vertical field of view, radians */
    float light_direction[3];       /* towards the light (normalised by the renderer) */
    float light_color[3];
    float ambient_color[3];
    float smoke_density_factor;
    float shadow_density_factor;
    float step_size;                /* box units */
    float shadow_step_factor;
    int shadow_steps;
    float phase_g;
} ss_render_desc;
/* defaults of the reference's graphics_settings (common/graphics/graphics.c:9-25)
 * and a camera outside the +z face looking at the box centre */
int ss_render_default(const ss_sim* sim, int width, int height, ss_render_desc* out);
/* rgba: width*height*4 bytes, device memory when on_device, else host */
int ss_render(ss_sim* sim, const ss_render_desc* desc, uint8_t* rgba, int on_device, void* stream);

/* ---- snapshots ---------------------------------------------------------- */
/* No counterpart in the reference (its state lives in GL textures).  One line
 * of JSON (format "smokesim-state", grid, and for every section its name,
 * dtype, shape, byte offset and length; padded to 64 bytes) followed by raw
 * little-endian sections: vx, vy[, vz], density, temperature, pressure
 * (FP32, x fastest) and the emitter / obstacle / box records.  Loading needs
 * a simulation with the same grid description; it restores the scene, then
 * the fields. */
int ss_save_state(ss_sim* sim, const char* path, void* stream);
int ss_load_state(ss_sim* sim, const char* path, void* stream);

/* Level data of the multigrid pyramid (pressure / residual), for tests. */
enum ss_level_field { SS_LEVEL_PRESSURE = 0, SS_LEVEL_RESIDUAL = 1, SS_LEVEL_FLUID_WEIGHT = 2 };
int ss_get_level(ss_sim* sim, int level, int what, float* host, size_t count, void* stream);
int ss_set_level(ss_sim* sim, int level, int what, const float* host, size_t count, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SMOKESIM_B200_H */
