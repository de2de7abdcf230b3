// k_fluid.cu - per-cell / per-face stages of the smoke step.
//
// Each kernel restates one or more reference compute shaders; the shader is
// cited at the kernel.  Velocities are read from the current ping-pong buffer
// and written to the other one (the reference's texture/image pairs,
// 3d/grid3d.c:104-162), smoke likewise.
#include <type_traits>

#include <cmath>

#include "common.cuh"
#include "ss_internal.h"

namespace ss {

struct FluidArgs {
    int nx, ny, nz, nch;
    const float* u;
    const float* v;
    const float* w;
    float* uo;
    float* vo;
    float* wo;
    const uint8_t* flags;
    const float* dens;
    const float* temp;
    float* dens_o;
    float* temp_o;
    const float* sv0;
    const float* sv1;
    const float* sv2;
    StepConsts c;
};

static FluidArgs fluid_args(ss_sim* s, const StepConsts& c) {
    FluidArgs a;
    a.nx = s->nx; a.ny = s->ny; a.nz = s->nz; a.nch = s->nch;
    a.u = s->vel[0][s->vi[0]]; a.v = s->vel[1][s->vi[1]]; a.w = s->dim == 3 ? s->vel[2][s->vi[2]] : nullptr;
    a.uo = s->vel[0][1 - s->vi[0]]; a.vo = s->vel[1][1 - s->vi[1]];
    a.wo = s->dim == 3 ? s->vel[2][1 - s->vi[2]] : nullptr;
    a.flags = s->flags;
    a.dens = s->dens[s->si]; a.temp = s->temp[s->si];
    a.dens_o = s->dens[1 - s->si]; a.temp_o = s->temp[1 - s->si];
    a.sv0 = s->svel_active ? s->svel[0] : nullptr;
    a.sv1 = s->svel_active ? s->svel[1] : nullptr;
    a.sv2 = s->svel_active ? s->svel[2] : nullptr;
    a.c = c;
    return a;
}

SS_D bool solid_oob1(const uint8_t* __restrict__ f, int x, int y, int z, int nx, int ny, int nz) {
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return true;
    return f[idx3(x, y, z, nx, ny)] & F_SOLID;
}
SS_D bool solid_oob0(const uint8_t* __restrict__ f, int x, int y, int z, int nx, int ny, int nz) {
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return false;
    return f[idx3(x, y, z, nx, ny)] & F_SOLID;
}

static inline dim3 grid_for(int ax, int ay, int az, dim3 b) {
    return dim3((ax + b.x - 1) / b.x, (ay + b.y - 1) / b.y, (az + b.z - 1) / b.z);
}

// ------------------------------------------------------------------ emitters
// handle_emitters (shaders3d/compute/handle_emitters.comp:49-76; 2D :47-74) on
// the bounding box of the active emitters, in place, plus the face-velocity
// extension.  Emitters are applied in array order, like the shader's loop.
template <int DIM>
__global__ void k_emitters(FluidArgs a, const ss_emitter* __restrict__ em, int ne, int lox, int loy, int loz,
                           int ex, int ey, int ez, float* __restrict__ dens, float* __restrict__ temp,
                           float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
                           float3 force, int forced) {
    int x = lox + blockIdx.x * blockDim.x + threadIdx.x;
    int y = loy + blockIdx.y * blockDim.y + threadIdx.y;
    int z = loz + blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= lox + ex || y >= loy + ey || z >= loz + ez) return;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const float dt = a.c.dt;
    if (x < nx && y < ny && z < nz) {
        const int c = idx3(x, y, z, nx, ny);
        const size_t ncell = (size_t)nx * ny * nz;
        float sm[3] = {0.f, 0.f, 0.f};
        for (int ch = 0; ch < a.nch; ++ch) sm[ch] = dens[ch * ncell + c];
        float t = temp[c];
        bool hit = false;
        for (int k = 0; k < ne; ++k) {
            const ss_emitter& e = em[k];
            if (!(e.emit > 0)) continue;
            float dx = (float)x - e.pos[0], dy = (float)y - e.pos[1];
            float d2 = dx * dx + dy * dy;
            if constexpr (DIM == 3) { float dz = (float)z - e.pos[2]; d2 = d2 + dz * dz; }
            float dist = sqrtf(d2);
            float rad = e.radius;
            if (dist < rad) {
                float falloff;
                if (e.falloff > 0) {
                    float tt = (dist - rad) / (0.f - rad);
                    tt = clampt(tt, 0.f, 1.f);
                    falloff = tt * tt * (3.f - 2.f * tt);
                } else {
                    falloff = 1.f;
                }
                for (int ch = 0; ch < a.nch; ++ch) sm[ch] = sm[ch] + e.density[ch] * falloff * dt;
                t = t + e.temperature * falloff * dt;
                hit = true;
            }
        }
        if (hit) {
            for (int ch = 0; ch < a.nch; ++ch) dens[ch * ncell + c] = sm[ch];
            temp[c] = t;
        }
    }
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        float val = 0.f;
        bool hit = false, inside = false;
        for (int k = 0; k < ne; ++k) {
            const ss_emitter& e = em[k];
            if (!(e.emit > 0)) continue;
            float dx = (float)x - e.pos[0], dy = (float)y - e.pos[1];
            float d2 = dx * dx + dy * dy;
            if constexpr (DIM == 3) { float dz = (float)z - e.pos[2]; d2 = d2 + dz * dz; }
            if (sqrtf(d2) < e.radius) {
                inside = true;
                if (e.set_velocity) { val = e.velocity[comp]; hit = true; }
            }
        }
        // control force (an extension for the adjoint's inverse problems):
        // dt * force on every face inside an active emitter, after the set
        if (hit || (forced && inside)) {
            float* dst = comp == 0 ? u : comp == 1 ? v : w;
            const int i = idx3(x, y, z, ax, ay);
            float out = hit ? val : dst[i];
            if (forced && inside) out = out + dt * (comp == 0 ? force.x : comp == 1 ? force.y : force.z);
            dst[i] = out;
        }
    }
}

int launch_emitters(ss_sim* s, const StepConsts& c, cudaStream_t st) {
    // bounding box (cells and faces) of the active emitters
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-1, -1, -1};
    int active = 0;
    for (const ss_emitter& e : s->em) {
        if (!(e.emit > 0)) continue;
        ++active;
        for (int d = 0; d < s->dim; ++d) {
            int a = (int)floorf(e.pos[d] - e.radius) - 1, b = (int)ceilf(e.pos[d] + e.radius) + 2;
            lo[d] = lo[d] < a ? lo[d] : a;
            hi[d] = hi[d] > b ? hi[d] : b;
        }
    }
    if (!active) return SS_OK;
    if (s->dim == 2) { lo[2] = 0; hi[2] = 1; }
    const int ext[3] = {s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1};
    for (int d = 0; d < 3; ++d) {
        lo[d] = lo[d] < 0 ? 0 : lo[d];
        hi[d] = hi[d] > ext[d] ? ext[d] : hi[d];
        if (hi[d] <= lo[d]) return SS_OK;
    }
    FluidArgs a = fluid_args(s, c);
    const float3 f = make_float3(s->force[0], s->force[1], s->force[2]);
    const int forced = (s->force[0] != 0.f || s->force[1] != 0.f || s->force[2] != 0.f) ? 1 : 0;
    dim3 b(32, 4, 1);
    dim3 g = grid_for(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], b);
    float* u = s->vel[0][s->vi[0]];
    float* v = s->vel[1][s->vi[1]];
    float* w = s->dim == 3 ? s->vel[2][s->vi[2]] : nullptr;
    if (s->dim == 3)
        k_emitters<3><<<g, b, 0, st>>>(a, s->d_em, (int)s->em.size(), lo[0], lo[1], lo[2], hi[0] - lo[0],
                                       hi[1] - lo[1], hi[2] - lo[2], s->dens[s->si], s->temp[s->si], u, v, w, f, forced);
    else
        k_emitters<2><<<g, b, 0, st>>>(a, s->d_em, (int)s->em.size(), lo[0], lo[1], lo[2], hi[0] - lo[0],
                                       hi[1] - lo[1], hi[2] - lo[2], s->dens[s->si], s->temp[s->si], u, v, w, f, forced);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_emitters");
}

// ------------------------------------------------- coarse control force field
// Extension (inverse control): F, three components on n^3 cell-centred samples
// over the domain, sampled at each face position with GL_LINEAR +
// CLAMP_TO_EDGE arithmetic (the pressure prolongation's) and added as dt * F.
SS_D void coarse_taps(int n, float t, int* a, int* b, float* w) {
    const float f = floorf(t);
    const int i = (int)f;
    *w = t - f;
    *a = min(max(i, 0), n - 1);
    *b = min(max(i + 1, 0), n - 1);
}

// face (x, y, z) of axis comp in the coarse texel frame
SS_D void force_field_coords(int comp, int x, int y, int z, int nx, int ny, int nz, int n, float* tx, float* ty,
                             float* tz) {
    const float xf = (float)x + (comp == 0 ? 0.f : 0.5f);
    const float yf = (float)y + (comp == 1 ? 0.f : 0.5f);
    const float zf = (float)z + (comp == 2 ? 0.f : 0.5f);
    *tx = (xf / (float)nx) * (float)n - 0.5f;
    *ty = (yf / (float)ny) * (float)n - 0.5f;
    *tz = (zf / (float)nz) * (float)n - 0.5f;
}

__global__ void __launch_bounds__(256) k_force_field(float* __restrict__ u, float* __restrict__ v,
                                                     float* __restrict__ w, int nx, int ny, int nz,
                                                     const float* __restrict__ F, int n, float dt) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const size_t nn = (size_t)n * n * n;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        float tx, ty, tz;
        force_field_coords(comp, x, y, z, nx, ny, nz, n, &tx, &ty, &tz);
        int xa, xb, ya, yb, za, zb;
        float wx, wy, wz;
        coarse_taps(n, tx, &xa, &xb, &wx);
        coarse_taps(n, ty, &ya, &yb, &wy);
        coarse_taps(n, tz, &za, &zb, &wz);
        const float* f = F + comp * nn;
        const float c0 = lerp_(lerp_(__ldg(f + idx3(xa, ya, za, n, n)), __ldg(f + idx3(xb, ya, za, n, n)), wx),
                               lerp_(__ldg(f + idx3(xa, yb, za, n, n)), __ldg(f + idx3(xb, yb, za, n, n)), wx), wy);
        const float c1 = lerp_(lerp_(__ldg(f + idx3(xa, ya, zb, n, n)), __ldg(f + idx3(xb, ya, zb, n, n)), wx),
                               lerp_(__ldg(f + idx3(xa, yb, zb, n, n)), __ldg(f + idx3(xb, yb, zb, n, n)), wx), wy);
        const float val = lerp_(c0, c1, wz);
        float* dst = comp == 0 ? u : comp == 1 ? v : w;
        const int i = idx3(x, y, z, ax, ay);
        dst[i] = dst[i] + dt * val;
    }
}

int launch_force_field(ss_sim* s, const StepConsts& c, cudaStream_t st) {
    if (s->ff_n <= 0 || s->dim != 3) return SS_OK;
    dim3 b(32, 8, 1);
    dim3 g = grid_for(s->nx + 1, s->ny + 1, s->nz + 1, b);
    k_force_field<<<g, b, 0, st>>>(s->vel[0][s->vi[0]], s->vel[1][s->vi[1]], s->vel[2][s->vi[2]], s->nx, s->ny, s->nz,
                                   s->ffield, s->ff_n, c.dt);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_force_field");
}

// ------------------------------------------------------- velocity advection
// advect_vx / advect_vy / advect_vz (shaders3d/compute/advect_vx.comp:54-77,
// advect_vy.comp:55-79, advect_vz.comp:55-78; 2D advect_vx.comp:50-73,
// advect_vy.comp:51-75).  With BUOY, apply_buoyancy (apply_buoyancy.comp:39-52)
// is fused into the y faces: a y face touching solid (out of grid = fluid)
// keeps the value the reference's write buffer holds there, which after the
// advection swap is the pre-advection velocity.
// mean of a cell array at the two cells either side of the y face (x, y, z):
// texel (x, y-1/2, z), weights 0 / 0.5 / 0
template <int DIM>
SS_D float yface_mean(const float* __restrict__ a, int nx, int ny, int nz, int x, int y, int z, float border) {
    return lerp_(fetch_b(a, nx, ny, nz, x, y - 1, z, border), fetch_b(a, nx, ny, nz, x, y, z, border), 0.5f);
}

template <int DIM, bool BUOY>
__global__ void __launch_bounds__(256) k_advect_velocity(FluidArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const float cfl = a.c.cfl;
    // linear indices of position (x, y, z) in the cell / w array (c), the u
    // array and the v array, and the plane sizes: every tap of the face
    // averages below is one of these plus a fixed offset
    const int zy = z * ny + y;
    const int c = zy * nx + x;
    const int iu = c + zy, iv = c + z * nx;
    const int ux = nx + 1, pl = nx * ny, plu = ux * ny, plv = nx * (ny + 1);
    const bool in_cell = x < nx && y < ny && z < nz;
    // solid flags of this cell and of its -x, -y, -z neighbours (out of grid = solid)
    const bool s_c = !in_cell || (a.flags[c] & F_SOLID);
    // every tap of the face velocities below lies inside the arrays
    const bool interior = x >= 1 && y >= 1 && (DIM == 2 || z >= 1) && in_cell;
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        const float* __restrict__ src = comp == 0 ? a.u : comp == 1 ? a.v : a.w;
        float* __restrict__ dst = comp == 0 ? a.uo : comp == 1 ? a.vo : a.wo;
        const int i = comp == 0 ? iu : comp == 1 ? iv : c;
        const int id = comp == 0 ? x : comp == 1 ? y : z;
        // the cell on the face's low side: out of grid (id == 0) counts solid
        const bool s_lo = id == 0 || (a.flags[c - (comp == 0 ? 1 : comp == 1 ? nx : pl)] & F_SOLID);
        float out;
        if (id == 0 && a.c.wind[comp] != 0.f) {
            out = a.c.wind[comp];
        } else if (s_c || s_lo) {
            out = 0.f;
        } else {
            float vel[3];
            if (interior) {
                // vel_at_face_interior's values, its taps addressed from i, c
                if (comp == 0) {
                    vel[0] = __ldg(a.u + iu);
                    const float* pv = a.v + iv - 1;
                    vel[1] = lerp_(lerp_(__ldg(pv), __ldg(pv + 1), 0.5f), lerp_(__ldg(pv + nx), __ldg(pv + nx + 1), 0.5f),
                                   0.5f);
                    if constexpr (DIM == 3) {
                        const float* pw = a.w + c - 1;
                        vel[2] = lerp_(lerp_(__ldg(pw), __ldg(pw + 1), 0.5f),
                                       lerp_(__ldg(pw + pl), __ldg(pw + pl + 1), 0.5f), 0.5f);
                    } else {
                        vel[2] = 0.f;
                    }
                } else if (comp == 1) {
                    const float* pu = a.u + iu - ux;
                    vel[0] = lerp_(lerp_(__ldg(pu), __ldg(pu + 1), 0.5f), lerp_(__ldg(pu + ux), __ldg(pu + ux + 1), 0.5f),
                                   0.5f);
                    vel[1] = __ldg(a.v + iv);
                    if constexpr (DIM == 3) {
                        const float* pw = a.w + c - nx;
                        vel[2] = lerp_(lerp_(__ldg(pw), __ldg(pw + nx), 0.5f),
                                       lerp_(__ldg(pw + pl), __ldg(pw + pl + nx), 0.5f), 0.5f);
                    } else {
                        vel[2] = 0.f;
                    }
                } else {
                    const float* pu = a.u + iu - plu;
                    vel[0] = lerp_(lerp_(__ldg(pu), __ldg(pu + 1), 0.5f), lerp_(__ldg(pu + plu), __ldg(pu + plu + 1), 0.5f),
                                   0.5f);
                    const float* pv = a.v + iv - plv;
                    vel[1] = lerp_(lerp_(__ldg(pv), __ldg(pv + nx), 0.5f), lerp_(__ldg(pv + plv), __ldg(pv + plv + nx), 0.5f),
                                   0.5f);
                    vel[2] = __ldg(a.w + c);
                }
            } else if (comp == 0) {
                vel_at_xface<DIM>(a.u, a.v, a.w, nx, ny, nz, x, y, z, vel);
            } else if (comp == 1) {
                vel_at_yface<DIM>(a.u, a.v, a.w, nx, ny, nz, x, y, z, vel);
            } else {
                vel_at_zface(a.u, a.v, a.w, nx, ny, nz, x, y, z, vel);
            }
            const float gx = (float)x + (comp == 0 ? 0.f : 0.5f);
            const float gy = (float)y + (comp == 1 ? 0.f : 0.5f);
            const float gz = DIM == 3 ? (float)z + (comp == 2 ? 0.f : 0.5f) : 0.f;
            const float bx = gx - vel[0] * cfl, by = gy - vel[1] * cfl, bz = gz - vel[2] * cfl;
            const Taps t = make_taps<DIM>(ax, ay, az, bx - (comp == 0 ? 0.f : 0.5f), by - (comp == 1 ? 0.f : 0.5f),
                                          bz - (comp == 2 ? 0.f : 0.5f));
            out = sample_taps_fast<DIM>(src, ax, ay, az, t, 0.f);
        }
        if constexpr (BUOY) {
            if (comp == 1) {
                // the y face's two cells (out of grid = fluid)
                const bool solid_hi = y < ny && in_cell && (a.flags[c] & F_SOLID);
                const bool solid_lo = y > 0 && x < nx && z < nz && (a.flags[c - nx] & F_SOLID);
                if (solid_hi || solid_lo) {
                    out = __ldg(src + i);
                } else {
                    const size_t ncell = (size_t)nx * ny * nz;
                    float total = yface_mean<DIM>(a.dens, nx, ny, nz, x, y, z, 0.f);
                    if (a.nch == 3) {
                        total = total + yface_mean<DIM>(a.dens + ncell, nx, ny, nz, x, y, z, 0.f);
                        total = total + yface_mean<DIM>(a.dens + 2 * ncell, nx, ny, nz, x, y, z, 0.f);
                    }
                    const float T = yface_mean<DIM>(a.temp, nx, ny, nz, x, y, z, a.c.t_amb);
                    const float buoy = -a.c.alpha * total + a.c.beta * (T - a.c.t_amb);
                    out = out + buoy * a.c.dt;
                }
            }
        }
        dst[i] = out;
    }
}

int launch_advect_velocities(ss_sim* s, const StepConsts& c, bool fuse_buoyancy, cudaStream_t st) {
    FluidArgs a = fluid_args(s, c);
    dim3 b(32, 8, 1);
    dim3 g = grid_for(s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1, b);
    if (s->dim == 3) {
        if (fuse_buoyancy) k_advect_velocity<3, true><<<g, b, 0, st>>>(a);
        else k_advect_velocity<3, false><<<g, b, 0, st>>>(a);
    } else {
        if (fuse_buoyancy) k_advect_velocity<2, true><<<g, b, 0, st>>>(a);
        else k_advect_velocity<2, false><<<g, b, 0, st>>>(a);
    }
    for (int d = 0; d < s->dim; ++d) s->vi[d] ^= 1;
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_advect_velocity");
}

// ----------------------------------------------------------------- buoyancy
// apply_buoyancy (shaders3d/compute/apply_buoyancy.comp:39-52; 2D :37-50) as a
// stand-alone stage: faces touching solid are not written.
template <int DIM>
__global__ void k_buoyancy(FluidArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    if (x >= nx || y >= ny + 1 || z >= nz) return;
    if (solid_oob0(a.flags, x, y, z, nx, ny, nz) || solid_oob0(a.flags, x, y - 1, z, nx, ny, nz)) return;
    const size_t ncell = (size_t)nx * ny * nz;
    float total = yface_mean<DIM>(a.dens, nx, ny, nz, x, y, z, 0.f);
    if (a.nch == 3) {
        total = total + yface_mean<DIM>(a.dens + ncell, nx, ny, nz, x, y, z, 0.f);
        total = total + yface_mean<DIM>(a.dens + 2 * ncell, nx, ny, nz, x, y, z, 0.f);
    }
    const float T = yface_mean<DIM>(a.temp, nx, ny, nz, x, y, z, a.c.t_amb);
    const float buoy = -a.c.alpha * total + a.c.beta * (T - a.c.t_amb);
    const int i = idx3(x, y, z, nx, ny + 1);
    a.vo[i] = a.v[i] + buoy * a.c.dt;
}

int launch_buoyancy(ss_sim* s, const StepConsts& c, cudaStream_t st) {
    FluidArgs a = fluid_args(s, c);
    dim3 b(32, 8, 1);
    dim3 g = grid_for(s->nx, s->ny + 1, s->nz, b);
    if (s->dim == 3) k_buoyancy<3><<<g, b, 0, st>>>(a);
    else k_buoyancy<2><<<g, b, 0, st>>>(a);
    s->vi[1] ^= 1;
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_buoyancy");
}

// ---------------------------------------------------------------- vorticity
// calculate_vorticity (shaders3d/compute/calculate_vorticity.comp:59-84; 2D
// :51-69).  Velocity fetches outside the face arrays read 0.
template <int DIM>
__global__ void k_vorticity(FluidArgs a, float* __restrict__ vort) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    if (x >= nx || y >= ny || z >= nz) return;
    const int c = idx3(x, y, z, nx, ny);
    const size_t ncell = (size_t)nx * ny * nz;
    const float two_h = 2.f * a.c.vort_k;
    if (a.flags[c] & F_SOLID) {
        vort[c] = 0.f;
        if constexpr (DIM == 3) { vort[ncell + c] = 0.f; vort[2 * ncell + c] = 0.f; vort[3 * ncell + c] = 0.f; }
        return;
    }
    const float* u = a.u;
    const float* v = a.v;
    const float* w = a.w;
#define CCX(X, Y, Z) ((fetch_b(u, nx + 1, ny, nz, X, Y, Z, 0.f) + fetch_b(u, nx + 1, ny, nz, (X) + 1, Y, Z, 0.f)) * 0.5f)
#define CCY(X, Y, Z) ((fetch_b(v, nx, ny + 1, nz, X, Y, Z, 0.f) + fetch_b(v, nx, ny + 1, nz, X, (Y) + 1, Z, 0.f)) * 0.5f)
#define CCZ(X, Y, Z) ((fetch_b(w, nx, ny, nz + 1, X, Y, Z, 0.f) + fetch_b(w, nx, ny, nz + 1, X, Y, (Z) + 1, 0.f)) * 0.5f)
    if constexpr (DIM == 2) {
        const float z1 = CCY(x + 1, y, 0) - CCY(x - 1, y, 0);
        const float z2 = CCX(x, y + 1, 0) - CCX(x, y - 1, 0);
        vort[c] = (z1 - z2) / two_h;
    } else {
        const float x1 = CCZ(x, y + 1, z) - CCZ(x, y - 1, z);
        const float x2 = CCY(x, y, z + 1) - CCY(x, y, z - 1);
        const float y1 = CCX(x, y, z + 1) - CCX(x, y, z - 1);
        const float y2 = CCZ(x + 1, y, z) - CCZ(x - 1, y, z);
        const float z1 = CCY(x + 1, y, z) - CCY(x - 1, y, z);
        const float z2 = CCX(x, y + 1, z) - CCX(x, y - 1, z);
        const float o0 = (x1 - x2) / two_h, o1 = (y1 - y2) / two_h, o2 = (z1 - z2) / two_h;
        vort[c] = o0;
        vort[ncell + c] = o1;
        vort[2 * ncell + c] = o2;
        // |w|, read six times by the neighbours' confinement force
        vort[3 * ncell + c] = sqrtf(o0 * o0 + o1 * o1 + o2 * o2);
    }
#undef CCX
#undef CCY
#undef CCZ
}

template <int DIM>
SS_D float vmag(const float* __restrict__ vort, int x, int y, int z, int nx, int ny, int nz) {
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0.f;
    const int c = idx3(x, y, z, nx, ny);
    if constexpr (DIM == 2) {
        return fabsf(__ldg(vort + c));
    } else {
        // |w| stored by k_vorticity with the same expression
        return __ldg(vort + 3 * (size_t)nx * ny * nz + c);
    }
}

// apply_vorticity_x/y/z (shaders3d/compute/apply_vorticity_x.comp:43-63 and
// siblings; 2D apply_vorticity_x.comp:41-60, apply_vorticity_y.comp:41-60).
template <int DIM>
__global__ void __launch_bounds__(256) k_apply_vorticity(FluidArgs a, const float* __restrict__ vort) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const float two_h = 2.f * a.c.vort_k, eps = 1e-20f;
    const size_t ncell = (size_t)nx * ny * nz;
    // the force of cell (x,y,z) is shared by its three faces of the same index
    float f[3] = {0.f, 0.f, 0.f};
    bool have = false;
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        if (!have) {
            const float dx = vmag<DIM>(vort, x + 1, y, z, nx, ny, nz) - vmag<DIM>(vort, x - 1, y, z, nx, ny, nz);
            const float dy = vmag<DIM>(vort, x, y + 1, z, nx, ny, nz) - vmag<DIM>(vort, x, y - 1, z, nx, ny, nz);
            const bool in = x < nx && y < ny && z < nz;
            const int c = in ? idx3(x, y, z, nx, ny) : 0;
            if constexpr (DIM == 3) {
                const float dz = vmag<DIM>(vort, x, y, z + 1, nx, ny, nz) - vmag<DIM>(vort, x, y, z - 1, nx, ny, nz);
                const float gx = dx / two_h, gy = dy / two_h, gz = dz / two_h;
                const float len = sqrtf(gx * gx + gy * gy + gz * gz) + eps;
                const float nxv = gx / len, nyv = gy / len, nzv = gz / len;
                const float o0 = in ? __ldg(vort + c) : 0.f;
                const float o1 = in ? __ldg(vort + ncell + c) : 0.f;
                const float o2 = in ? __ldg(vort + 2 * ncell + c) : 0.f;
                f[0] = nyv * o2 - o1 * nzv;
                f[1] = nzv * o0 - o2 * nxv;
                f[2] = nxv * o1 - o0 * nyv;
            } else {
                const float gx = dx / two_h, gy = dy / two_h;
                const float len = sqrtf(gx * gx + gy * gy) + eps;
                const float nxv = gx / len, nyv = gy / len;
                const float o0 = in ? __ldg(vort + c) : 0.f;
                f[0] = -nyv * o0;
                f[1] = -nxv * o0;
            }
            have = true;
        }
        const float* __restrict__ src = comp == 0 ? a.u : comp == 1 ? a.v : a.w;
        float* __restrict__ dst = comp == 0 ? a.uo : comp == 1 ? a.vo : a.wo;
        const int i = idx3(x, y, z, ax, ay);
        dst[i] = __ldg(src + i) + (f[comp] * 0.5f * a.c.eps * a.c.vort_k * a.c.dt) / a.c.rho;
    }
}

// ------------------------------------------------- fused vorticity (3D)
// k_vorticity + k_apply_vorticity in one pass.  A block owns a 32x8 column of
// cells and marches up a chunk of z: each z-plane of u, v, w faces (with a
// two-cell x/y halo) is loaded once into a 4-plane ring in shared memory, w
// and |w| of plane z+1 are computed from the rings, and the confinement force
// of plane z updates its faces.  The per-cell expressions and their order are
// those of the two kernels above; w never goes through global memory.
// v is a power of two whose reciprocal is a normal float too
static bool pow2_normal(float v) {
    if (!(v > 0.f) || !std::isfinite(v)) return false;
    int e;
    return std::frexp(v, &e) == 0.5f && v >= 1.1754944e-38f && v <= 8.5070592e37f;
}

constexpr int kMX = 32, kMY = 8, kMZ = 32;   // tile and largest z chunk
constexpr int kUW = kMX + 3, kUH = kMY + 4;  // u faces x0-1 .. x0+kMX+1, rows y0-2 .. y0+kMY+1
constexpr int kVW = kMX + 4, kVH = kMY + 3;  // v faces: cols x0-2 .. x0+kMX+1, face rows y0-1 .. y0+kMY+1
constexpr int kWW = kMX + 4, kWH = kMY + 4;  // w faces: cols x0-2 .. x0+kMX+1, rows y0-2 .. y0+kMY+1
constexpr int kHW = kMX + 2, kHH = kMY + 2;  // |w|: cells x0-1 .. x0+kMX, y0-1 .. y0+kMY
constexpr int kMT = kMX * kMY;               // threads
constexpr int kUL = (kUW * kUH + kMT - 1) / kMT, kVL = (kVW * kVH + kMT - 1) / kMT, kWL = (kWW * kWH + kMT - 1) / kMT;

struct VortSmem {
    float u[4][kUH][kUW];
    float v[4][kVH][kVW];
    float w[4][kWH][kWW];
    float m[4][kHH][kHW];
    float o[2][3][kMY][kMX];
};

// POW2: 2h and rho are powers of two, so dividing by them is multiplying by
// their exact reciprocals (inv_2h, inv_rho) - the same correctly rounded value.
template <bool POW2>
__global__ void __launch_bounds__(kMT) k_vorticity_march(FluidArgs a, float inv_2h, float inv_rho, int planes) {
    __shared__ VortSmem S;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int x0 = blockIdx.x * kMX, y0 = blockIdx.y * kMY;
    const int zb = blockIdx.z * planes, ze = min(zb + planes, nz);
    const int tid = threadIdx.x;
    // in-plane offsets of this thread's loads (-1: outside the face array)
    int ou[kUL], ov[kVL], ow[kWL];
#pragma unroll
    for (int j = 0; j < kUL; ++j) {
        const int i = tid + j * kMT, X = x0 - 1 + i % kUW, Y = y0 - 2 + i / kUW;
        ou[j] = (i < kUW * kUH && X >= 0 && X <= nx && Y >= 0 && Y < ny) ? Y * (nx + 1) + X : -1;
    }
#pragma unroll
    for (int j = 0; j < kVL; ++j) {
        const int i = tid + j * kMT, X = x0 - 2 + i % kVW, Y = y0 - 1 + i / kVW;
        ov[j] = (i < kVW * kVH && X >= 0 && X < nx && Y >= 0 && Y <= ny) ? Y * nx + X : -1;
    }
#pragma unroll
    for (int j = 0; j < kWL; ++j) {
        const int i = tid + j * kMT, X = x0 - 2 + i % kWW, Y = y0 - 2 + i / kWW;
        ow[j] = (i < kWW * kWH && X >= 0 && X < nx && Y >= 0 && Y < ny) ? Y * nx + X : -1;
    }
    const size_t pu = (size_t)(nx + 1) * ny, pv = (size_t)nx * (ny + 1), pw = (size_t)nx * ny;
    float ru[kUL], rv[kVL], rw[kWL];
    // plane z of the three face arrays into registers (0 outside, as fetch_b)
    auto fetch_plane = [&](int z) {
        const bool zu = z >= 0 && z < nz, zw = z >= 0 && z <= nz;
#pragma unroll
        for (int j = 0; j < kUL; ++j) ru[j] = (zu && ou[j] >= 0) ? __ldg(a.u + z * pu + ou[j]) : 0.f;
#pragma unroll
        for (int j = 0; j < kVL; ++j) rv[j] = (zu && ov[j] >= 0) ? __ldg(a.v + z * pv + ov[j]) : 0.f;
#pragma unroll
        for (int j = 0; j < kWL; ++j) rw[j] = (zw && ow[j] >= 0) ? __ldg(a.w + z * pw + ow[j]) : 0.f;
    };
    auto store_plane = [&](int z) {
        const int sl = (z + 4) & 3;
#pragma unroll
        for (int j = 0; j < kUL; ++j) {
            const int i = tid + j * kMT;
            if (i < kUW * kUH) (&S.u[sl][0][0])[i] = ru[j];
        }
#pragma unroll
        for (int j = 0; j < kVL; ++j) {
            const int i = tid + j * kMT;
            if (i < kVW * kVH) (&S.v[sl][0][0])[i] = rv[j];
        }
#pragma unroll
        for (int j = 0; j < kWL; ++j) {
            const int i = tid + j * kMT;
            if (i < kWW * kWH) (&S.w[sl][0][0])[i] = rw[j];
        }
    };
    const float two_h = 2.f * a.c.vort_k;
    // This thread's (at most two) cells of the |w| tile, fixed for the
    // launch: halo index i = hy * kHW + hx.  The rows of the u / v, w rings
    // are one / two floats wider than the tile's, so a cell's ring offsets
    // are i + hy and i + 2 hy; only the ring slots change from plane to plane.
    constexpr int kHN = kHW * kHH;
    int hrow[2], fxy[2];
    bool hin[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int i = tid + j * kMT;
        hrow[j] = i / kHW;
        const int hx = i - hrow[j] * kHW;
        const int x = x0 - 1 + hx, y = y0 - 1 + hrow[j];
        hin[j] = i < kHN && x >= 0 && y >= 0 && x < nx && y < ny;
        fxy[j] = y * nx + x;
    }
    const int pl = nx * ny;
    // w and |w| of plane k from the rings (planes k-1 .. k+1 resident)
    auto vorticity_plane = [&](int k) {
        const int sm = (k + 3) & 3, s0 = (k + 4) & 3, sp = (k + 5) & 3;
        const float* U0 = &S.u[s0][0][0];
        const float* Um = &S.u[sm][0][0];
        const float* Up = &S.u[sp][0][0];
        const float* V0 = &S.v[s0][0][0];
        const float* Vm = &S.v[sm][0][0];
        const float* Vp = &S.v[sp][0][0];
        const float* W0 = &S.w[s0][0][0];
        const float* Wp = &S.w[sp][0][0];
        float* M0 = &S.m[s0][0][0];
        float* O = &S.o[k & 1][0][0][0];
        const bool kin = k >= 0 && k < nz;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int i = tid + j * kMT;
            if (i >= kHN) break;
            const int hy = hrow[j], hx = i - hy * kHW;
            const int ub = i + hy, vb = i + 2 * hy;
            float o0 = 0.f, o1 = 0.f, o2 = 0.f, m = 0.f;
            if (hin[j] && kin && !(a.flags[k * pl + fxy[j]] & F_SOLID)) {
                const float x1 = ((W0[vb + 2 * kWW + 1] + Wp[vb + 2 * kWW + 1]) * 0.5f) -
                                 ((W0[vb + 1] + Wp[vb + 1]) * 0.5f);
                const float x2 = ((Vp[vb + 1] + Vp[vb + kVW + 1]) * 0.5f) - ((Vm[vb + 1] + Vm[vb + kVW + 1]) * 0.5f);
                const float y1 = ((Up[ub + kUW] + Up[ub + kUW + 1]) * 0.5f) - ((Um[ub + kUW] + Um[ub + kUW + 1]) * 0.5f);
                const float y2 = ((W0[vb + kWW + 2] + Wp[vb + kWW + 2]) * 0.5f) - ((W0[vb + kWW] + Wp[vb + kWW]) * 0.5f);
                const float z1 = ((V0[vb + 2] + V0[vb + kVW + 2]) * 0.5f) - ((V0[vb] + V0[vb + kVW]) * 0.5f);
                const float z2 = ((U0[ub + 2 * kUW] + U0[ub + 2 * kUW + 1]) * 0.5f) - ((U0[ub] + U0[ub + 1]) * 0.5f);
                o0 = POW2 ? (x1 - x2) * inv_2h : (x1 - x2) / two_h;
                o1 = POW2 ? (y1 - y2) * inv_2h : (y1 - y2) / two_h;
                o2 = POW2 ? (z1 - z2) * inv_2h : (z1 - z2) / two_h;
                m = sqrtf(o0 * o0 + o1 * o1 + o2 * o2);
            }
            M0[i] = m;
            if (hx >= 1 && hy >= 1 && hx <= kMX && hy <= kMY) {
                const int ob = i - 2 * hy - kMX - 1;   // (hy - 1) * kMX + hx - 1
                O[ob] = o0;
                O[kMT + ob] = o1;
                O[2 * kMT + ob] = o2;
            }
        }
    };
    // prologue: planes zb-2 .. zb+1 of the faces, |w| of zb-1 and zb
    for (int z = zb - 2; z <= zb + 1; ++z) {
        fetch_plane(z);
        store_plane(z);
    }
    fetch_plane(zb + 2);
    __syncthreads();
    vorticity_plane(zb - 1);
    vorticity_plane(zb);
    __syncthreads();   // plane zb-2's slot is refilled next
    const int tx = tid % kMX, ty = tid / kMX;
    const int x = x0 + tx, y = y0 + ty;
    const float eps = 1e-20f;
    // this thread's ring offsets and output indices in the x-y plane
    const int mo = (ty + 1) * kHW + tx;
    const int uo_s = (ty + 2) * kUW + tx + 1, vo_s = (ty + 1) * kVW + tx + 2, wo_s = (ty + 2) * kWW + tx + 2;
    const int pu_o = (nx + 1) * ny, pv_o = nx * (ny + 1);
    const int uxy = y * (nx + 1) + x, vxy = y * nx + x;
    for (int z = zb; z < ze; ++z) {
        store_plane(z + 2);
        if (z + 1 < ze) fetch_plane(z + 3);
        __syncthreads();
        vorticity_plane(z + 1);
        __syncthreads();
        if (x < nx && y < ny) {
            const int sm = (z + 3) & 3, s0 = (z + 4) & 3, sp = (z + 5) & 3;
            const float* M0 = &S.m[s0][0][0];
            const float dx = M0[mo + 2] - M0[mo];
            const float dy = M0[mo + kHW + 1] - M0[mo - kHW + 1];
            const float dz = (&S.m[sp][0][0])[mo + 1] - (&S.m[sm][0][0])[mo + 1];
            const float gx = POW2 ? dx * inv_2h : dx / two_h;
            const float gy = POW2 ? dy * inv_2h : dy / two_h;
            const float gz = POW2 ? dz * inv_2h : dz / two_h;
            const float len = sqrtf(gx * gx + gy * gy + gz * gz) + eps;
            const float nxv = gx / len, nyv = gy / len, nzv = gz / len;
            const float* O = &S.o[z & 1][0][0][0];
            const float o0 = O[tid], o1 = O[kMT + tid], o2 = O[2 * kMT + tid];
            const float f0 = nyv * o2 - o1 * nzv, f1 = nzv * o0 - o2 * nxv, f2 = nxv * o1 - o0 * nyv;
            const float k = a.c.eps, vk = a.c.vort_k, dt = a.c.dt, rho = a.c.rho;
            auto term = [&](float f) {
                const float t = f * 0.5f * k * vk * dt;
                return POW2 ? t * inv_rho : t / rho;
            };
            const float* U0 = &S.u[s0][0][0];
            const float* V0 = &S.v[s0][0][0];
            const float* W0 = &S.w[s0][0][0];
            const int ui = z * pu_o + uxy, vi = z * pv_o + vxy, wi = z * pl + vxy;
            a.uo[ui] = U0[uo_s] + term(f0);
            a.vo[vi] = V0[vo_s] + term(f1);
            a.wo[wi] = W0[wo_s] + term(f2);
            // faces past the last cell: the force there is +0 (w = 0 outside the grid)
            const float zero_term = term(0.f);
            if (x == nx - 1) a.uo[ui + 1] = U0[uo_s + 1] + zero_term;
            if (y == ny - 1) a.vo[vi + nx] = V0[vo_s + kVW] + zero_term;
            if (z == nz - 1) a.wo[wi + pl] = (&S.w[sp][0][0])[wo_s] + zero_term;
        }
    }
}

int launch_vorticity(ss_sim* s, const StepConsts& c, cudaStream_t st) {
    FluidArgs a = fluid_args(s, c);
    a.c.vort_k = s->h;
    dim3 b(32, 8, 1);
    dim3 gc = grid_for(s->nx, s->ny, s->nz, b);
    dim3 gf = grid_for(s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1, b);
    if (s->dim == 3) {
        const int tx = (s->nx + kMX - 1) / kMX, ty = (s->ny + kMY - 1) / kMY;
        const int planes = z_planes((long long)tx * ty, s->nz, kMZ, 4);
        dim3 gt(tx, ty, (s->nz + planes - 1) / planes);
        const float two_h = 2.f * s->h;
        if (pow2_normal(two_h) && pow2_normal(c.rho))
            k_vorticity_march<true><<<gt, kMT, 0, st>>>(a, 1.f / two_h, 1.f / c.rho, planes);
        else
            k_vorticity_march<false><<<gt, kMT, 0, st>>>(a, 0.f, 0.f, planes);
        s->nlaunch += 1;
    } else {
        k_vorticity<2><<<gc, b, 0, st>>>(a, s->vort);
        k_apply_vorticity<2><<<gf, b, 0, st>>>(a, s->vort);
        s->nlaunch += 2;
    }
    for (int d = 0; d < s->dim; ++d) s->vi[d] ^= 1;
    return check_cuda(cudaGetLastError(), "vorticity confinement");
}

// the vorticity of the given velocities into out (3 planes in 3D, plus |w|):
// what the adjoint of vorticity confinement reads
int launch_vorticity_field(ss_sim* s, const StepConsts& c, const float* const vel[3], float* out, cudaStream_t st) {
    FluidArgs a = fluid_args(s, c);
    a.u = vel[0]; a.v = vel[1]; a.w = s->dim == 3 ? vel[2] : nullptr;
    a.c.vort_k = s->h;
    dim3 b(32, 8, 1);
    dim3 gc = grid_for(s->nx, s->ny, s->nz, b);
    if (s->dim == 3) k_vorticity<3><<<gc, b, 0, st>>>(a, out);
    else k_vorticity<2><<<gc, b, 0, st>>>(a, out);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_vorticity");
}

// -------------------------------------------------------- projection update
// update_vx/vy/vz (shaders3d/compute/update_vx.comp:45-62 and siblings; 2D
// :43-60): faces touching solid (out of grid = fluid) take the solid map's
// velocity of cell idx (0 outside the grid).
// P = double: the mixed-precision solve's FP64 pressure; the face update is
// then evaluated in FP64 (k64 = -dt/(rho h)) and rounded once to FP32.
// Each thread takes kUpdPlanes face positions up z; the pressure and solid
// flag of the cell below (z-1) carry over from the previous plane.
constexpr int kUpdPlanes = 8;

// p0_out (FP64 pressure only): also store each cell's pressure rounded to
// FP32 - the pressure field of the API - in the same pass.
template <int DIM, typename P = float>
__global__ void __launch_bounds__(256) k_update_velocity(FluidArgs a, const P* __restrict__ p, int planes,
                                                         double k64 = 0.0, float* __restrict__ p0_out = nullptr) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int zb = blockIdx.z * planes;
    const int zend = min(zb + planes, DIM == 3 ? nz + 1 : 1);
    const bool inxy = x < nx && y < ny;
    P p_back = P(0);
    bool s_back = false;
    if (DIM == 3 && inxy && zb > 0) {
        p_back = __ldg(p + idx3(x, y, zb - 1, nx, ny));
        s_back = a.flags[idx3(x, y, zb - 1, nx, ny)] & F_SOLID;
    }
    // a plane's loads, issued one plane ahead so they are in flight across
    // the plane before: the cell's pressure and solid flag, and per x / y face
    // the face velocity and the lower cell's pressure and flag (z faces take
    // the lower cell from the previous plane); every address is in range
    struct Plane {
        P pc, plo[2];
        float src[3];
        bool sc, slo[2];
    };
    auto fetch = [&](int z, Plane& L) {
        const bool in = inxy && z < nz;
        L.pc = in ? __ldg(p + idx3(x, y, z, nx, ny)) : P(0);
        L.sc = in && (a.flags[idx3(x, y, z, nx, ny)] & F_SOLID);
#pragma unroll
        for (int comp = 0; comp < DIM; ++comp) {
            const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
            L.src[comp] = 0.f;
            if (comp < 2) { L.plo[comp] = P(0); L.slo[comp] = false; }
            if (x >= ax || y >= ay || z >= az) continue;
            const float* __restrict__ src = comp == 0 ? a.u : comp == 1 ? a.v : a.w;
            L.src[comp] = __ldg(src + idx3(x, y, z, ax, ay));
            if (comp < 2) {
                const int xm = x - (comp == 0), ym = y - (comp == 1);
                L.slo[comp] = solid_oob0(a.flags, xm, ym, z, nx, ny, nz);
                L.plo[comp] = (xm < 0 || ym < 0) ? P(0) : __ldg(p + idx3(xm, ym, z, nx, ny));
            }
        }
    };
    Plane cur;
    fetch(zb, cur);
    for (int z = zb; z < zend; ++z) {
        Plane nxt = cur;
        if (z + 1 < zend) fetch(z + 1, nxt);
        const bool in = inxy && z < nz;
        const P pc = cur.pc;
        const bool sc = cur.sc;
        if (p0_out && in) p0_out[idx3(x, y, z, nx, ny)] = (float)pc;
#pragma unroll
        for (int comp = 0; comp < DIM; ++comp) {
            const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
            if (x >= ax || y >= ay || z >= az) continue;
            float* __restrict__ dst = comp == 0 ? a.uo : comp == 1 ? a.vo : a.wo;
            const int i = idx3(x, y, z, ax, ay);
            const bool s_lo = comp == 2 ? s_back : cur.slo[comp < 2 ? comp : 0];
            if (sc || s_lo) {
                const float* sv = comp == 0 ? a.sv0 : comp == 1 ? a.sv1 : a.sv2;
                dst[i] = (in && sv) ? sv[idx3(x, y, z, nx, ny)] : 0.f;
                continue;
            }
            const P plo = comp == 2 ? p_back : cur.plo[comp < 2 ? comp : 0];
            if constexpr (std::is_same<P, double>::value) dst[i] = (float)((double)cur.src[comp] + k64 * (pc - plo));
            else dst[i] = cur.src[comp] + a.c.k_upd * (pc - plo);
        }
        p_back = pc;
        s_back = sc;
        cur = nxt;
    }
}

int launch_update_velocities(ss_sim* s, const StepConsts& c, cudaStream_t st) {
    FluidArgs a = fluid_args(s, c);
    dim3 b(32, 8, 1);
    const int planes = z_planes((long long)((s->nx + 32) / 32) * ((s->ny + 8) / 8), s->nz + 1, kUpdPlanes);
    dim3 g = grid_for(s->nx + 1, s->ny + 1, s->dim == 3 ? (s->nz + planes) / planes : 1, b);
    if (s->dim == 3) k_update_velocity<3><<<g, b, 0, st>>>(a, s->p[0], planes);
    else k_update_velocity<2><<<g, b, 0, st>>>(a, s->p[0], planes);
    for (int d = 0; d < s->dim; ++d) s->vi[d] ^= 1;
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_update_velocity");
}

int launch_update_velocities_p64(ss_sim* s, const StepConsts& c, cudaStream_t st, float* p0_out) {
    FluidArgs a = fluid_args(s, c);
    dim3 b(32, 8, 1);
    const int planes = z_planes((long long)((s->nx + 32) / 32) * ((s->ny + 8) / 8), s->nz + 1, kUpdPlanes);
    dim3 g = grid_for(s->nx + 1, s->ny + 1, s->dim == 3 ? (s->nz + planes) / planes : 1, b);
    const double k64 = -(double)c.dt / ((double)c.rho * (double)s->h);
    if (s->dim == 3) k_update_velocity<3, double><<<g, b, 0, st>>>(a, s->p64, planes, k64, p0_out);
    else k_update_velocity<2, double><<<g, b, 0, st>>>(a, s->p64, planes, k64, p0_out);
    for (int d = 0; d < s->dim; ++d) s->vi[d] ^= 1;
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_update_velocity<p64>");
}

// ------------------------------------------------------------ smoke advection
// advect_smoke (shaders3d/compute/advect_smoke.comp:55-72; 2D :51-68).
// A thread takes kSmokePlanes cells up z (fewer, longer-lived blocks).
// With DIV the kernel also folds the squared divergence of the velocities it
// advects with - the projected velocities - into the statistics slot `slot`
// (the operator of k_divergence below, from the six faces already loaded
// here); the last block to finish sums the blocks' partials in a fixed order.
constexpr int kSmokePlanes = 4;
SS_D double block_sum(double v);

struct DivFold {
    double* partial;
    unsigned int* ticket;
    double* out;
    int slot;
};

template <int DIM, bool DIV>
__global__ void __launch_bounds__(256) k_advect_smoke(FluidArgs a, DivFold df, int planes) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int zb = blockIdx.z * planes, ze = min(zb + planes, nz);
    const size_t ncell = (size_t)nx * ny * nz;
    double acc = 0.0;
    // linear indices in the x-y plane; a plane adds pl (cells, w), plu (u), plv (v)
    const int pl = nx * ny, plu = (nx + 1) * ny, plv = nx * (ny + 1);
    const int cxy = y * nx + x, uxy = y * (nx + 1) + x;
    for (int z = zb; z < ze && x < nx && y < ny; ++z) {
        const int c = z * pl + cxy;
        const int iu = z * plu + uxy, iv = z * plv + cxy;
        // the cell's faces always exist: loaded before the solid test
        const float f_left = __ldg(a.u + iu), f_right = __ldg(a.u + iu + 1);
        const float f_bottom = __ldg(a.v + iv), f_top = __ldg(a.v + iv + nx);
        float f_back = 0.f, f_front = 0.f;
        if constexpr (DIM == 3) {
            f_back = __ldg(a.w + c);
            f_front = __ldg(a.w + c + pl);
        }
        // vel_at_centre's values
        const float vel[3] = {lerp_(f_left, f_right, 0.5f), lerp_(f_bottom, f_top, 0.5f),
                              DIM == 3 ? lerp_(f_back, f_front, 0.5f) : 0.f};
        const uint8_t fl = a.flags[c];
        if (fl & F_SOLID) {
            for (int ch = 0; ch < a.nch; ++ch) a.dens_o[ch * ncell + c] = 0.f;
            a.temp_o[c] = a.c.t_amb;
            continue;
        }
        if constexpr (DIV) {
            if (!(fl & 0x7Eu)) {
                // no face borders a solid: the faces as loaded, the same operations
                float d = f_right - f_left + f_top - f_bottom;
                if constexpr (DIM == 3) d = d + f_front - f_back;
                acc += (double)d * (double)d;
            } else {
                const bool sv = a.sv0 != nullptr;
                const float v_top = (fl & F_TOP) ? (sv ? a.sv1[c + nx] : 0.f) : f_top;
                const float v_bottom = (fl & F_BOTTOM) ? (sv ? a.sv1[c - nx] : 0.f) : f_bottom;
                const float v_right = (fl & F_RIGHT) ? (sv ? a.sv0[c + 1] : 0.f) : f_right;
                const float v_left = (fl & F_LEFT) ? (sv ? a.sv0[c - 1] : 0.f) : f_left;
                float d = v_right - v_left + v_top - v_bottom;
                if constexpr (DIM == 3) {
                    const float v_front = (fl & F_FRONT) ? (sv ? a.sv2[c + pl] : 0.f) : f_front;
                    const float v_back = (fl & F_BACK) ? (sv ? a.sv2[c - pl] : 0.f) : f_back;
                    d = d + v_front - v_back;
                }
                acc += (double)d * (double)d;
            }
        }
        const float gx = (float)x + 0.5f, gy = (float)y + 0.5f, gz = DIM == 3 ? (float)z + 0.5f : 0.f;
        const float cfl = a.c.cfl;
        const float bx = gx - vel[0] * cfl, by = gy - vel[1] * cfl, bz = gz - vel[2] * cfl;
        const Taps t = make_taps<DIM>(nx, ny, nz, bx - 0.5f, by - 0.5f, bz - 0.5f);
        // sample_taps_fast's values, its range test and base index formed once
        // for every channel
        const bool tin = t.x0 >= 0 && t.x0 + 1 < nx && t.y0 >= 0 && t.y0 + 1 < ny &&
                         (DIM == 2 || (t.z0 >= 0 && t.z0 + 1 < nz));
        const int tb = tin ? idx3(t.x0, t.y0, t.z0, nx, ny) : 0;
        auto sample = [&](const float* __restrict__ f, float border) -> float {
            if (!tin) return sample_taps<DIM>(f, nx, ny, nz, t, border);
            const float* q = f + tb;
            const float c00 = __ldg(q), c10 = __ldg(q + 1), c01 = __ldg(q + nx), c11 = __ldg(q + nx + 1);
            if constexpr (DIM == 2) {
                return lerp_(lerp_(c00, c10, t.wx), lerp_(c01, c11, t.wx), t.wy);
            } else {
                const float d00 = __ldg(q + pl), d10 = __ldg(q + pl + 1), d01 = __ldg(q + pl + nx),
                            d11 = __ldg(q + pl + nx + 1);
                const float c0 = lerp_(lerp_(c00, c10, t.wx), lerp_(c01, c11, t.wx), t.wy);
                const float c1 = lerp_(lerp_(d00, d10, t.wx), lerp_(d01, d11, t.wx), t.wy);
                return lerp_(c0, c1, t.wz);
            }
        };
        for (int ch = 0; ch < a.nch; ++ch) a.dens_o[ch * ncell + c] = sample(a.dens + ch * ncell, 0.f);
        a.temp_o[c] = sample(a.temp, a.c.t_amb);
    }
    if constexpr (DIV) {
        const double bs = block_sum(acc);
        const int tid = threadIdx.x + blockDim.x * threadIdx.y;
        const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
        __shared__ bool last;
        if (tid == 0) {
            df.partial[bid] = bs;
            __threadfence();
            last = atomicAdd(df.ticket, 1u) == nb - 1;
        }
        __syncthreads();
        if (!last) return;
        const double total = block_sum(fold_sum(df.partial, nb, tid, blockDim.x * blockDim.y));
        if (tid == 0) {
            df.out[df.slot] = total;
            *df.ticket = 0u;
        }
    }
}

int launch_advect_smoke(ss_sim* s, const StepConsts& c, cudaStream_t st, int div_slot) {
    FluidArgs a = fluid_args(s, c);
    dim3 b(32, 8, 1);
    // the divergence fold ends each block with a reduction: twice the planes
    // a thread spread its barrier over twice the cells
    const int planes = z_planes((long long)((s->nx + 31) / 32) * ((s->ny + 7) / 8), s->nz,
                                div_slot >= 0 ? 2 * kSmokePlanes : kSmokePlanes);
    dim3 g = grid_for(s->nx, s->ny, (s->nz + planes - 1) / planes, b);
    DivFold df{s->red.partial, s->red.ticket, s->red.out, div_slot};
    if (div_slot >= 0 && (int)(g.x * g.y * g.z) > s->red.max_blocks)
        return set_error(SS_E_INVALID, "reduction scratch too small");
    if (s->dim == 3) {
        if (div_slot >= 0) k_advect_smoke<3, true><<<g, b, 0, st>>>(a, df, planes);
        else k_advect_smoke<3, false><<<g, b, 0, st>>>(a, df, planes);
    } else {
        if (div_slot >= 0) k_advect_smoke<2, true><<<g, b, 0, st>>>(a, df, planes);
        else k_advect_smoke<2, false><<<g, b, 0, st>>>(a, df, planes);
    }
    s->si ^= 1;
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_advect_smoke");
}

// ---------------------------------------------------------------- divergence
// Level-0 divergence with solid-velocity substitution, the delta_v of
// smooth.comp:105-113 (out of grid = fluid) and, for open domains, of
// compute_residual.comp:116-124 (out of grid = solid, velocity 0).  Optional
// FP64 sum of squares over fluid cells into per-block partials.
SS_D double block_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __shared__ double warp_part[32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    if ((tid & 31) == 0) warp_part[tid >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (tid < 32) {
        r = tid < (nthreads + 31) / 32 ? warp_part[tid] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

// position of cell (x,y,z) in the colour-split level-0 arrays (k_rb.cu): the
// colour-(x+y+z)&1 half, row-major with nx/2 entries per row (nx even)
SS_D int rb_slot(int x, int y, int z, int nx, int ny, int nz) {
    const int half = nx >> 1;
    return (((x + y + z) & 1) ? half * ny * nz : 0) + (z * ny + y) * half + (x >> 1);
}

// Optional level-0 right-hand sides of the pressure operators, computed once
// per solve with the operations the reference evaluates in every sweep:
// rhs_s = rho*h*div/dt (smooth.comp:129), rhs_r = rho*div/(dt*h)
// (compute_residual.comp:124), each with its out-of-grid rule, stored
// colour-split for the level-0 kernels of k_rb.cu.
struct RhsOut {
    float* rhs_s;
    float* rhs_r;
    float rho_h, dt, rho, dt_h;
    int s_solid, r_solid;   // out-of-grid neighbours count as solid in the smoother / residual
};

// Each thread takes kDivPlanes cells up z (the face between two of them is
// loaded once), so a block reduces up to 256 * kDivPlanes cells.
constexpr int kDivPlanes = 8;

// ep / eq (optional): the mixed solve's extrapolated warm start, elementwise
// over the same cells (ep = 2 ep - eq in FP64, eq = the old ep), riding on this
// pass, whose own traffic leaves HBM bandwidth to spare.
template <int DIM>
__global__ void __launch_bounds__(256) k_divergence(FluidArgs a, float* __restrict__ div0, float* __restrict__ div0r,
                                                    double* __restrict__ partial, RhsOut ro, int planes,
                                                    double* __restrict__ ep, double* __restrict__ eq) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int zb = blockIdx.z * planes;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    double acc = 0.0;
    if (x < nx && y < ny) {
        const int ze = min(zb + planes, nz);
        float f_back = 0.f;
        if constexpr (DIM == 3) f_back = __ldg(a.w + idx3(x, y, zb, nx, ny));
        // the cell's six faces always exist: a plane's five new faces and its
        // flag are loaded one plane ahead, in flight across the plane before
        struct Faces {
            float t, b, r, l, f;
            uint8_t fl;
            double ep, eq;
        };
        auto fetch = [&](int z, Faces& F) {
            F.t = __ldg(a.v + idx3(x, y + 1, z, nx, ny + 1));
            F.b = __ldg(a.v + idx3(x, y, z, nx, ny + 1));
            F.r = __ldg(a.u + idx3(x + 1, y, z, nx + 1, ny));
            F.l = __ldg(a.u + idx3(x, y, z, nx + 1, ny));
            F.f = DIM == 3 ? __ldg(a.w + idx3(x, y, z + 1, nx, ny)) : 0.f;
            F.fl = __ldg(a.flags + idx3(x, y, z, nx, ny));
            if (ep) {
                F.ep = ep[idx3(x, y, z, nx, ny)];
                F.eq = eq[idx3(x, y, z, nx, ny)];
            }
        };
        Faces cur;
        fetch(zb, cur);
        for (int z = zb; z < ze; ++z) {
            const int c = idx3(x, y, z, nx, ny);
            Faces nxt = cur;
            if (z + 1 < ze) fetch(z + 1, nxt);
            const float f_top = cur.t, f_bottom = cur.b, f_right = cur.r, f_left = cur.l, f_front = cur.f;
            const uint8_t fl = cur.fl;
            if (ep) {
                ep[c] = 2.0 * cur.ep - cur.eq;
                eq[c] = cur.ep;
            }
            cur = nxt;
            if (!(fl & F_SOLID)) {
                const bool sv = a.sv0 != nullptr;
                const float v_top = (fl & F_TOP) ? (sv ? a.sv1[c + nx] : 0.f) : f_top;
                const float v_bottom = (fl & F_BOTTOM) ? (sv ? a.sv1[c - nx] : 0.f) : f_bottom;
                const float v_right = (fl & F_RIGHT) ? (sv ? a.sv0[c + 1] : 0.f) : f_right;
                const float v_left = (fl & F_LEFT) ? (sv ? a.sv0[c - 1] : 0.f) : f_left;
                float d = v_right - v_left + v_top - v_bottom;
                float v_front = 0.f, v_back = 0.f;
                if constexpr (DIM == 3) {
                    const int pl = nx * ny;
                    v_front = (fl & F_FRONT) ? (sv ? a.sv2[c + pl] : 0.f) : f_front;
                    v_back = (fl & F_BACK) ? (sv ? a.sv2[c - pl] : 0.f) : f_back;
                    d = d + v_front - v_back;
                }
                if (div0) div0[c] = d;
                if (div0r || ro.rhs_s) {
                    // residual rule: out-of-grid neighbours are solid with velocity 0
                    const float rt = y + 1 >= ny ? 0.f : v_top, rb = y == 0 ? 0.f : v_bottom;
                    const float rr = x + 1 >= nx ? 0.f : v_right, rl = x == 0 ? 0.f : v_left;
                    float dr = rr - rl + rt - rb;
                    if constexpr (DIM == 3) {
                        const float rf = z + 1 >= nz ? 0.f : v_front, rk = z == 0 ? 0.f : v_back;
                        dr = dr + rf - rk;
                    }
                    if (div0r) div0r[c] = dr;
                    if (ro.rhs_s) {
                        const int q = rb_slot(x, y, z, nx, ny, nz);
                        ro.rhs_s[q] = ro.rho_h * (ro.s_solid ? dr : d) / ro.dt;
                        ro.rhs_r[q] = ro.rho * (ro.r_solid ? dr : d) / ro.dt_h;
                    }
                }
                acc += (double)d * (double)d;
            } else if (ro.rhs_s) {
                const int q = rb_slot(x, y, z, nx, ny, nz);
                ro.rhs_s[q] = 0.f;
                ro.rhs_r[q] = 0.f;
            }
            f_back = f_front;
        }
    }
    if (partial) {
        const double bs = block_sum(acc);
        if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0)
            partial[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = bs;
    }
}

int launch_divergence(ss_sim* s, bool write, int slot, cudaStream_t st, const StepConsts* sc, int quirks,
                      double* ep, double* eq) {
    StepConsts c{};
    FluidArgs a = fluid_args(s, c);
    RhsOut ro{};
    if (write && sc && quirks >= 0 && rb_supported(s, quirks)) {
        ro.rhs_s = s->rhs_s;
        ro.rhs_r = s->rhs_r;
        s->rhs_r_is_s = 0;   // both forms written, each with its own out-of-grid rule
        ro.rho_h = sc->rho_h; ro.dt = sc->dt; ro.rho = sc->rho; ro.dt_h = sc->dt_h;
        ro.s_solid = quirks ? 0 : s->enclosed;
        ro.r_solid = quirks ? 1 : s->enclosed;
    }
    dim3 b(32, 8, 1);
    const int planes = z_planes((long long)((s->nx + 31) / 32) * ((s->ny + 7) / 8), s->nz, kDivPlanes);
    dim3 g = grid_for(s->nx, s->ny, (s->nz + planes - 1) / planes, b);
    const int nblocks = (int)(g.x * g.y * g.z);
    float* d0 = write ? s->div0 : nullptr;
    float* d0r = (write && s->div0r != s->div0) ? s->div0r : nullptr;
    double* part = slot >= 0 ? s->red.partial : nullptr;
    if ((ep == nullptr) != (eq == nullptr)) return set_error(SS_E_INVALID, "extrapolation needs both buffers");
    if (s->dim == 3) k_divergence<3><<<g, b, 0, st>>>(a, d0, d0r, part, ro, planes, ep, eq);
    else k_divergence<2><<<g, b, 0, st>>>(a, d0, d0r, part, ro, planes, ep, eq);
    s->nlaunch += 1;
    int rc = check_cuda(cudaGetLastError(), "k_divergence");
    if (rc || slot < 0) return rc;
    return launch_reduce_final(s, nblocks, slot, st);
}

// Fixed-order final sum of the per-block partials (deterministic).
__global__ void k_reduce_final(const double* __restrict__ partial, int n, double* __restrict__ out, int slot) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    __shared__ double sh[1024];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[slot] = sh[0];
}

// Sum (or maximum) of each group of 1024 consecutive partials, in a fixed
// order: the single block that finishes a reduction then reads one value per
// group instead of walking every partial in a long dependent chain.
template <bool MAX>
__global__ void __launch_bounds__(256) k_reduce_stage(const double* __restrict__ in, int n, double* __restrict__ out) {
    __shared__ double sh[256];
    const int base = blockIdx.x * 1024;
    double a = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = base + threadIdx.x + 256 * j;
        if (i < n) a = MAX ? fmax(a, in[i]) : a + in[i];
    }
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] = MAX ? fmax(sh[threadIdx.x], sh[threadIdx.x + o]) : sh[threadIdx.x] + sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

int reduce_stage1(ss_sim* s, const double* in, int n, bool is_max, const double** res, int* nres, cudaStream_t st) {
    if (n <= 1024) {
        *res = in;
        *nres = n;
        return SS_OK;
    }
    const int nb = (n + 1023) / 1024;
    if (nb > s->red.stage2) return set_error(SS_E_INVALID, "reduction scratch too small");
    double* out = s->red.partial2 + (is_max ? s->red.stage2 : 0);
    if (is_max) k_reduce_stage<true><<<nb, 256, 0, st>>>(in, n, out);
    else k_reduce_stage<false><<<nb, 256, 0, st>>>(in, n, out);
    s->nlaunch += 1;
    *res = out;
    *nres = nb;
    return check_cuda(cudaGetLastError(), "k_reduce_stage");
}

int launch_reduce_final(ss_sim* s, int nblocks, int slot, cudaStream_t st) {
    const double* in;
    int n;
    int rc = reduce_stage1(s, s->red.partial, nblocks, false, &in, &n, st);
    if (rc) return rc;
    k_reduce_final<<<1, 1024, 0, st>>>(in, n, s->red.out, slot);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_reduce_final");
}

}  // namespace ss
