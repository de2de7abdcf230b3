// k_adjoint.cu - hand-written adjoints (transposes) of the step's stages.
//
// Each kernel here is the transpose of one forward kernel of k_fluid.cu /
// k_mg.cu / k_rb.cu for the same inputs: it maps the adjoint of the stage's
// output to the adjoint of its input, evaluated at the forward state the
// stage saw (semi-Lagrangian advection and vorticity confinement are
// nonlinear; the rest are linear).  No counterpart in the reference, which has
// no derivatives; the forward operators they transpose are restatements of
// its shaders (cited at the forward kernels).
//
//  - advection: the trilinear gather becomes a scatter-add into the advected
//    array (atomicAdd, warp-aggregated along x for the smoke; or the
//    deterministic owner-computes gather below), plus the chain rule through
//    the back-traced point into the velocity that traced it;
//  - buoyancy: a 2-tap average per y face, transposed into the two cells;
//  - vorticity confinement: f = N x w with N = grad|w| / (|grad|w|| + 1e-20),
//    w = curl of the cell-centred velocity; its Jacobian-transpose in three
//    passes (force -> w and grad|w|, grad|w| -> |w| -> w, w -> faces);
//  - projection: the update's pressure gradient transposes into a
//    divergence-like gather; each V-cycle of the fixed schedule is transposed
//    operator by operator (red-black colour updates in reverse order,
//    residual + restriction, prolongation), and the right-hand side's
//    divergence into a face scatter.
#include "common.cuh"
#include "ss_internal.h"

namespace ss {

static inline dim3 grid_of(int ax, int ay, int az, dim3 b) {
    return dim3((ax + b.x - 1) / b.x, (ay + b.y - 1) / b.y, (az + b.z - 1) / b.z);
}

SS_D bool in3(int x, int y, int z, int ax, int ay, int az) {
    return x >= 0 && y >= 0 && z >= 0 && x < ax && y < ay && z < az;
}
SS_D bool solid1(const uint8_t* f, int x, int y, int z, int nx, int ny, int nz) {   // out of grid = solid
    if (!in3(x, y, z, nx, ny, nz)) return true;
    return f[idx3(x, y, z, nx, ny)] & F_SOLID;
}
SS_D bool solid0(const uint8_t* f, int x, int y, int z, int nx, int ny, int nz) {   // out of grid = fluid
    if (!in3(x, y, z, nx, ny, nz)) return false;
    return f[idx3(x, y, z, nx, ny)] & F_SOLID;
}
SS_D void scatter(float* a, int ax, int ay, int az, int x, int y, int z, float v) {
    if (in3(x, y, z, ax, ay, az) && v != 0.f) atomicAdd(a + idx3(x, y, z, ax, ay), v);
}

// Adjoint of one border-filtered trilinear sample with taps t: scatters
// g * weight into abar at the in-range taps and returns d(sample)/d(w) per
// axis in dw (tap values outside the array read `border`).
template <int DIM>
SS_D void adj_sample(const float* __restrict__ a, float* __restrict__ abar, int ax, int ay, int az, const Taps& t,
                     float border, float g, float dw[3]) {
    const int x0 = t.x0, y0 = t.y0, z0 = t.z0;
    const float wx = t.wx, wy = t.wy, wz = t.wz;
    if constexpr (DIM == 2) {
        const float c00 = fetch_b(a, ax, ay, 1, x0, y0, 0, border), c10 = fetch_b(a, ax, ay, 1, x0 + 1, y0, 0, border);
        const float c01 = fetch_b(a, ax, ay, 1, x0, y0 + 1, 0, border), c11 = fetch_b(a, ax, ay, 1, x0 + 1, y0 + 1, 0, border);
        dw[0] = (1.f - wy) * (c10 - c00) + wy * (c11 - c01);
        dw[1] = lerp_(c01, c11, wx) - lerp_(c00, c10, wx);
        dw[2] = 0.f;
        if (abar) {
            scatter(abar, ax, ay, 1, x0, y0, 0, g * (1.f - wx) * (1.f - wy));
            scatter(abar, ax, ay, 1, x0 + 1, y0, 0, g * wx * (1.f - wy));
            scatter(abar, ax, ay, 1, x0, y0 + 1, 0, g * (1.f - wx) * wy);
            scatter(abar, ax, ay, 1, x0 + 1, y0 + 1, 0, g * wx * wy);
        }
    } else {
        float c[2][2][2];
#pragma unroll
        for (int k = 0; k < 2; ++k)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int i = 0; i < 2; ++i) c[k][j][i] = fetch_b(a, ax, ay, az, x0 + i, y0 + j, z0 + k, border);
        const float e0 = (1.f - wy) * (c[0][0][1] - c[0][0][0]) + wy * (c[0][1][1] - c[0][1][0]);
        const float e1 = (1.f - wy) * (c[1][0][1] - c[1][0][0]) + wy * (c[1][1][1] - c[1][1][0]);
        dw[0] = (1.f - wz) * e0 + wz * e1;
        const float f0 = lerp_(c[0][1][0], c[0][1][1], wx) - lerp_(c[0][0][0], c[0][0][1], wx);
        const float f1 = lerp_(c[1][1][0], c[1][1][1], wx) - lerp_(c[1][0][0], c[1][0][1], wx);
        dw[1] = (1.f - wz) * f0 + wz * f1;
        const float s0 = lerp_(lerp_(c[0][0][0], c[0][0][1], wx), lerp_(c[0][1][0], c[0][1][1], wx), wy);
        const float s1 = lerp_(lerp_(c[1][0][0], c[1][0][1], wx), lerp_(c[1][1][0], c[1][1][1], wx), wy);
        dw[2] = s1 - s0;
        if (abar) {
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int j = 0; j < 2; ++j)
#pragma unroll
                    for (int i = 0; i < 2; ++i) {
                        const float w = (i ? wx : 1.f - wx) * (j ? wy : 1.f - wy) * (k ? wz : 1.f - wz);
                        scatter(abar, ax, ay, az, x0 + i, y0 + j, z0 + k, g * w);
                    }
        }
    }
}

// d(tap weight)/d(texel coordinate): 1 inside the clamp range, 0 where
// make_taps clamped the coordinate
SS_D float clamp_grad(float t, int a) { return (t > -2.f && t < (float)(a + 1)) ? 1.f : 0.f; }

struct AdjFluid {
    int nx, ny, nz, nch;
    const float* u;   // forward velocity the stage read
    const float* v;
    const float* w;
    const uint8_t* flags;
    const float* dens;   // forward smoke the stage read
    const float* temp;
    StepConsts c;
};

// --------------------------------------------------------- smoke advection^T
// Forward (k_advect_smoke): out(c) = sample(in, centre(c) - cfl * vel_centre(c)),
// solid cells set to (0, t_amb).  Adjoint: scatter into din/tin, and the
// position gradient into a per-cell velocity adjoint (vcb, 3 arrays), spread to
// the faces by k_adj_centre_to_faces.
// Per-cell part, shared with the owner-computes trace pass: the position
// gradient vb, the back-traced point clamped as make_taps clamps it (tc), and,
// when din / tin are given, the scatter of the adjoints into them.  Returns
// false for a solid cell, which scatters nothing.
template <int DIM>
SS_D bool smoke_cell_adj(const AdjFluid& a, int x, int y, int z, const float* __restrict__ dout,
                         const float* __restrict__ tout, float* din, float* tin, float vb[3], float tc[3]) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int c = idx3(x, y, z, nx, ny);
    const size_t ncell = (size_t)nx * ny * nz;
    vb[0] = vb[1] = vb[2] = 0.f;
    if (a.flags[c] & F_SOLID) return false;
    float vel[3];
    vel_at_centre<DIM>(a.u, a.v, a.w, nx, ny, nz, x, y, z, vel);
    const float cfl = a.c.cfl;
    const float gx = (float)x + 0.5f, gy = (float)y + 0.5f, gz = DIM == 3 ? (float)z + 0.5f : 0.f;
    const float tx = gx - vel[0] * cfl - 0.5f, ty = gy - vel[1] * cfl - 0.5f, tz = gz - vel[2] * cfl - 0.5f;
    const Taps t = make_taps<DIM>(nx, ny, nz, tx, ty, tz);
    float bb[3] = {0.f, 0.f, 0.f};
    float dw[3];
    for (int ch = 0; ch <= a.nch; ++ch) {
        const bool is_t = ch == a.nch;
        const float g = is_t ? tout[c] : dout[ch * ncell + c];
        if (g == 0.f) continue;
        const float* src = is_t ? a.temp : a.dens + ch * ncell;
        float* dst = din ? (is_t ? tin : din + ch * ncell) : nullptr;
        adj_sample<DIM>(src, dst, nx, ny, nz, t, is_t ? a.c.t_amb : 0.f, g, dw);
        bb[0] += g * dw[0];
        bb[1] += g * dw[1];
        bb[2] += g * dw[2];
    }
    vb[0] = -cfl * bb[0] * clamp_grad(tx, nx);
    vb[1] = -cfl * bb[1] * clamp_grad(ty, ny);
    vb[2] = DIM == 3 ? -cfl * bb[2] * clamp_grad(tz, nz) : 0.f;
    tc[0] = clampt(tx, -2.f, (float)(nx + 1));
    tc[1] = clampt(ty, -2.f, (float)(ny + 1));
    tc[2] = DIM == 3 ? clampt(tz, -2.f, (float)(nz + 1)) : 0.f;
    return true;
}

// Warp-aggregated scatter of one tap row: c0 into (x0, y, z), c1 into
// (x0 + 1, y, z).  The 32 lanes of a warp hold consecutive x of one row, so a
// lane's x0 + 1 is usually the next lane's x0: that lane then adds the
// previous lane's c1 to its own c0 and one atomic serves both.  The merge
// decision (row_merge, from the lanes' packed tap coordinates; key < 0: no
// sample) is shared by every array scattered through the same taps; every
// lane of the warp makes both calls.
struct RowMerge {
    bool take, given;
};
SS_D long long row_key(bool live, int x0, int y, int z) {
    return live ? (((long long)(z + 2) << 42) | ((long long)(y + 2) << 21) | (long long)(x0 + 2)) : -1;
}
SS_D RowMerge row_merge(long long key) {
    const int lane = threadIdx.x & 31;
    const long long pk = __shfl_up_sync(0xffffffffu, key, 1);
    RowMerge m;
    m.take = lane > 0 && key >= 0 && pk >= 0 && pk + 1 == key;
    m.given = __shfl_down_sync(0xffffffffu, (int)m.take, 1) != 0 && lane < 31;
    return m;
}
SS_D void row_scatter(float* a, int ax, int ay, int az, int x0, int y, int z, float c0, float c1, bool live,
                      const RowMerge& m) {
    const float pc1 = __shfl_up_sync(0xffffffffu, c1, 1);
    if (m.take) c0 += pc1;
    if (live) {
        scatter(a, ax, ay, az, x0, y, z, c0);
        if (!m.given) scatter(a, ax, ay, az, x0 + 1, y, z, c1);
    }
}

// Atomic variant: the per-cell part without its scatter, then the samples'
// adjoints of every channel through warp-aggregated tap rows (blocks of 32
// lanes along x; no early exit, every lane takes part in the shuffles).
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_advect_smoke(AdjFluid a, const float* __restrict__ dout, const float* __restrict__ tout,
                                                          float* __restrict__ din, float* __restrict__ tin,
                                                          float* __restrict__ vcb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const bool in = x < nx && y < ny && z < nz;
    const int c = in ? idx3(x, y, z, nx, ny) : 0;
    const size_t ncell = (size_t)nx * ny * nz;
    float vb[3] = {0.f, 0.f, 0.f}, tc[3] = {0.f, 0.f, 0.f};
    const bool live = in && smoke_cell_adj<DIM>(a, x, y, z, dout, tout, nullptr, nullptr, vb, tc);
    if (in) {
        vcb[c] = vb[0];
        vcb[ncell + c] = vb[1];
        if (DIM == 3) vcb[2 * ncell + c] = vb[2];
    }
    const float fx = floorf(tc[0]), fy = floorf(tc[1]), fz = DIM == 3 ? floorf(tc[2]) : 0.f;
    const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
    const float wx = tc[0] - fx, wy = tc[1] - fy, wz = tc[2] - fz;
    constexpr int KZ = DIM == 3 ? 2 : 1;
    RowMerge m[KZ][2];
#pragma unroll
    for (int k = 0; k < KZ; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j) m[k][j] = row_merge(row_key(live, x0, y0 + j, z0 + k));
    for (int ch = 0; ch <= a.nch; ++ch) {
        const bool is_t = ch == a.nch;
        const float g = live ? (is_t ? tout[c] : dout[ch * ncell + c]) : 0.f;
        float* dst = is_t ? tin : din + ch * ncell;
#pragma unroll
        for (int k = 0; k < KZ; ++k)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                float c0, c1;
                if constexpr (DIM == 3) {
                    const float wyz = j ? wy : 1.f - wy, wzk = k ? wz : 1.f - wz;
                    c0 = g * ((1.f - wx) * wyz * wzk);
                    c1 = g * (wx * wyz * wzk);
                } else {
                    c0 = g * (1.f - wx) * (j ? wy : 1.f - wy);
                    c1 = g * wx * (j ? wy : 1.f - wy);
                }
                row_scatter(dst, nx, ny, DIM == 3 ? nz : 1, x0, y0 + j, z0 + k, c0, c1, live, m[k][j]);
            }
    }
}

// faces += 0.5 * (per-cell velocity adjoint of the two cells sharing the face)
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_centre_to_faces(const float* __restrict__ vcb, int nx, int ny, int nz,
                                                             float* __restrict__ ub, float* __restrict__ vbar,
                                                             float* __restrict__ wb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const size_t ncell = (size_t)nx * ny * nz;
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        const int xm = x - (comp == 0), ym = y - (comp == 1), zm = z - (comp == 2);
        float s = 0.f;
        if (in3(x, y, z, nx, ny, nz)) s += 0.5f * vcb[comp * ncell + idx3(x, y, z, nx, ny)];
        if (in3(xm, ym, zm, nx, ny, nz)) s += 0.5f * vcb[comp * ncell + idx3(xm, ym, zm, nx, ny)];
        float* dst = comp == 0 ? ub : comp == 1 ? vbar : wb;
        dst[idx3(x, y, z, ax, ay)] += s;
    }
}

// ------------------------------------------------------ projection update^T
// Forward (k_update_velocity): faces touching solid (out of grid = fluid) take
// the solid velocity, the rest u + k_upd * (p_hi - p_lo) (out of grid p = 0).
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_update_faces(const uint8_t* __restrict__ flags, int nx, int ny, int nz,
                                                          float* __restrict__ ub, float* __restrict__ vbar,
                                                          float* __restrict__ wb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        const bool touching = solid0(flags, x, y, z, nx, ny, nz) ||
                              solid0(flags, x - (comp == 0), y - (comp == 1), z - (comp == 2), nx, ny, nz);
        if (touching) (comp == 0 ? ub : comp == 1 ? vbar : wb)[idx3(x, y, z, ax, ay)] = 0.f;
    }
}

// pbar(c) += k_upd * sum over axes (ubar(low face of c) - ubar(high face of c)),
// ubar already zero on faces that touch solid
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_update_pressure(const float* __restrict__ ub, const float* __restrict__ vbar,
                                                             const float* __restrict__ wb, int nx, int ny, int nz,
                                                             float k_upd, float* __restrict__ pbar) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    float s = ub[idx3(x, y, z, nx + 1, ny)] - ub[idx3(x + 1, y, z, nx + 1, ny)];
    s += vbar[idx3(x, y, z, nx, ny + 1)] - vbar[idx3(x, y + 1, z, nx, ny + 1)];
    if constexpr (DIM == 3) s += wb[idx3(x, y, z, nx, ny)] - wb[idx3(x, y, z + 1, nx, ny)];
    pbar[idx3(x, y, z, nx, ny)] += k_upd * s;
}

// ------------------------------------------------------------- divergence^T
// Forward (k_divergence, smoother rule): div(c) = sum of +-face velocities,
// the face towards a solid neighbour replaced by the solid's velocity.
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_divergence(const float* __restrict__ dbar, const uint8_t* __restrict__ flags,
                                                        int nx, int ny, int nz, float* __restrict__ ub,
                                                        float* __restrict__ vbar, float* __restrict__ wb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        const int xm = x - (comp == 0), ym = y - (comp == 1), zm = z - (comp == 2);
        const uint8_t lo_bit = comp == 0 ? F_RIGHT : comp == 1 ? F_TOP : F_FRONT;   // face seen from the low cell
        const uint8_t hi_bit = comp == 0 ? F_LEFT : comp == 1 ? F_BOTTOM : F_BACK;  // seen from the high cell
        float s = 0.f;
        if (in3(x, y, z, nx, ny, nz)) {
            const int c = idx3(x, y, z, nx, ny);
            const uint8_t f = flags[c];
            if (!(f & F_SOLID) && !(f & hi_bit)) s -= dbar[c];
        }
        if (in3(xm, ym, zm, nx, ny, nz)) {
            const int c = idx3(xm, ym, zm, nx, ny);
            const uint8_t f = flags[c];
            if (!(f & F_SOLID) && !(f & lo_bit)) s += dbar[c];
        }
        (comp == 0 ? ub : comp == 1 ? vbar : wb)[idx3(x, y, z, ax, ay)] += s;
    }
}

// ------------------------------------------------------------- V-cycle^T
// One multigrid level for the transposed operators, natural layout.  Level 0
// reads the fluid mask (weights 0/1, count of fluid neighbours), coarse levels
// the FP16-rounded solid fraction alpha (weights 1 - alpha, out of grid
// 1 - oobA).  The forward operators are smooth_cell / residual_cell /
// k_prolong (corrected out-of-grid rule) and the level-0 kernels of k_rb.cu.
struct AdjLevel {
    int nx, ny, nz;
    const uint8_t* fmask;   // level 0
    const float* alpha;     // level >= 1
    float oobA;
    float beta;    // smoother right-hand-side factor: rho*h/dt (level 0, on div), h_L^2 (level >= 1)
    float rcoef;   // residual right-hand-side factor: rho/(dt*h) (level 0), 1 (level >= 1)
    float hh;
    float* pbar;
    float* bbar;
    float* T;
};

// weight of cell (x,y,z)'s pressure in a neighbour's equation, and the
// cell's own diagonal d (sum of its neighbours' weights); updated: the
// forward smoother writes this cell
template <int DIM, bool L0>
SS_D void cell_weights(const AdjLevel& a, int x, int y, int z, float& wself, float& d, bool& fluid) {
    const int c = idx3(x, y, z, a.nx, a.ny);
    if constexpr (L0) {
        const uint8_t m = a.fmask[c];
        fluid = m & M_FLUID;
        wself = fluid ? 1.f : 0.f;
        d = (float)__popc(m & 0x7Eu);
    } else {
        const float al = a.alpha[c];
        fluid = al < 1.f;
        wself = 1.f - al;
        auto f = [&](int X, int Y, int Z) {
            return 1.f - (in3(X, Y, Z, a.nx, a.ny, a.nz) ? a.alpha[idx3(X, Y, Z, a.nx, a.ny)] : a.oobA);
        };
        float s = f(x, y + 1, z) + f(x, y - 1, z);
        s = s + f(x + 1, y, z);
        s = s + f(x - 1, y, z);
        if constexpr (DIM == 3) s = s + f(x, y, z + 1) + f(x, y, z - 1);
        d = s;
    }
}

template <int DIM>
SS_D float nbr_sum(const float* __restrict__ T, int x, int y, int z, int nx, int ny, int nz) {
    float s = 0.f;
    if (y + 1 < ny) s += T[idx3(x, y + 1, z, nx, ny)];
    if (y > 0) s += T[idx3(x, y - 1, z, nx, ny)];
    if (x + 1 < nx) s += T[idx3(x + 1, y, z, nx, ny)];
    if (x > 0) s += T[idx3(x - 1, y, z, nx, ny)];
    if constexpr (DIM == 3) {
        if (z + 1 < nz) s += T[idx3(x, y, z + 1, nx, ny)];
        if (z > 0) s += T[idx3(x, y, z - 1, nx, ny)];
    }
    return s;
}

// One colour's half of consecutive transposed colour updates:
//  B (the gather half of the previous transpose): pbar += w_self * sum of the
//    neighbours' T;
//  A (this colour's transpose): t = pbar / d, T = t, pbar = 0, bbar -= beta*t.
template <int DIM, bool L0>
__global__ void __launch_bounds__(256) k_adj_smooth(AdjLevel a, int colour, int do_b, int do_a) {
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int x = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((y + z + colour) & 1);
    if (x >= a.nx || y >= a.ny || z >= a.nz) return;
    const int c = idx3(x, y, z, a.nx, a.ny);
    float wself, d;
    bool fluid;
    cell_weights<DIM, L0>(a, x, y, z, wself, d, fluid);
    float pb = a.pbar[c];
    if (do_b) pb += wself * nbr_sum<DIM>(a.T, x, y, z, a.nx, a.ny, a.nz);
    if (do_a) {
        if (fluid && d != 0.f) {
            const float t = pb / d;
            a.T[c] = t;
            pb = 0.f;
            a.bbar[c] -= a.beta * t;
        } else {
            a.T[c] = 0.f;
        }
    }
    a.pbar[c] = pb;
}

// residual adjoint of a fine cell from its coarse parent
template <int DIM, bool L0>
SS_D float res_bar(const AdjLevel& a, const float* __restrict__ rcb, int cx, int cy, int cz, int x, int y, int z) {
    const int X = x >> 1, Y = y >> 1, Z = DIM == 3 ? z >> 1 : 0;
    if (X >= cx || Y >= cy || Z >= cz) return 0.f;
    const int c = idx3(x, y, z, a.nx, a.ny);
    const bool fluid = L0 ? (a.fmask[c] & M_FLUID) != 0 : a.alpha[c] < 1.f;
    if (!fluid) return 0.f;
    return rcb[idx3(X, Y, Z, cx, cy)] / (DIM == 3 ? 8.f : 4.f);
}

// Transpose of residual + restriction: r_c(X) = mean of the children's
// residuals b - (sum_j w_j p_j - d p) / h^2.
template <int DIM, bool L0>
__global__ void __launch_bounds__(256) k_adj_residual_restrict(AdjLevel a, const float* __restrict__ rcb, int cx, int cy, int cz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    if (x >= nx || y >= ny || z >= nz) return;
    const int c = idx3(x, y, z, nx, ny);
    float wself, d;
    bool fluid;
    cell_weights<DIM, L0>(a, x, y, z, wself, d, fluid);
    const float rs = res_bar<DIM, L0>(a, rcb, cx, cy, cz, x, y, z);
    float nb = 0.f;
    if (y + 1 < ny) nb += res_bar<DIM, L0>(a, rcb, cx, cy, cz, x, y + 1, z);
    if (y > 0) nb += res_bar<DIM, L0>(a, rcb, cx, cy, cz, x, y - 1, z);
    if (x + 1 < nx) nb += res_bar<DIM, L0>(a, rcb, cx, cy, cz, x + 1, y, z);
    if (x > 0) nb += res_bar<DIM, L0>(a, rcb, cx, cy, cz, x - 1, y, z);
    if constexpr (DIM == 3) {
        if (z + 1 < nz) nb += res_bar<DIM, L0>(a, rcb, cx, cy, cz, x, y, z + 1);
        if (z > 0) nb += res_bar<DIM, L0>(a, rcb, cx, cy, cz, x, y, z - 1);
    }
    a.pbar[c] += (d * rs - wself * nb) / a.hh;
    a.bbar[c] += a.rcoef * rs;
}

// per-axis interpolation coefficient of fine index x on coarse index K
SS_D float prolong_coef(int x, int af, int cf, int K) {
    const float tx = (((float)x + 0.5f) / (float)af) * (float)cf - 0.5f;
    const float fx = floorf(tx);
    const int x0 = (int)fx;
    const float w = tx - fx;
    const int lo = min(max(x0, 0), cf - 1), hi = min(max(x0 + 1, 0), cf - 1);
    return (lo == K ? 1.f - w : 0.f) + (hi == K ? w : 0.f);
}

// Transpose of p_f += trilinear(p_c): p_c_bar(K) = sum over the fine cells
// whose interpolation stencil holds K.  W = 6 takes the fine window
// [2K-2, 2K+3] of any size ratio; W = 4 the window [2K-1, 2K+2], which holds
// every nonzero coefficient when each fine extent is exactly twice the
// coarse one (the two outer cells of the 6-window then weigh 0), so both
// give the same sums.
template <int DIM, int W>
__global__ void __launch_bounds__(256) k_adj_prolong(const float* __restrict__ pfb, int ax, int ay, int az,
                                                     float* __restrict__ pcb, int cx, int cy, int cz) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y * blockDim.y + threadIdx.y;
    const int Z = blockIdx.z * blockDim.z + threadIdx.z;
    if (X >= cx || Y >= cy || Z >= cz) return;
    constexpr int o = W == 4 ? 1 : 2;
    // per-axis coefficients of the fine window (0 outside the grid)
    float wx[W], wy[W], wz[W];
#pragma unroll
    for (int j = 0; j < W; ++j) {
        const int x = 2 * X - o + j, y = 2 * Y - o + j, z = 2 * Z - o + j;
        wx[j] = (x >= 0 && x < ax) ? prolong_coef(x, ax, cx, X) : 0.f;
        wy[j] = (y >= 0 && y < ay) ? prolong_coef(y, ay, cy, Y) : 0.f;
        wz[j] = DIM == 3 ? ((z >= 0 && z < az) ? prolong_coef(z, az, cz, Z) : 0.f) : (j == o ? 1.f : 0.f);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < W; ++k) {
        if (wz[k] == 0.f) continue;
        const int z = DIM == 3 ? 2 * Z - o + k : 0;
#pragma unroll
        for (int j = 0; j < W; ++j) {
            if (wy[j] == 0.f) continue;
            const int y = 2 * Y - o + j;
            float row = 0.f;
#pragma unroll
            for (int i = 0; i < W; ++i)
                if (wx[i] != 0.f) row += wx[i] * pfb[idx3(2 * X - o + i, y, z, ax, ay)];
            s += wz[k] * wy[j] * row;
        }
    }
    pcb[idx3(X, Y, Z, cx, cy)] = s;
}

// ------------------------------------------------------------ vorticity^T
// Forward: w(c) = curl of the cell-centred velocity (k_vorticity, solid cells
// 0), N = g / (|g| + 1e-20) with g = central difference of |w| / 2h (k_apply_
// vorticity), f = N x w (2D: f = (-N_y w, -N_x w)), u(face c) += kappa * f(c).
// Pass 1 (per cell): fbar = kappa * (ubar, vbar, wbar at the faces of index c);
// wbar_direct = fbar x N (the part through w(c) itself); dbar = dL/d(central
// difference of |w|) through N.
template <int DIM>
SS_D float vmag_at(const float* __restrict__ vort, int x, int y, int z, int nx, int ny, int nz) {
    if (!in3(x, y, z, nx, ny, nz)) return 0.f;
    const int c = idx3(x, y, z, nx, ny);
    if constexpr (DIM == 2) {
        return fabsf(vort[c]);
    } else {
        const size_t n = (size_t)nx * ny * nz;
        const float o0 = vort[c], o1 = vort[n + c], o2 = vort[2 * n + c];
        return sqrtf(o0 * o0 + o1 * o1 + o2 * o2);
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_adj_vort1(const float* __restrict__ vort, const float* __restrict__ ub,
                                                   const float* __restrict__ vbar, const float* __restrict__ wb,
                                                   int nx, int ny, int nz, float two_h, float kappa,
                                                   float* __restrict__ wdir, float* __restrict__ dbar) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const size_t n = (size_t)nx * ny * nz;
    const int c = idx3(x, y, z, nx, ny);
    const float fb0 = kappa * ub[idx3(x, y, z, nx + 1, ny)];
    const float fb1 = kappa * vbar[idx3(x, y, z, nx, ny + 1)];
    const float fb2 = DIM == 3 ? kappa * wb[idx3(x, y, z, nx, ny)] : 0.f;
    const float dx = vmag_at<DIM>(vort, x + 1, y, z, nx, ny, nz) - vmag_at<DIM>(vort, x - 1, y, z, nx, ny, nz);
    const float dy = vmag_at<DIM>(vort, x, y + 1, z, nx, ny, nz) - vmag_at<DIM>(vort, x, y - 1, z, nx, ny, nz);
    const float dz = DIM == 3 ? vmag_at<DIM>(vort, x, y, z + 1, nx, ny, nz) - vmag_at<DIM>(vort, x, y, z - 1, nx, ny, nz) : 0.f;
    const float gx = dx / two_h, gy = dy / two_h, gz = dz / two_h;
    const float gl = sqrtf(gx * gx + gy * gy + gz * gz);
    const float len = gl + 1e-20f;
    const float Nx = gx / len, Ny = gy / len, Nz = gz / len;
    float Nb[3];
    if constexpr (DIM == 3) {
        const float o0 = vort[c], o1 = vort[n + c], o2 = vort[2 * n + c];
        // f = N x w: Nbar = w x fbar, wbar = fbar x N
        Nb[0] = o1 * fb2 - o2 * fb1;
        Nb[1] = o2 * fb0 - o0 * fb2;
        Nb[2] = o0 * fb1 - o1 * fb0;
        wdir[c] = fb1 * Nz - fb2 * Ny;
        wdir[n + c] = fb2 * Nx - fb0 * Nz;
        wdir[2 * n + c] = fb0 * Ny - fb1 * Nx;
    } else {
        const float o0 = vort[c];
        Nb[0] = -o0 * fb1;
        Nb[1] = -o0 * fb0;
        Nb[2] = 0.f;
        wdir[c] = -Ny * fb0 - Nx * fb1;
    }
    // N = g / (|g| + eps): gbar = Nbar / len - g (g . Nbar) / (|g| len^2)
    const float gdot = gx * Nb[0] + gy * Nb[1] + gz * Nb[2];
    const float q = gl > 0.f ? gdot / (gl * len * len) : 0.f;
    dbar[c] = (Nb[0] / len - gx * q) / two_h;
    dbar[n + c] = (Nb[1] / len - gy * q) / two_h;
    if (DIM == 3) dbar[2 * n + c] = (Nb[2] / len - gz * q) / two_h;
}

// Pass 2 (per cell): |w|bar from the neighbours' central differences, then
// wbar = wbar_direct + |w|bar * w / |w| (solid cells: 0, their w is fixed).
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_vort2(const float* __restrict__ vort, const float* __restrict__ wdir,
                                                   const float* __restrict__ dbar, const uint8_t* __restrict__ flags,
                                                   int nx, int ny, int nz, float* __restrict__ wbar) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const size_t n = (size_t)nx * ny * nz;
    const int c = idx3(x, y, z, nx, ny);
    if (flags[c] & F_SOLID) {
        wbar[c] = 0.f;
        if (DIM == 3) { wbar[n + c] = 0.f; wbar[2 * n + c] = 0.f; }
        return;
    }
    float mb = 0.f;
    if (x > 0) mb += dbar[idx3(x - 1, y, z, nx, ny)];
    if (x + 1 < nx) mb -= dbar[idx3(x + 1, y, z, nx, ny)];
    if (y > 0) mb += dbar[n + idx3(x, y - 1, z, nx, ny)];
    if (y + 1 < ny) mb -= dbar[n + idx3(x, y + 1, z, nx, ny)];
    if constexpr (DIM == 3) {
        if (z > 0) mb += dbar[2 * n + idx3(x, y, z - 1, nx, ny)];
        if (z + 1 < nz) mb -= dbar[2 * n + idx3(x, y, z + 1, nx, ny)];
        const float o0 = vort[c], o1 = vort[n + c], o2 = vort[2 * n + c];
        const float m = sqrtf(o0 * o0 + o1 * o1 + o2 * o2);
        const float s = m > 0.f ? mb / m : 0.f;
        wbar[c] = wdir[c] + s * o0;
        wbar[n + c] = wdir[n + c] + s * o1;
        wbar[2 * n + c] = wdir[2 * n + c] + s * o2;
    } else {
        const float o0 = vort[c];
        wbar[c] = wdir[c] + (o0 > 0.f ? mb : o0 < 0.f ? -mb : 0.f);
    }
}

// Pass 3 (per face): the cell-centred velocities' adjoints from wbar (curl
// transposed), then each face gets half of its two cells'.
template <int DIM>
SS_D float wb_at(const float* __restrict__ wbar, int comp, int x, int y, int z, int nx, int ny, int nz) {
    if (!in3(x, y, z, nx, ny, nz)) return 0.f;
    return wbar[(size_t)comp * nx * ny * nz + idx3(x, y, z, nx, ny)];
}

// adjoint of the cell-centred velocity component `comp` at cell position P
template <int DIM>
SS_D float cc_bar(const float* __restrict__ wbar, int comp, int x, int y, int z, int nx, int ny, int nz, float inv2h) {
    if constexpr (DIM == 2) {
        // w = (CCY(x+1) - CCY(x-1) - (CCX(y+1) - CCX(y-1))) / 2h
        if (comp == 1) return (wb_at<2>(wbar, 0, x - 1, y, z, nx, ny, nz) - wb_at<2>(wbar, 0, x + 1, y, z, nx, ny, nz)) * inv2h;
        return (wb_at<2>(wbar, 0, x, y + 1, z, nx, ny, nz) - wb_at<2>(wbar, 0, x, y - 1, z, nx, ny, nz)) * inv2h;
    } else {
        if (comp == 0)   // w_y uses +CCX(z+1) - CCX(z-1); w_z uses -CCX(y+1) + CCX(y-1)
            return (wb_at<3>(wbar, 1, x, y, z - 1, nx, ny, nz) - wb_at<3>(wbar, 1, x, y, z + 1, nx, ny, nz) -
                    wb_at<3>(wbar, 2, x, y - 1, z, nx, ny, nz) + wb_at<3>(wbar, 2, x, y + 1, z, nx, ny, nz)) * inv2h;
        if (comp == 1)   // w_z uses +CCY(x+1) - CCY(x-1); w_x uses -CCY(z+1) + CCY(z-1)
            return (wb_at<3>(wbar, 2, x - 1, y, z, nx, ny, nz) - wb_at<3>(wbar, 2, x + 1, y, z, nx, ny, nz) -
                    wb_at<3>(wbar, 0, x, y, z - 1, nx, ny, nz) + wb_at<3>(wbar, 0, x, y, z + 1, nx, ny, nz)) * inv2h;
        // w_x uses +CCZ(y+1) - CCZ(y-1); w_y uses -CCZ(x+1) + CCZ(x-1)
        return (wb_at<3>(wbar, 0, x, y - 1, z, nx, ny, nz) - wb_at<3>(wbar, 0, x, y + 1, z, nx, ny, nz) -
                wb_at<3>(wbar, 1, x - 1, y, z, nx, ny, nz) + wb_at<3>(wbar, 1, x + 1, y, z, nx, ny, nz)) * inv2h;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_adj_vort3(const float* __restrict__ wbar, int nx, int ny, int nz, float inv2h,
                                                   float* __restrict__ ub, float* __restrict__ vbar,
                                                   float* __restrict__ wb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        // the face (x,y,z) of axis comp is the high face of cell P-1 and the low face of cell P
        const int xm = x - (comp == 0), ym = y - (comp == 1), zm = z - (comp == 2);
        const float s = 0.5f * (cc_bar<DIM>(wbar, comp, x, y, z, nx, ny, nz, inv2h) +
                                cc_bar<DIM>(wbar, comp, xm, ym, zm, nx, ny, nz, inv2h));
        (comp == 0 ? ub : comp == 1 ? vbar : wb)[idx3(x, y, z, ax, ay)] += s;
    }
}

// --------------------------------------------------- velocity advection^T
// Forward: k_advect_velocity<DIM, BUOY>.  gin: adjoint of the advected
// (and buoyancy-forced) velocity; outputs accumulate (atomically) into
// ubar/vbar/wbar (input velocity) and dbar/tbar (smoke, through buoyancy).
//
// Per-face part, shared with the owner-computes trace pass: what the face of
// axis comp with adjoint g != 0 passes back, as flags: kKeep (a y face next
// to solid keeps its pre-advection value: g goes to the face itself), kBuoy
// (the y face's buoyancy: g goes to the two cells' smoke), kSample (a traced
// sample: tc = the back-traced point clamped as make_taps clamps it, vb = the
// position gradient; with srcb the sample's adjoint is scattered into it).
enum { kKeep = 1, kBuoy = 2, kSample = 4 };
template <int DIM, bool BUOY>
SS_D int vel_face_adj(const AdjFluid& a, int comp, int x, int y, int z, float g, bool s_c, float* srcb, float tc[3],
                      float vb[3]) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
    int f = 0;
    if (BUOY && comp == 1) {
        if (solid0(a.flags, x, y, z, nx, ny, nz) || solid0(a.flags, x, y - 1, z, nx, ny, nz)) return kKeep;
        f = kBuoy;
    }
    const int id = comp == 0 ? x : comp == 1 ? y : z;
    if (id == 0 && a.c.wind[comp] != 0.f) return f;
    if (s_c || solid1(a.flags, x - (comp == 0), y - (comp == 1), z - (comp == 2), nx, ny, nz)) return f;
    const float cfl = a.c.cfl;
    const float* src = comp == 0 ? a.u : comp == 1 ? a.v : a.w;
    float vel[3];
    if (comp == 0) vel_at_xface<DIM>(a.u, a.v, a.w, nx, ny, nz, x, y, z, vel);
    else if (comp == 1) vel_at_yface<DIM>(a.u, a.v, a.w, nx, ny, nz, x, y, z, vel);
    else vel_at_zface(a.u, a.v, a.w, nx, ny, nz, x, y, z, vel);
    const float gx = (float)x + (comp == 0 ? 0.f : 0.5f);
    const float gy = (float)y + (comp == 1 ? 0.f : 0.5f);
    const float gz = DIM == 3 ? (float)z + (comp == 2 ? 0.f : 0.5f) : 0.f;
    const float tx = gx - vel[0] * cfl - (comp == 0 ? 0.f : 0.5f);
    const float ty = gy - vel[1] * cfl - (comp == 1 ? 0.f : 0.5f);
    const float tz = gz - vel[2] * cfl - (comp == 2 ? 0.f : 0.5f);
    const Taps t = make_taps<DIM>(ax, ay, az, tx, ty, tz);
    float dw[3];
    adj_sample<DIM>(src, srcb, ax, ay, az, t, 0.f, g, dw);
    // back-trace position -> the velocity that traced it
    vb[0] = -cfl * g * dw[0] * clamp_grad(tx, ax);
    vb[1] = -cfl * g * dw[1] * clamp_grad(ty, ay);
    vb[2] = DIM == 3 ? -cfl * g * dw[2] * clamp_grad(tz, az) : 0.f;
    tc[0] = clampt(tx, -2.f, (float)(ax + 1));
    tc[1] = clampt(ty, -2.f, (float)(ay + 1));
    tc[2] = DIM == 3 ? clampt(tz, -2.f, (float)(az + 1)) : 0.f;
    return f | kSample;
}

template <int DIM, bool BUOY>
__global__ void __launch_bounds__(256) k_adj_advect_velocity(AdjFluid a, const float* __restrict__ gu, const float* __restrict__ gv,
                                                             const float* __restrict__ gw, float* __restrict__ ub,
                                                             float* __restrict__ vbar, float* __restrict__ wb,
                                                             float* __restrict__ dbar, float* __restrict__ tbar) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const bool s_c = solid1(a.flags, x, y, z, nx, ny, nz);
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        const int i = idx3(x, y, z, ax, ay);
        const float g = (comp == 0 ? gu : comp == 1 ? gv : gw)[i];
        if (g == 0.f) continue;
        float* srcb = comp == 0 ? ub : comp == 1 ? vbar : wb;
        float tc[3], vb[3];
        const int f = vel_face_adj<DIM, BUOY>(a, comp, x, y, z, g, s_c, srcb, tc, vb);
        if (f & kKeep) atomicAdd(srcb + i, g);
        if (f & kBuoy) {
            // buoyancy: dt*(-alpha*sum_ch mean(dens) + beta*(mean(T) - t_amb)), means over the cells y-1, y
            const size_t ncell = (size_t)nx * ny * nz;
            const float gd = -a.c.alpha * g * a.c.dt * 0.5f;
            const float gt = a.c.beta * g * a.c.dt * 0.5f;
            for (int ch = 0; ch < a.nch; ++ch) {
                scatter(dbar + ch * ncell, nx, ny, nz, x, y - 1, z, gd);
                scatter(dbar + ch * ncell, nx, ny, nz, x, y, z, gd);
            }
            scatter(tbar, nx, ny, nz, x, y - 1, z, gt);
            scatter(tbar, nx, ny, nz, x, y, z, gt);
        }
        if (!(f & kSample)) continue;
        const float q0 = 0.25f * vb[0], q1 = 0.25f * vb[1], q2 = 0.25f * vb[2];
        if (comp == 0) {
            atomicAdd(ub + i, vb[0]);
            // v at (i-1/2, j+1/2, k): v(i-1,j), v(i,j), v(i-1,j+1), v(i,j+1)
            scatter(vbar, nx, ny + 1, nz, x - 1, y, z, q1); scatter(vbar, nx, ny + 1, nz, x, y, z, q1);
            scatter(vbar, nx, ny + 1, nz, x - 1, y + 1, z, q1); scatter(vbar, nx, ny + 1, nz, x, y + 1, z, q1);
            if (DIM == 3) {
                scatter(wb, nx, ny, nz + 1, x - 1, y, z, q2); scatter(wb, nx, ny, nz + 1, x, y, z, q2);
                scatter(wb, nx, ny, nz + 1, x - 1, y, z + 1, q2); scatter(wb, nx, ny, nz + 1, x, y, z + 1, q2);
            }
        } else if (comp == 1) {
            atomicAdd(vbar + i, vb[1]);
            scatter(ub, nx + 1, ny, nz, x, y - 1, z, q0); scatter(ub, nx + 1, ny, nz, x + 1, y - 1, z, q0);
            scatter(ub, nx + 1, ny, nz, x, y, z, q0); scatter(ub, nx + 1, ny, nz, x + 1, y, z, q0);
            if (DIM == 3) {
                scatter(wb, nx, ny, nz + 1, x, y - 1, z, q2); scatter(wb, nx, ny, nz + 1, x, y, z, q2);
                scatter(wb, nx, ny, nz + 1, x, y - 1, z + 1, q2); scatter(wb, nx, ny, nz + 1, x, y, z + 1, q2);
            }
        } else {
            atomicAdd(wb + i, vb[2]);
            scatter(ub, nx + 1, ny, nz, x, y, z - 1, q0); scatter(ub, nx + 1, ny, nz, x + 1, y, z - 1, q0);
            scatter(ub, nx + 1, ny, nz, x, y, z, q0); scatter(ub, nx + 1, ny, nz, x + 1, y, z, q0);
            scatter(vbar, nx, ny + 1, nz, x, y, z - 1, q1); scatter(vbar, nx, ny + 1, nz, x, y + 1, z - 1, q1);
            scatter(vbar, nx, ny + 1, nz, x, y, z, q1); scatter(vbar, nx, ny + 1, nz, x, y + 1, z, q1);
        }
    }
}

// Stand-alone buoyancy^T (k_buoyancy): faces touching solid are not written
// by the forward (their output is the other buffer's content, independent of
// the input), the rest are v + dt * buoyancy.
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_buoyancy(AdjFluid a, float* __restrict__ vbar, float* __restrict__ dbar,
                                                      float* __restrict__ tbar) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    if (x >= nx || y >= ny + 1 || z >= nz) return;
    const int i = idx3(x, y, z, nx, ny + 1);
    if (solid0(a.flags, x, y, z, nx, ny, nz) || solid0(a.flags, x, y - 1, z, nx, ny, nz)) {
        vbar[i] = 0.f;
        return;
    }
    const float g = vbar[i];
    const size_t ncell = (size_t)nx * ny * nz;
    const float gd = -a.c.alpha * g * a.c.dt * 0.5f;
    const float gt = a.c.beta * g * a.c.dt * 0.5f;
    for (int ch = 0; ch < a.nch; ++ch) {
        scatter(dbar + ch * ncell, nx, ny, nz, x, y - 1, z, gd);
        scatter(dbar + ch * ncell, nx, ny, nz, x, y, z, gd);
    }
    scatter(tbar, nx, ny, nz, x, y - 1, z, gt);
    scatter(tbar, nx, ny, nz, x, y, z, gt);
}

// ---------------------------------------------------------------- emitters^T
// Forward (k_emitters): smoke gets constants added (identity adjoint); the
// faces of an active set_velocity emitter are overwritten (adjoint 0); a
// control force adds dt * force to every face inside an active emitter.
// fgrad: per-block partial sums of dt * ubar over the forced faces (3 each).
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_emitters(const ss_emitter* __restrict__ em, int ne, int nx, int ny, int nz,
                                                      float dt, int forced, float* __restrict__ ub,
                                                      float* __restrict__ vbar, float* __restrict__ wb,
                                                      double* __restrict__ fpart, int3 lo, int3 ext) {
    // launched over the active emitters' bounding box of faces
    const int tx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ty = blockIdx.y * blockDim.y + threadIdx.y;
    const int tz = blockIdx.z * blockDim.z + threadIdx.z;
    const bool in_box = tx < ext.x && ty < ext.y && tz < ext.z;
    const int x = in_box ? lo.x + tx : 1 << 30, y = lo.y + ty, z = lo.z + tz;
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        bool inside = false, set = false;
        for (int k = 0; k < ne; ++k) {
            const ss_emitter& e = em[k];
            if (!(e.emit > 0)) continue;
            float dx = (float)x - e.pos[0], dy = (float)y - e.pos[1];
            float d2 = dx * dx + dy * dy;
            if constexpr (DIM == 3) { float dz = (float)z - e.pos[2]; d2 = d2 + dz * dz; }
            if (sqrtf(d2) < e.radius) {
                inside = true;
                if (e.set_velocity) set = true;
            }
        }
        float* dst = comp == 0 ? ub : comp == 1 ? vbar : wb;
        const int i = idx3(x, y, z, ax, ay);
        if (forced && inside) acc[comp] = (double)dt * (double)dst[i];
        if (set) dst[i] = 0.f;
    }
    if (fpart) {
        // block sums of the three force components
        __shared__ double sh[3][256];
        const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
        for (int q = 0; q < 3; ++q) sh[q][tid] = acc[q];
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1) {
            if (tid < o)
                for (int q = 0; q < 3; ++q) sh[q][tid] += sh[q][tid + o];
            __syncthreads();
        }
        if (tid == 0) {
            const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
            for (int q = 0; q < 3; ++q) fpart[3 * b + q] = sh[q][0];
        }
    }
}

__global__ void k_sum3(const double* __restrict__ part, int n, double* __restrict__ out) {
    __shared__ double sh[3][256];
    double a[3] = {0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int q = 0; q < 3; ++q) a[q] += part[3 * i + q];
    for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] = a[q];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; ++q) out[q] = sh[q][0];
}

// ------------------------------------------ deterministic owner-computes
// The scatter-adds above sum in the order the atomics land, so two reverse
// passes agree only to rounding.  The owner-computes variant fixes the order:
// a trace pass stores, per source element, its back-traced point clamped as
// make_taps clamps it (w = 0 when the element scatters nothing) and the
// per-axis reach of its taps (block maxima of s - x0 and x0 - s, where x0 =
// floor of the point); a gather pass then lets every destination element d
// enumerate the box of sources whose taps can cover it (the inverse footprint:
// s in [d - max(x0 - s) - 1, d + max(s - x0)] per axis), in a fixed order,
// and add their weighted adjoints itself.  Integer maxima commute, so the
// boxes do not depend on the order the blocks finish in either.

// block maximum of the tap reaches, into win[0..5]: s - x0 per axis, then x0 - s
SS_D void reach_max(int* win, const int v[6]) {
    __shared__ int sw[6];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if (tid < 6) sw[tid] = 0;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int m = __reduce_max_sync(0xffffffffu, v[q]);
        if ((tid & 31) == 0 && m > 0) atomicMax(&sw[q], m);
    }
    __syncthreads();
    if (tid < 6 && sw[tid] > 0) atomicMax(win + tid, sw[tid]);
}

SS_D void reach_of(const float tc[3], int x, int y, int z, int dim, int v[6]) {
    const int p[3] = {x, y, z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int x0 = d < dim ? (int)floorf(tc[d]) : p[d];
        v[d] = p[d] - x0;
        v[3 + d] = x0 - p[d];
    }
}

// Longest tap reach the gather passes enumerate (boxes of at most 2 * 8 + 2
// sources per axis); longer back-traces set the error word kOwnerErr of the
// reach array, which the host reports, instead of running for minutes.
constexpr int kOwnerMaxReach = 8;
constexpr int kOwnerErr = 23;

// the box of sources whose taps can cover the element (x, y, z) of an
// (ax, ay, az) array, from the reaches win[0..5]; false (and the error word
// err set) when a reach exceeds kOwnerMaxReach
SS_D bool owner_box(const int* __restrict__ win, int* err, int x, int y, int z, int ax, int ay, int az, int dim,
                    int lo[3], int hi[3]) {
    const int p[3] = {x, y, z}, n[3] = {ax, ay, az};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d >= dim) { lo[d] = hi[d] = p[d]; continue; }
        const int back = __ldg(win + 3 + d), fwd = __ldg(win + d);
        if (back > kOwnerMaxReach || fwd > kOwnerMaxReach) {
            *err = 1;
            return false;
        }
        lo[d] = max(p[d] - back - 1, 0);
        hi[d] = min(p[d] + fwd, n[d] - 1);
    }
    return true;
}

// trilinear weight with which the sample at the traced point t covers the
// element (x, y, z); false when it is not one of the sample's taps
template <int DIM>
SS_D bool cover(const float4& t, int x, int y, int z, float* w) {
    const float fx = floorf(t.x), fy = floorf(t.y);
    const int ix = x - (int)fx, iy = y - (int)fy;
    if ((unsigned)ix > 1u || (unsigned)iy > 1u) return false;
    const float wx = t.x - fx, wy = t.y - fy;
    float r = (ix ? wx : 1.f - wx) * (iy ? wy : 1.f - wy);
    if constexpr (DIM == 3) {
        const float fz = floorf(t.z);
        const int iz = z - (int)fz;
        if ((unsigned)iz > 1u) return false;
        const float wz = t.z - fz;
        r = r * (iz ? wz : 1.f - wz);
    }
    *w = r;
    return true;
}

// smoke advection, trace pass: vcb as k_adj_advect_smoke writes it, tr = the
// cell's clamped back-traced point (w = 1; 0 for a solid cell), reaches into win
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_trace_smoke(AdjFluid a, const float* __restrict__ dout,
                                                         const float* __restrict__ tout, float* __restrict__ vcb,
                                                         float4* __restrict__ tr, int* __restrict__ win) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    int v[6] = {0, 0, 0, 0, 0, 0};
    if (x < nx && y < ny && z < nz) {
        const int c = idx3(x, y, z, nx, ny);
        const size_t ncell = (size_t)nx * ny * nz;
        float vb[3], tc[3];
        const bool live = smoke_cell_adj<DIM>(a, x, y, z, dout, tout, nullptr, nullptr, vb, tc);
        vcb[c] = vb[0];
        vcb[ncell + c] = vb[1];
        if (DIM == 3) vcb[2 * ncell + c] = vb[2];
        tr[c] = live ? make_float4(tc[0], tc[1], tc[2], 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
        if (live) reach_of(tc, x, y, z, DIM, v);
    }
    reach_max(win, v);
}

// smoke advection, gather pass: every cell adds the sampled adjoints of the
// cells whose back-traced sample covers it, sources in z, y, x order
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_gather_smoke(const float4* __restrict__ tr, const int* __restrict__ win,
                                                          int* __restrict__ err, int nx, int ny, int nz, int nch,
                                                          const float* __restrict__ dout, const float* __restrict__ tout,
                                                          float* __restrict__ din, float* __restrict__ tin) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const size_t ncell = (size_t)nx * ny * nz;
    int lo[3], hi[3];
    if (!owner_box(win, err, x, y, z, nx, ny, nz, DIM, lo, hi)) return;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};   // channels 0..2, temperature
    for (int sz = lo[2]; sz <= hi[2]; ++sz)
        for (int sy = lo[1]; sy <= hi[1]; ++sy)
            for (int sx = lo[0]; sx <= hi[0]; ++sx) {
                const int s = idx3(sx, sy, sz, nx, ny);
                const float4 t = __ldg(tr + s);
                float w;
                if (t.w == 0.f || !cover<DIM>(t, x, y, z, &w)) continue;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    if (ch >= nch) break;
                    const float g = __ldg(dout + ch * ncell + s);
                    if (g != 0.f) acc[ch] += g * w;
                }
                const float g = __ldg(tout + s);
                if (g != 0.f) acc[3] += g * w;
            }
    const int c = idx3(x, y, z, nx, ny);
#pragma unroll
    for (int ch = 0; ch < 3; ++ch)
        if (ch < nch) din[ch * ncell + c] += acc[ch];
    tin[c] += acc[3];
}

struct OwnerFaces {
    float4* tr[3];   // per face: clamped back-traced point, w = g (0: no sample)
    float4* vq[3];   // per face: position gradient (x, y, z), w = g kept by the face itself
    int* win;        // 6 reaches per component
};

// velocity advection, trace pass: per face the outcome of vel_face_adj,
// nothing scattered
template <int DIM, bool BUOY>
__global__ void __launch_bounds__(256) k_adj_trace_velocity(AdjFluid a, const float* __restrict__ gu, const float* __restrict__ gv,
                                                            const float* __restrict__ gw, OwnerFaces o) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const bool s_c = solid1(a.flags, x, y, z, nx, ny, nz);
#pragma unroll
    for (int comp = 0; comp < DIM; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        int v[6] = {0, 0, 0, 0, 0, 0};
        if (x < ax && y < ay && z < az) {
            const int i = idx3(x, y, z, ax, ay);
            const float g = (comp == 0 ? gu : comp == 1 ? gv : gw)[i];
            float4 t = make_float4(0.f, 0.f, 0.f, 0.f), q = make_float4(0.f, 0.f, 0.f, 0.f);
            if (g != 0.f) {
                float tc[3], vb[3];
                const int f = vel_face_adj<DIM, BUOY>(a, comp, x, y, z, g, s_c, nullptr, tc, vb);
                if (f & kKeep) q.w = g;
                if (f & kSample) {
                    t = make_float4(tc[0], tc[1], tc[2], g);
                    q.x = vb[0]; q.y = vb[1]; q.z = vb[2];
                    reach_of(tc, x, y, z, DIM, v);
                }
            }
            o.tr[comp][i] = t;
            o.vq[comp][i] = q;
        }
        reach_max(o.win + 6 * comp, v);
    }
}

SS_D float comp_of(const float4& q, int d) { return d == 0 ? q.x : d == 1 ? q.y : q.z; }

// velocity advection, gather pass: every face adds, in this order, the
// sampled adjoints of the faces of its axis whose sample covers it (sources
// in z, y, x order), its own position gradient, the quarter position
// gradients of the four faces of each other axis whose interpolated velocity
// it entered (offsets +a e_c - b e_d), and the value a solid-adjacent y face
// keeps; every cell then adds the buoyancy of its y faces y and y + 1.
template <int DIM, bool BUOY>
__global__ void __launch_bounds__(256) k_adj_gather_velocity(AdjFluid a, const float* __restrict__ gv, OwnerFaces o,
                                                             float* __restrict__ ub, float* __restrict__ vbar,
                                                             float* __restrict__ wb, float* __restrict__ dbar,
                                                             float* __restrict__ tbar) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const int ax = nx + (d == 0), ay = ny + (d == 1), az = nz + (d == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        const int i = idx3(x, y, z, ax, ay);
        float* dst = d == 0 ? ub : d == 1 ? vbar : wb;
        float acc = dst[i];
        int lo[3], hi[3];
        if (!owner_box(o.win + 6 * d, o.win + kOwnerErr, x, y, z, ax, ay, az, DIM, lo, hi)) return;
        const float4* tr = o.tr[d];
        for (int sz = lo[2]; sz <= hi[2]; ++sz)
            for (int sy = lo[1]; sy <= hi[1]; ++sy)
                for (int sx = lo[0]; sx <= hi[0]; ++sx) {
                    const float4 t = __ldg(tr + idx3(sx, sy, sz, ax, ay));
                    float w;
                    if (t.w != 0.f && cover<DIM>(t, x, y, z, &w)) acc += t.w * w;
                }
        const float4 own = __ldg(o.vq[d] + i);
        acc += comp_of(own, d);
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
            if (c == d) continue;
            const int cx = nx + (c == 0), cy = ny + (c == 1), cz = nz + (c == 2);
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int sx = x + (c == 0 ? e : 0) - (d == 0 ? b : 0);
                    const int sy = y + (c == 1 ? e : 0) - (d == 1 ? b : 0);
                    const int sz = z + (c == 2 ? e : 0) - (d == 2 ? b : 0);
                    if (!in3(sx, sy, sz, cx, cy, cz)) continue;
                    const float qv = 0.25f * comp_of(__ldg(o.vq[c] + idx3(sx, sy, sz, cx, cy)), d);
                    if (qv != 0.f) acc += qv;
                }
        }
        if (BUOY && d == 1) acc += own.w;
        dst[i] = acc;
    }
    if (BUOY && x < nx && y < ny && z < nz) {
        const size_t ncell = (size_t)nx * ny * nz;
        const int c = idx3(x, y, z, nx, ny);
        float dsum = 0.f, tsum = 0.f;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int fy = y + k;   // the face below, then the face above the cell
            const float g = gv[idx3(x, fy, z, nx, ny + 1)];
            if (g == 0.f) continue;
            if (solid0(a.flags, x, fy, z, nx, ny, nz) || solid0(a.flags, x, fy - 1, z, nx, ny, nz)) continue;
            dsum += -a.c.alpha * g * a.c.dt * 0.5f;
            tsum += a.c.beta * g * a.c.dt * 0.5f;
        }
        if (dsum != 0.f)
            for (int ch = 0; ch < a.nch; ++ch) dbar[ch * ncell + c] += dsum;
        if (tsum != 0.f) tbar[c] += tsum;
    }
}

// stand-alone buoyancy^T, owner-computes: each cell gathers its two y faces
// (read before any face is cleared: a face is cleared only when it touches
// solid, and then it contributes nothing)
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_buoyancy_owner(AdjFluid a, float* __restrict__ vbar, float* __restrict__ dbar,
                                                            float* __restrict__ tbar) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    if (x >= nx || y >= ny + 1 || z >= nz) return;
    const bool solid_face = solid0(a.flags, x, y, z, nx, ny, nz) || solid0(a.flags, x, y - 1, z, nx, ny, nz);
    if (y < ny) {
        const size_t ncell = (size_t)nx * ny * nz;
        const int c = idx3(x, y, z, nx, ny);
        float dsum = 0.f, tsum = 0.f;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int fy = y + k;
            if (solid0(a.flags, x, fy, z, nx, ny, nz) || solid0(a.flags, x, fy - 1, z, nx, ny, nz)) continue;
            const float g = vbar[idx3(x, fy, z, nx, ny + 1)];
            if (g == 0.f) continue;
            dsum += -a.c.alpha * g * a.c.dt * 0.5f;
            tsum += a.c.beta * g * a.c.dt * 0.5f;
        }
        if (dsum != 0.f)
            for (int ch = 0; ch < a.nch; ++ch) dbar[ch * ncell + c] += dsum;
        if (tsum != 0.f) tbar[c] += tsum;
    }
    if (solid_face) vbar[idx3(x, y, z, nx, ny + 1)] = 0.f;
}

// ------------------------------------------------------------------- host
static AdjFluid adj_fluid(const ss_sim* s, const StepConsts& c, const float* const vel[3], const float* dens,
                          const float* temp) {
    AdjFluid a;
    a.nx = s->nx; a.ny = s->ny; a.nz = s->nz; a.nch = s->nch;
    a.u = vel[0]; a.v = vel[1]; a.w = s->dim == 3 ? vel[2] : nullptr;
    a.flags = s->flags;
    a.dens = dens; a.temp = temp;
    a.c = c;
    return a;
}

static const dim3 kB(32, 8, 1);

int adj_advect_smoke(ss_sim* s, const StepConsts& c, const float* const vel[3], const float* dens, const float* temp,
                     const float* dout, const float* tout, float* din, float* tin, float* vcb, float* const vb[3],
                     cudaStream_t st, const AdjOwner* own) {
    AdjFluid a = adj_fluid(s, c, vel, dens, temp);
    dim3 g = grid_of(s->nx, s->ny, s->nz, kB);
    dim3 gf = grid_of(s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1, kB);
    if (own) {
        float4* tr = (float4*)own->tr[0];
        TRY_ADJ(check_cuda(cudaMemsetAsync(own->win, 0, 6 * sizeof(int), st), "memset"));
        if (s->dim == 3) {
            k_adj_trace_smoke<3><<<g, kB, 0, st>>>(a, dout, tout, vcb, tr, own->win);
            k_adj_gather_smoke<3><<<g, kB, 0, st>>>(tr, own->win, own->win + kOwnerErr, s->nx, s->ny, s->nz, s->nch, dout, tout, din, tin);
            k_adj_centre_to_faces<3><<<gf, kB, 0, st>>>(vcb, s->nx, s->ny, s->nz, vb[0], vb[1], vb[2]);
        } else {
            k_adj_trace_smoke<2><<<g, kB, 0, st>>>(a, dout, tout, vcb, tr, own->win);
            k_adj_gather_smoke<2><<<g, kB, 0, st>>>(tr, own->win, own->win + kOwnerErr, s->nx, s->ny, s->nz, s->nch, dout, tout, din, tin);
            k_adj_centre_to_faces<2><<<gf, kB, 0, st>>>(vcb, s->nx, s->ny, s->nz, vb[0], vb[1], nullptr);
        }
        s->nlaunch += 3;
        return check_cuda(cudaGetLastError(), "adjoint of advect_smoke (owner-computes)");
    }
    if (s->dim == 3) {
        k_adj_advect_smoke<3><<<g, kB, 0, st>>>(a, dout, tout, din, tin, vcb);
        k_adj_centre_to_faces<3><<<gf, kB, 0, st>>>(vcb, s->nx, s->ny, s->nz, vb[0], vb[1], vb[2]);
    } else {
        k_adj_advect_smoke<2><<<g, kB, 0, st>>>(a, dout, tout, din, tin, vcb);
        k_adj_centre_to_faces<2><<<gf, kB, 0, st>>>(vcb, s->nx, s->ny, s->nz, vb[0], vb[1], nullptr);
    }
    s->nlaunch += 2;
    return check_cuda(cudaGetLastError(), "adjoint of advect_smoke");
}

int adj_update(ss_sim* s, const StepConsts& c, float* const vb[3], float* pbar, cudaStream_t st) {
    dim3 g = grid_of(s->nx, s->ny, s->nz, kB);
    dim3 gf = grid_of(s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1, kB);
    if (s->dim == 3) {
        k_adj_update_faces<3><<<gf, kB, 0, st>>>(s->flags, s->nx, s->ny, s->nz, vb[0], vb[1], vb[2]);
        k_adj_update_pressure<3><<<g, kB, 0, st>>>(vb[0], vb[1], vb[2], s->nx, s->ny, s->nz, c.k_upd, pbar);
    } else {
        k_adj_update_faces<2><<<gf, kB, 0, st>>>(s->flags, s->nx, s->ny, s->nz, vb[0], vb[1], nullptr);
        k_adj_update_pressure<2><<<g, kB, 0, st>>>(vb[0], vb[1], nullptr, s->nx, s->ny, s->nz, c.k_upd, pbar);
    }
    s->nlaunch += 2;
    return check_cuda(cudaGetLastError(), "adjoint of update_velocities");
}

int adj_divergence(ss_sim* s, const float* dbar, float* const vb[3], cudaStream_t st) {
    dim3 gf = grid_of(s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1, kB);
    if (s->dim == 3) k_adj_divergence<3><<<gf, kB, 0, st>>>(dbar, s->flags, s->nx, s->ny, s->nz, vb[0], vb[1], vb[2]);
    else k_adj_divergence<2><<<gf, kB, 0, st>>>(dbar, s->flags, s->nx, s->ny, s->nz, vb[0], vb[1], nullptr);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "adjoint of the divergence");
}

// --- V-cycle^T
static AdjLevel adj_level(ss_sim* s, const StepConsts& c, int L, const AdjScratch& w) {
    AdjLevel a;
    a.nx = s->lv[L].n[0]; a.ny = s->lv[L].n[1]; a.nz = s->lv[L].n[2];
    a.fmask = s->fmask;
    a.alpha = L > 0 ? s->alpha[L] : nullptr;
    a.oobA = s->enclosed ? 1.f : 0.f;
    a.hh = s->lv[L].hh;
    a.beta = L == 0 ? c.rho_h / c.dt : s->lv[L].hh;
    a.rcoef = L == 0 ? c.rho / c.dt_h : 1.f;
    a.pbar = w.pbar[L];
    a.bbar = w.bbar[L];
    a.T = w.T[L];
    return a;
}

static int adj_sweeps(ss_sim* s, const AdjLevel& a, int L, int iterations, cudaStream_t st) {
    if (iterations <= 0) return SS_OK;
    dim3 g = grid_of((a.nx + 1) / 2, a.ny, a.nz, kB);
    // forward: per sweep colour 0 then 1; transpose: per sweep colour 1 then 0,
    // each colour's gather half fused with the next colour's update half
    auto launch = [&](int colour, int do_b, int do_a) {
        if (s->dim == 3) {
            if (L == 0) k_adj_smooth<3, true><<<g, kB, 0, st>>>(a, colour, do_b, do_a);
            else k_adj_smooth<3, false><<<g, kB, 0, st>>>(a, colour, do_b, do_a);
        } else {
            if (L == 0) k_adj_smooth<2, true><<<g, kB, 0, st>>>(a, colour, do_b, do_a);
            else k_adj_smooth<2, false><<<g, kB, 0, st>>>(a, colour, do_b, do_a);
        }
    };
    launch(1, 0, 1);
    int colour = 1;
    for (int k = 1; k < 2 * iterations; ++k) {
        colour ^= 1;
        launch(colour, 1, 1);
    }
    launch(colour ^ 1, 1, 0);
    s->nlaunch += 2 * iterations + 1;
    return check_cuda(cudaGetLastError(), "k_adj_smooth");
}

// ------------------------------------------------ single-block lower V-cycle^T
// The transpose of k_bottom: levels Lb..coarsest in one thread block with the
// adjoint arrays (pbar, bbar, T of every level) in shared memory - the
// 2*n_coarse + 1 launches of the coarsest level's transposed sweeps alone
// would otherwise dominate.  Same per-cell operations as the level kernels
// above, one __syncthreads per half-step.
struct AdjBottomArgs {
    int nlev;
    int n[SS_MAX_LEVELS][3];
    int off[SS_MAX_LEVELS];
    float hh[SS_MAX_LEVELS];
    const float* alpha[SS_MAX_LEVELS];
    float* pbar0;   // global adjoint pressure of level Lb (in/out)
    float* bbar0;   // global right-hand-side adjoint of level Lb (accumulated)
    int total;
    int n_pre, n_post, n_coarse;
    float oobA;
    const float* cresp;   // coarsest level's response matrix, or null
};

SS_D AdjLevel bottom_adj_level(const AdjBottomArgs& b, int l, float* sp, float* sb, float* sT) {
    AdjLevel a;
    a.nx = b.n[l][0]; a.ny = b.n[l][1]; a.nz = b.n[l][2];
    a.fmask = nullptr;
    a.alpha = b.alpha[l];
    a.oobA = b.oobA;
    a.hh = b.hh[l];
    a.beta = b.hh[l];
    a.rcoef = 1.f;
    a.pbar = sp + b.off[l];
    a.bbar = sb + b.off[l];
    a.T = sT + b.off[l];
    return a;
}

template <int DIM>
SS_D void bottom_adj_half(const AdjLevel& a, int colour, bool do_b, bool do_a) {
    const int n = a.nx * a.ny * a.nz;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const int x = q % a.nx, t = q / a.nx, y = t % a.ny, z = t / a.ny;
        if (((x + y + z) & 1) != colour) continue;
        float wself, d;
        bool fluid;
        cell_weights<DIM, false>(a, x, y, z, wself, d, fluid);
        float pb = a.pbar[q];
        if (do_b) pb += wself * nbr_sum<DIM>(a.T, x, y, z, a.nx, a.ny, a.nz);
        if (do_a) {
            if (fluid && d != 0.f) {
                const float tt = pb / d;
                a.T[q] = tt;
                pb = 0.f;
                a.bbar[q] -= a.beta * tt;
            } else {
                a.T[q] = 0.f;
            }
        }
        a.pbar[q] = pb;
    }
    __syncthreads();
}

// A level of at most two cells per active thread (the coarsest one): the
// cells' weights and neighbour masks stay in registers for all the sweeps.
template <int DIM, int CELLS>
SS_D void bottom_adj_sweeps_cached(const AdjLevel& a, int iterations, int nt) {
    const int n = a.nx * a.ny * a.nz;
    const int nx = a.nx, ny = a.ny, pl = nx * ny;
    // per cell: bits 0-5 neighbour in grid (+y,-y,+x,-x,+z,-z), 6 colour,
    // 7 present, 8 updated by the forward smoother
    int fl[CELLS];
    float ws[CELLS], dd[CELLS];
#pragma unroll
    for (int k = 0; k < CELLS; ++k) {
        const int c = threadIdx.x + k * nt;
        fl[k] = 0; ws[k] = 0.f; dd[k] = 1.f;
        if (c >= n) continue;
        const int x = c % nx, t = c / nx, y = t % ny, z = t / ny;
        bool fluid;
        cell_weights<DIM, false>(a, x, y, z, ws[k], dd[k], fluid);
        fl[k] = (y + 1 < ny ? 1 : 0) | (y > 0 ? 2 : 0) | (x + 1 < nx ? 4 : 0) | (x > 0 ? 8 : 0) |
                (z + 1 < a.nz ? 16 : 0) | (z > 0 ? 32 : 0) | (((x + y + z) & 1) << 6) | 128 |
                ((fluid && dd[k] != 0.f) ? 256 : 0);
    }
    auto half = [&](int colour, bool do_b, bool do_a) {
#pragma unroll
        for (int k = 0; k < CELLS; ++k) {
            const int m = fl[k];
            if (!(m & 128) || ((m >> 6) & 1) != colour) continue;
            const int c = threadIdx.x + k * nt;
            float pb = a.pbar[c];
            if (do_b) {
                float sum = 0.f;
                if (m & 1) sum += a.T[c + nx];
                if (m & 2) sum += a.T[c - nx];
                if (m & 4) sum += a.T[c + 1];
                if (m & 8) sum += a.T[c - 1];
                if (DIM == 3 && (m & 16)) sum += a.T[c + pl];
                if (DIM == 3 && (m & 32)) sum += a.T[c - pl];
                pb += ws[k] * sum;
            }
            if (do_a) {
                if (m & 256) {
                    const float tt = pb / dd[k];
                    a.T[c] = tt;
                    pb = 0.f;
                    a.bbar[c] -= a.beta * tt;
                } else {
                    a.T[c] = 0.f;
                }
            }
            a.pbar[c] = pb;
        }
        if (nt == (int)blockDim.x) __syncthreads();
        else asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
    };
    // half-steps h = 0..2*iterations: colour 1, 0, 1, ..., the first without
    // the gather, the last without the update (one call site keeps the code small)
    for (int h = 0; h <= 2 * iterations; ++h) half((h & 1) ? 0 : 1, h > 0, h < 2 * iterations);
}

template <int DIM>
SS_D void bottom_adj_sweeps(const AdjLevel& a, int iterations) {
    if (iterations <= 0) return;
    const int n = a.nx * a.ny * a.nz;
    int nt = blockDim.x;
    // the fewest threads that still give every cell its own thread (the
    // coarsest 8^3 level: 512); measured faster than two cells a thread
    while (nt > 128 && (n + nt / 2 - 1) / (nt / 2) <= 1) nt /= 2;
    if ((n + nt - 1) / nt <= 2) {
        if ((int)threadIdx.x < nt) bottom_adj_sweeps_cached<DIM, 2>(a, iterations, nt);
        __syncthreads();
        return;
    }
    if ((n + (int)blockDim.x - 1) / (int)blockDim.x <= 4) {
        bottom_adj_sweeps_cached<DIM, 4>(a, iterations, blockDim.x);
        __syncthreads();
        return;
    }
    bottom_adj_half<DIM>(a, 1, false, true);
    int colour = 1;
    for (int k = 1; k < 2 * iterations; ++k) {
        colour ^= 1;
        bottom_adj_half<DIM>(a, colour, true, true);
    }
    bottom_adj_half<DIM>(a, colour ^ 1, true, false);
}

template <int DIM>
__global__ void __launch_bounds__(1024) k_adj_bottom(AdjBottomArgs b) {
    extern __shared__ float sm[];
    float* sp = sm;
    float* sb = sm + b.total;
    float* sT = sm + 2 * b.total;
    const int n0 = b.n[0][0] * b.n[0][1] * b.n[0][2];
    for (int c = threadIdx.x; c < b.total; c += blockDim.x) {
        sp[c] = c < n0 ? b.pbar0[c] : 0.f;
        sb[c] = 0.f;
        sT[c] = 0.f;
    }
    __syncthreads();
    const int last = b.nlev - 1;
    // down: post-smoothing^T, then prolongation^T into the (fresh) coarse pbar
    for (int l = 0; l < last; ++l) {
        const AdjLevel a = bottom_adj_level(b, l, sp, sb, sT);
        bottom_adj_sweeps<DIM>(a, b.n_post);
        const int cx = b.n[l + 1][0], cy = b.n[l + 1][1], cz = b.n[l + 1][2];
        float* pc = sp + b.off[l + 1];
        for (int q = threadIdx.x; q < cx * cy * cz; q += blockDim.x) {
            const int X = q % cx, t = q / cx, Y = t % cy, Z = t / cy;
            // per-axis coefficients of the fine window [2K-2, 2K+3] (0 outside the grid)
            float wx[6], wy[6], wz[6];
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                const int x = 2 * X - 2 + j, y = 2 * Y - 2 + j, z = 2 * Z - 2 + j;
                wx[j] = (x >= 0 && x < a.nx) ? prolong_coef(x, a.nx, cx, X) : 0.f;
                wy[j] = (y >= 0 && y < a.ny) ? prolong_coef(y, a.ny, cy, Y) : 0.f;
                wz[j] = DIM == 3 ? ((z >= 0 && z < a.nz) ? prolong_coef(z, a.nz, cz, Z) : 0.f) : (j == 2 ? 1.f : 0.f);
            }
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                if (wz[k] == 0.f) continue;
                const int z = DIM == 3 ? 2 * Z - 2 + k : 0;
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    if (wy[j] == 0.f) continue;
                    const int y = 2 * Y - 2 + j;
#pragma unroll
                    for (int i = 0; i < 6; ++i)
                        if (wx[i] != 0.f) s += wx[i] * wy[j] * wz[k] * a.pbar[idx3(2 * X - 2 + i, y, z, a.nx, a.ny)];
                }
            }
            pc[q] = s;
        }
        __syncthreads();
    }
    if (b.cresp) {
        // the coarsest sweeps as one product: bbar += D^T pbar, D = d(p after
        // the sweeps)/d(right-hand side); the adjoint of their initial guess
        // (zero) is not needed.  Threads split the sum over j into `parts`
        // slices whose partial sums meet in the T arrays (unused outside the
        // sweeps), then add in slice order.
        const AdjLevel ac = bottom_adj_level(b, last, sp, sb, sT);
        const int n = ac.nx * ac.ny * ac.nz;
        int parts = (int)blockDim.x / n;
        if (parts > b.total / n) parts = b.total / n;
        if (parts < 1) parts = 1;
        const int chunk = (n + parts - 1) / parts;
        for (int t = threadIdx.x; t < n * parts; t += blockDim.x) {
            const int i = t % n, part = t / n;
            const int j0 = part * chunk, j1 = min(j0 + chunk, n);
            const float* col = b.cresp + i;
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
            int j = j0;
            for (; j + 4 <= j1; j += 4) {
                s0 += __ldg(col + (size_t)j * n) * ac.pbar[j];
                s1 += __ldg(col + (size_t)(j + 1) * n) * ac.pbar[j + 1];
                s2 += __ldg(col + (size_t)(j + 2) * n) * ac.pbar[j + 2];
                s3 += __ldg(col + (size_t)(j + 3) * n) * ac.pbar[j + 3];
            }
            for (; j < j1; ++j) s0 += __ldg(col + (size_t)j * n) * ac.pbar[j];
            sT[t] = (s0 + s1) + (s2 + s3);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            float acc = 0.f;
            for (int part = 0; part < parts; ++part) acc += sT[part * n + i];
            ac.bbar[i] += acc;
        }
        __syncthreads();
    } else {
        bottom_adj_sweeps<DIM>(bottom_adj_level(b, last, sp, sb, sT), b.n_coarse);
    }
    // up: residual + restriction^T, then pre-smoothing^T
    for (int l = last - 1; l >= 0; --l) {
        const AdjLevel a = bottom_adj_level(b, l, sp, sb, sT);
        const int cx = b.n[l + 1][0], cy = b.n[l + 1][1], cz = b.n[l + 1][2];
        const float* rcb = sb + b.off[l + 1];
        const int n = a.nx * a.ny * a.nz;
        for (int q = threadIdx.x; q < n; q += blockDim.x) {
            const int x = q % a.nx, t = q / a.nx, y = t % a.ny, z = t / a.ny;
            float wself, d;
            bool fluid;
            cell_weights<DIM, false>(a, x, y, z, wself, d, fluid);
            const float rs = res_bar<DIM, false>(a, rcb, cx, cy, cz, x, y, z);
            float nb = 0.f;
            if (y + 1 < a.ny) nb += res_bar<DIM, false>(a, rcb, cx, cy, cz, x, y + 1, z);
            if (y > 0) nb += res_bar<DIM, false>(a, rcb, cx, cy, cz, x, y - 1, z);
            if (x + 1 < a.nx) nb += res_bar<DIM, false>(a, rcb, cx, cy, cz, x + 1, y, z);
            if (x > 0) nb += res_bar<DIM, false>(a, rcb, cx, cy, cz, x - 1, y, z);
            if constexpr (DIM == 3) {
                if (z + 1 < a.nz) nb += res_bar<DIM, false>(a, rcb, cx, cy, cz, x, y, z + 1);
                if (z > 0) nb += res_bar<DIM, false>(a, rcb, cx, cy, cz, x, y, z - 1);
            }
            a.pbar[q] += (d * rs - wself * nb) / a.hh;
            a.bbar[q] += rs;
        }
        __syncthreads();
        bottom_adj_sweeps<DIM>(a, b.n_pre);
    }
    for (int c = threadIdx.x; c < n0; c += blockDim.x) {
        b.pbar0[c] = sp[c];
        b.bbar0[c] += sb[c];
    }
}

static int adj_bottom(ss_sim* s, const ss_mg_schedule& mg, int L, const AdjScratch& w, cudaStream_t st) {
    AdjBottomArgs b{};
    b.nlev = s->levels - L;
    int off = 0;
    for (int l = 0; l < b.nlev; ++l) {
        const ss::Level& lv = s->lv[L + l];
        b.n[l][0] = lv.n[0]; b.n[l][1] = lv.n[1]; b.n[l][2] = lv.n[2];
        b.off[l] = off;
        b.hh[l] = lv.hh;
        b.alpha[l] = s->alpha[L + l];
        off += lv.n[0] * lv.n[1] * lv.n[2];
    }
    b.total = off;
    b.pbar0 = w.pbar[L];
    b.bbar0 = w.bbar[L];
    b.n_pre = mg.n_pre; b.n_post = mg.n_post; b.n_coarse = mg.n_coarse;
    b.oobA = s->enclosed ? 1.f : 0.f;
    b.cresp = w.cresp;
    const size_t smem = (size_t)3 * off * sizeof(float);
    if (smem > (size_t)kBottomSmemBytes) return set_error(SS_E_INVALID, "adjoint bottom levels exceed shared memory");
    cudaError_t e = s->dim == 3
        ? cudaFuncSetAttribute(k_adj_bottom<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBottomSmemBytes)
        : cudaFuncSetAttribute(k_adj_bottom<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBottomSmemBytes);
    if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute(k_adj_bottom)");
    if (s->dim == 3) k_adj_bottom<3><<<1, 1024, smem, st>>>(b);
    else k_adj_bottom<2><<<1, 1024, smem, st>>>(b);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_adj_bottom");
}

// Transposed V-cycle from level L: on entry w.pbar[L] holds the adjoint of the
// level's output pressure; on return it holds the adjoint of its input
// pressure and w.bbar[L] has the right-hand side's adjoint added.
static int adj_v_cycle_rec(ss_sim* s, const StepConsts& c, const ss_mg_schedule& mg, int L, const AdjScratch& w,
                           cudaStream_t st) {
    const AdjLevel a = adj_level(s, c, L, w);
    if (L >= 1 && L >= s->bottom) return adj_bottom(s, mg, L, w, st);
    if (L == s->levels - 1) return adj_sweeps(s, a, L, mg.n_coarse, st);
    TRY_ADJ(adj_sweeps(s, a, L, mg.n_post, st));
    const int cx = s->lv[L + 1].n[0], cy = s->lv[L + 1].n[1], cz = s->lv[L + 1].n[2];
    const size_t nc = (size_t)cx * cy * cz;
    // p_L += P p_{L+1}  ->  pbar_{L+1} = P^T pbar_L
    dim3 gc = grid_of(cx, cy, cz, kB);
    const bool halves = a.nx == 2 * cx && a.ny == 2 * cy && (s->dim == 2 || a.nz == 2 * cz);
    if (s->dim == 3) {
        if (halves) k_adj_prolong<3, 4><<<gc, kB, 0, st>>>(a.pbar, a.nx, a.ny, a.nz, w.pbar[L + 1], cx, cy, cz);
        else k_adj_prolong<3, 6><<<gc, kB, 0, st>>>(a.pbar, a.nx, a.ny, a.nz, w.pbar[L + 1], cx, cy, cz);
    } else if (halves) {
        k_adj_prolong<2, 4><<<gc, kB, 0, st>>>(a.pbar, a.nx, a.ny, a.nz, w.pbar[L + 1], cx, cy, cz);
    } else {
        k_adj_prolong<2, 6><<<gc, kB, 0, st>>>(a.pbar, a.nx, a.ny, a.nz, w.pbar[L + 1], cx, cy, cz);
    }
    s->nlaunch += 1;
    TRY_ADJ(check_cuda(cudaMemsetAsync(w.bbar[L + 1], 0, nc * sizeof(float), st), "memset"));
    TRY_ADJ(adj_v_cycle_rec(s, c, mg, L + 1, w, st));
    // r_{L+1} = R(b_L - A p_L)
    dim3 gf = grid_of(a.nx, a.ny, a.nz, kB);
    if (s->dim == 3) {
        if (L == 0) k_adj_residual_restrict<3, true><<<gf, kB, 0, st>>>(a, w.bbar[L + 1], cx, cy, cz);
        else k_adj_residual_restrict<3, false><<<gf, kB, 0, st>>>(a, w.bbar[L + 1], cx, cy, cz);
    } else {
        if (L == 0) k_adj_residual_restrict<2, true><<<gf, kB, 0, st>>>(a, w.bbar[L + 1], cx, cy, cz);
        else k_adj_residual_restrict<2, false><<<gf, kB, 0, st>>>(a, w.bbar[L + 1], cx, cy, cz);
    }
    s->nlaunch += 1;
    TRY_ADJ(check_cuda(cudaGetLastError(), "adjoint of the V-cycle"));
    return adj_sweeps(s, a, L, mg.n_pre, st);
}

int adj_v_cycle(ss_sim* s, const StepConsts& c, const ss_mg_schedule& mg, const AdjScratch& w, cudaStream_t st) {
    return adj_v_cycle_rec(s, c, mg, 0, w, st);
}

// level-0 operator L p = sum_j w_j p_j - d p (fluid cells), for the mixed
// solve's refinement transpose: pbar -= k * L(rbar) (L is symmetric)
template <int DIM>
__global__ void __launch_bounds__(256) k_adj_apply_laplacian(const float* __restrict__ rb, const uint8_t* __restrict__ fmask,
                                                             int nx, int ny, int nz, float k, float* __restrict__ pbar) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const int c = idx3(x, y, z, nx, ny);
    const uint8_t m = fmask[c];
    if (!(m & M_FLUID)) return;
    float s = 0.f;
    if ((m & M_TOP) && y + 1 < ny) s += rb[c + nx];
    if ((m & M_BOTTOM) && y > 0) s += rb[c - nx];
    if ((m & M_RIGHT) && x + 1 < nx) s += rb[c + 1];
    if ((m & M_LEFT) && x > 0) s += rb[c - 1];
    if constexpr (DIM == 3) {
        if ((m & M_FRONT) && z + 1 < nz) s += rb[c + nx * ny];
        if ((m & M_BACK) && z > 0) s += rb[c - nx * ny];
    }
    pbar[c] -= k * (s - (float)__popc(m & 0x7Eu) * rb[c]);
}

int adj_apply_laplacian(ss_sim* s, const float* rb, float k, float* pbar, cudaStream_t st) {
    dim3 g = grid_of(s->nx, s->ny, s->nz, kB);
    if (s->dim == 3) k_adj_apply_laplacian<3><<<g, kB, 0, st>>>(rb, s->fmask, s->nx, s->ny, s->nz, k, pbar);
    else k_adj_apply_laplacian<2><<<g, kB, 0, st>>>(rb, s->fmask, s->nx, s->ny, s->nz, k, pbar);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_adj_apply_laplacian");
}

int adj_vorticity(ss_sim* s, const StepConsts& c, const float* vort, float* const vb[3], float* wdir, float* dbar,
                  float* wbar, cudaStream_t st) {
    dim3 g = grid_of(s->nx, s->ny, s->nz, kB);
    dim3 gf = grid_of(s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1, kB);
    const float two_h = 2.f * s->h;
    const float kappa = (0.5f * c.eps * s->h * c.dt) / c.rho;
    if (s->dim == 3) {
        k_adj_vort1<3><<<g, kB, 0, st>>>(vort, vb[0], vb[1], vb[2], s->nx, s->ny, s->nz, two_h, kappa, wdir, dbar);
        k_adj_vort2<3><<<g, kB, 0, st>>>(vort, wdir, dbar, s->flags, s->nx, s->ny, s->nz, wbar);
        k_adj_vort3<3><<<gf, kB, 0, st>>>(wbar, s->nx, s->ny, s->nz, 1.f / two_h, vb[0], vb[1], vb[2]);
    } else {
        k_adj_vort1<2><<<g, kB, 0, st>>>(vort, vb[0], vb[1], nullptr, s->nx, s->ny, s->nz, two_h, kappa, wdir, dbar);
        k_adj_vort2<2><<<g, kB, 0, st>>>(vort, wdir, dbar, s->flags, s->nx, s->ny, s->nz, wbar);
        k_adj_vort3<2><<<gf, kB, 0, st>>>(wbar, s->nx, s->ny, s->nz, 1.f / two_h, vb[0], vb[1], nullptr);
    }
    s->nlaunch += 3;
    return check_cuda(cudaGetLastError(), "adjoint of vorticity confinement");
}

int adj_advect_velocity(ss_sim* s, const StepConsts& c, bool buoy, const float* const vel[3], const float* dens,
                        const float* temp, const float* const gin[3], float* const vb[3], float* dbar, float* tbar,
                        cudaStream_t st, const AdjOwner* own) {
    AdjFluid a = adj_fluid(s, c, vel, dens, temp);
    dim3 gf = grid_of(s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1, kB);
    if (own) {
        OwnerFaces o;
        for (int d = 0; d < 3; ++d) {
            o.tr[d] = (float4*)own->tr[d];
            o.vq[d] = (float4*)own->vq[d];
        }
        o.win = own->win;
        TRY_ADJ(check_cuda(cudaMemsetAsync(own->win, 0, 18 * sizeof(int), st), "memset"));
        if (s->dim == 3) {
            if (buoy) {
                k_adj_trace_velocity<3, true><<<gf, kB, 0, st>>>(a, gin[0], gin[1], gin[2], o);
                k_adj_gather_velocity<3, true><<<gf, kB, 0, st>>>(a, gin[1], o, vb[0], vb[1], vb[2], dbar, tbar);
            } else {
                k_adj_trace_velocity<3, false><<<gf, kB, 0, st>>>(a, gin[0], gin[1], gin[2], o);
                k_adj_gather_velocity<3, false><<<gf, kB, 0, st>>>(a, gin[1], o, vb[0], vb[1], vb[2], dbar, tbar);
            }
        } else if (buoy) {
            k_adj_trace_velocity<2, true><<<gf, kB, 0, st>>>(a, gin[0], gin[1], nullptr, o);
            k_adj_gather_velocity<2, true><<<gf, kB, 0, st>>>(a, gin[1], o, vb[0], vb[1], nullptr, dbar, tbar);
        } else {
            k_adj_trace_velocity<2, false><<<gf, kB, 0, st>>>(a, gin[0], gin[1], nullptr, o);
            k_adj_gather_velocity<2, false><<<gf, kB, 0, st>>>(a, gin[1], o, vb[0], vb[1], nullptr, dbar, tbar);
        }
        s->nlaunch += 2;
        return check_cuda(cudaGetLastError(), "adjoint of advect_velocities (owner-computes)");
    }
    if (s->dim == 3) {
        if (buoy) k_adj_advect_velocity<3, true><<<gf, kB, 0, st>>>(a, gin[0], gin[1], gin[2], vb[0], vb[1], vb[2], dbar, tbar);
        else k_adj_advect_velocity<3, false><<<gf, kB, 0, st>>>(a, gin[0], gin[1], gin[2], vb[0], vb[1], vb[2], dbar, tbar);
    } else {
        if (buoy) k_adj_advect_velocity<2, true><<<gf, kB, 0, st>>>(a, gin[0], gin[1], nullptr, vb[0], vb[1], nullptr, dbar, tbar);
        else k_adj_advect_velocity<2, false><<<gf, kB, 0, st>>>(a, gin[0], gin[1], nullptr, vb[0], vb[1], nullptr, dbar, tbar);
    }
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "adjoint of advect_velocities");
}

// Adjoint of the coarse control force field (k_force_field): the face
// velocities pass their adjoint through unchanged, and each face scatters
// dt * ubar times its eight trilinear weights into the field's gradient (the
// weights of the forward's lerp chain; clamped taps that coincide add up).
SS_D void ff_taps(int n, float t, int* a, int* b, float* w) {
    const float f = floorf(t);
    const int i = (int)f;
    *w = t - f;
    *a = min(max(i, 0), n - 1);
    *b = min(max(i + 1, 0), n - 1);
}

__global__ void __launch_bounds__(256) k_adj_force_field(const float* __restrict__ ub, const float* __restrict__ vb,
                                                         const float* __restrict__ wb, int nx, int ny, int nz,
                                                         float* __restrict__ G, int n, float dt) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const size_t nn = (size_t)n * n * n;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
        const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
        if (x >= ax || y >= ay || z >= az) continue;
        const float* bar = comp == 0 ? ub : comp == 1 ? vb : wb;
        const float g = dt * bar[idx3(x, y, z, ax, ay)];
        if (g == 0.f) continue;
        const float xf = (float)x + (comp == 0 ? 0.f : 0.5f);
        const float yf = (float)y + (comp == 1 ? 0.f : 0.5f);
        const float zf = (float)z + (comp == 2 ? 0.f : 0.5f);
        int xa, xb, ya, yb, za, zb;
        float wx, wy, wz;
        ff_taps(n, (xf / (float)nx) * (float)n - 0.5f, &xa, &xb, &wx);
        ff_taps(n, (yf / (float)ny) * (float)n - 0.5f, &ya, &yb, &wy);
        ff_taps(n, (zf / (float)nz) * (float)n - 0.5f, &za, &zb, &wz);
        float* gc = G + comp * nn;
        const float ax0 = 1.f - wx, ay0 = 1.f - wy, az0 = 1.f - wz;
        atomicAdd(gc + idx3(xa, ya, za, n, n), g * ax0 * ay0 * az0);
        atomicAdd(gc + idx3(xb, ya, za, n, n), g * wx * ay0 * az0);
        atomicAdd(gc + idx3(xa, yb, za, n, n), g * ax0 * wy * az0);
        atomicAdd(gc + idx3(xb, yb, za, n, n), g * wx * wy * az0);
        atomicAdd(gc + idx3(xa, ya, zb, n, n), g * ax0 * ay0 * wz);
        atomicAdd(gc + idx3(xb, ya, zb, n, n), g * wx * ay0 * wz);
        atomicAdd(gc + idx3(xa, yb, zb, n, n), g * ax0 * wy * wz);
        atomicAdd(gc + idx3(xb, yb, zb, n, n), g * wx * wy * wz);
    }
}

// Owner-computes variant: one block per (coarse sample, component) sums
// dt * ubar times the sample's weight over the faces whose taps include it,
// each thread over a fixed subset in a fixed order, then a fixed tree.
// Candidate faces along an axis: t = ((i + off) / na) * n - 0.5 in
// [ci - 1, ci + 1) (every face below / above for the end samples, where the
// taps clamp), widened by 2 for rounding; ff_taps decides exactly.
SS_D void ff_range(int ci, int n, int na, float off, int a, int* lo, int* hi) {
    const float sc = (float)na / (float)n;
    int l = (int)floorf(((float)ci - 0.5f) * sc - off) - 2, h = (int)ceilf(((float)ci + 1.5f) * sc - off) + 2;
    if (ci == 0) l = 0;
    if (ci == n - 1) h = a - 1;
    *lo = max(l, 0);
    *hi = min(h, a - 1);
}
SS_D float ff_weight(int ci, int n, float t) {
    int ta, tb;
    float w;
    ff_taps(n, t, &ta, &tb, &w);
    return (ta == ci ? 1.f - w : 0.f) + (tb == ci ? w : 0.f);
}

__global__ void __launch_bounds__(256) k_adj_force_field_owner(const float* __restrict__ ub, const float* __restrict__ vb,
                                                               const float* __restrict__ wb, int nx, int ny, int nz,
                                                               float* __restrict__ G, int n, float dt) {
    const int node = blockIdx.x, comp = blockIdx.y;
    const int ci = node % n, cj = (node / n) % n, ck = node / (n * n);
    const int ax = nx + (comp == 0), ay = ny + (comp == 1), az = nz + (comp == 2);
    const float ox = comp == 0 ? 0.f : 0.5f, oy = comp == 1 ? 0.f : 0.5f, oz = comp == 2 ? 0.f : 0.5f;
    int lx, hx, ly, hy, lz, hz;
    ff_range(ci, n, nx, ox, ax, &lx, &hx);
    ff_range(cj, n, ny, oy, ay, &ly, &hy);
    ff_range(ck, n, nz, oz, az, &lz, &hz);
    const int ex = hx - lx + 1, ey = hy - ly + 1, ez = hz - lz + 1;
    const float* bar = comp == 0 ? ub : comp == 1 ? vb : wb;
    float acc = 0.f;
    const int total = ex * ey * ez;
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int x = lx + k % ex, y = ly + (k / ex) % ey, z = lz + k / (ex * ey);
        const float g = dt * bar[idx3(x, y, z, ax, ay)];
        if (g == 0.f) continue;
        const float wx = ff_weight(ci, n, (((float)x + ox) / (float)nx) * (float)n - 0.5f);
        const float wy = ff_weight(cj, n, (((float)y + oy) / (float)ny) * (float)n - 0.5f);
        const float wz = ff_weight(ck, n, (((float)z + oz) / (float)nz) * (float)n - 0.5f);
        const float w = wx * wy * wz;
        if (w != 0.f) acc += g * w;
    }
    __shared__ float sh[256];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0 && sh[0] != 0.f) G[(size_t)comp * n * n * n + node] += sh[0];
}

int adj_force_field(ss_sim* s, const StepConsts& c, float* const ub[3], float* grad, cudaStream_t st,
                    const AdjOwner* own) {
    if (s->ff_n <= 0 || s->dim != 3) return SS_OK;
    if (own) {
        const int n = s->ff_n;
        k_adj_force_field_owner<<<dim3((unsigned)(n * n * n), 3), 256, 0, st>>>(ub[0], ub[1], ub[2], s->nx, s->ny,
                                                                              s->nz, grad, n, c.dt);
    } else {
        dim3 b(32, 8, 1);
        dim3 g = grid_of(s->nx + 1, s->ny + 1, s->nz + 1, b);
        k_adj_force_field<<<g, b, 0, st>>>(ub[0], ub[1], ub[2], s->nx, s->ny, s->nz, grad, s->ff_n, c.dt);
    }
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_adj_force_field");
}

int adj_buoyancy(ss_sim* s, const StepConsts& c, float* vbar, float* dbar, float* tbar, cudaStream_t st,
                 const AdjOwner* own) {
    const float* vel[3] = {nullptr, nullptr, nullptr};
    AdjFluid a = adj_fluid(s, c, vel, nullptr, nullptr);
    dim3 g = grid_of(s->nx, s->ny + 1, s->nz, kB);
    if (own) {
        if (s->dim == 3) k_adj_buoyancy_owner<3><<<g, kB, 0, st>>>(a, vbar, dbar, tbar);
        else k_adj_buoyancy_owner<2><<<g, kB, 0, st>>>(a, vbar, dbar, tbar);
    } else if (s->dim == 3) {
        k_adj_buoyancy<3><<<g, kB, 0, st>>>(a, vbar, dbar, tbar);
    } else {
        k_adj_buoyancy<2><<<g, kB, 0, st>>>(a, vbar, dbar, tbar);
    }
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "adjoint of apply_buoyancy");
}

int adj_emitters(ss_sim* s, const StepConsts& c, int forced, float* const vb[3], double* fpart, double* fout,
                 const ss_emitter* em, int ne, cudaStream_t st) {
    // bounding box (faces) of the active emitters, as the forward launch takes it
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-1, -1, -1};
    int active = 0;
    for (int k = 0; k < ne; ++k) {
        if (!(em[k].emit > 0)) continue;
        ++active;
        for (int d = 0; d < s->dim; ++d) {
            const int a = (int)floorf(em[k].pos[d] - em[k].radius) - 1, b = (int)ceilf(em[k].pos[d] + em[k].radius) + 2;
            lo[d] = lo[d] < a ? lo[d] : a;
            hi[d] = hi[d] > b ? hi[d] : b;
        }
    }
    if (s->dim == 2) { lo[2] = 0; hi[2] = 1; }
    const int ext_all[3] = {s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1};
    for (int d = 0; d < 3; ++d) {
        lo[d] = lo[d] < 0 ? 0 : lo[d];
        hi[d] = hi[d] > ext_all[d] ? ext_all[d] : hi[d];
        if (hi[d] < lo[d]) hi[d] = lo[d];
    }
    if (!active) { lo[0] = lo[1] = lo[2] = 0; hi[0] = hi[1] = hi[2] = 0; }
    const int3 l = make_int3(lo[0], lo[1], lo[2]);
    const int3 e = make_int3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]);
    dim3 gf = grid_of(e.x > 0 ? e.x : 1, e.y > 0 ? e.y : 1, e.z > 0 ? e.z : 1, kB);
    const int nb = (int)(gf.x * gf.y * gf.z);
    if (nb > adj_force_blocks(s)) return set_error(SS_E_INVALID, "force scratch too small");
    if (s->dim == 3) k_adj_emitters<3><<<gf, kB, 0, st>>>(s->d_em, ne, s->nx, s->ny, s->nz, c.dt, forced, vb[0], vb[1], vb[2], fpart, l, e);
    else k_adj_emitters<2><<<gf, kB, 0, st>>>(s->d_em, ne, s->nx, s->ny, s->nz, c.dt, forced, vb[0], vb[1], nullptr, fpart, l, e);
    k_sum3<<<1, 256, 0, st>>>(fpart, nb, fout);
    s->nlaunch += 2;
    return check_cuda(cudaGetLastError(), "adjoint of handle_emitters");
}

int adj_force_blocks(const ss_sim* s) {
    dim3 gf = grid_of(s->nx + 1, s->ny + 1, s->dim == 3 ? s->nz + 1 : 1, kB);
    return (int)(gf.x * gf.y * gf.z);
}

}  // namespace ss
