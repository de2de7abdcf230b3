// k_rb.cu - level-0 pressure operators on colour-split arrays.
//
// For the duration of a pressure solve, level 0 keeps the pressure, the two
// right-hand sides and the fluid mask split by colour: cell (x,y,z) with
// colour c = (x+y+z) & 1 lives at index ((z*ny + y)*nx/2 + x/2) of the colour-c
// array (nx even).  A half-sweep of colour c then reads only the other
// colour's pressure plus its own right-hand side and mask and writes its own
// pressure - 6.5 B per cell and half-sweep, fully coalesced, with no halo
// and no shared memory.  The neighbours of a cell are at x/2 in the rows
// y+-1 and z+-1 of the other colour and at (x-1)/2 and (x+1)/2 in its own row.
//
// Arithmetic per cell is that of smooth.comp:79-136 / compute_residual.comp:
// 77-130 (value-identical; fluid mask with select instead of p*f, the division
// by the fluid-neighbour count through div_by_count, right-hand sides
// precomputed with the reference's operations by k_divergence).
#include "common.cuh"
#include "ss_internal.h"

namespace ss {

struct RBLevel {
    int nx, ny, nz, half;   // half = nx / 2
};

SS_D int rb_index(int x, int y, int z, const RBLevel& g) { return (z * g.ny + y) * g.half + (x >> 1); }

// natural <-> colour-split
template <bool SPLIT>
__global__ void k_rb_convert(float* __restrict__ nat, float* __restrict__ red, float* __restrict__ black, RBLevel g) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx) return;
    const int n = idx3(x, y, z, g.nx, g.ny);
    float* dst = ((x + y + z) & 1) ? black : red;
    const int i = rb_index(x, y, z, g);
    if (SPLIT) dst[i] = nat[n];
    else nat[n] = dst[i];
}

template <typename T>
__global__ void k_rb_split_any(const T* __restrict__ nat, T* __restrict__ red, T* __restrict__ black, RBLevel g) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx) return;
    T* dst = ((x + y + z) & 1) ? black : red;
    dst[rb_index(x, y, z, g)] = nat[idx3(x, y, z, g.nx, g.ny)];
}

// p_sum of the reference's smoother/residual over the other colour's array,
// in its order (+y, -y, +x, -x, +z, -z); out-of-grid pressure is 0.
template <int DIM>
SS_D float rb_psum(const float* __restrict__ po, int x, int y, int z, uint8_t m, const RBLevel& g) {
    const int xh = x >> 1;
    const int row = (z * g.ny + y) * g.half;
    const float p_top = (m & M_TOP) && y + 1 < g.ny ? __ldg(po + row + g.half + xh) : 0.f;
    const float p_bottom = (m & M_BOTTOM) && y > 0 ? __ldg(po + row - g.half + xh) : 0.f;
    const float p_right = (m & M_RIGHT) && x + 1 < g.nx ? __ldg(po + row + ((x + 1) >> 1)) : 0.f;
    const float p_left = (m & M_LEFT) && x > 0 ? __ldg(po + row + ((x - 1) >> 1)) : 0.f;
    float s = p_top + p_bottom;
    s = s + p_right;
    s = s + p_left;
    if constexpr (DIM == 3) {
        const int pl = g.ny * g.half;
        const float p_front = (m & M_FRONT) && z + 1 < g.nz ? __ldg(po + row + pl + xh) : 0.f;
        const float p_back = (m & M_BACK) && z > 0 ? __ldg(po + row - pl + xh) : 0.f;
        s = s + p_front;
        s = s + p_back;
    }
    return s;
}

// One colour of a red-black sweep (colour 0 = red, the reference's parity 0).
template <int DIM>
__global__ void __launch_bounds__(256) k_rb_smooth(float* __restrict__ pc, const float* __restrict__ po,
                                                   const float* __restrict__ rhs_c, const uint8_t* __restrict__ mask_c,
                                                   RBLevel g, int colour) {
    const int xh = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (xh >= g.half || y >= g.ny) return;
    const int x = 2 * xh + ((y + z + colour) & 1);
    const int i = (z * g.ny + y) * g.half + xh;
    const uint8_t m = mask_c[i];
    const int fs = __popc(m & 0x7E);
    if (!(m & M_FLUID) || fs == 0) return;
    const float p_sum = rb_psum<DIM>(po, x, y, z, m, g);
    pc[i] = div_by_count(p_sum - __ldg(rhs_c + i), fs);
}

// Residual of every fine cell, restricted into the coarse level (natural
// layout): one thread per coarse cell and its 2^DIM children.
template <int DIM, bool POW2>
__global__ void __launch_bounds__(256) k_rb_residual_restrict(const float* __restrict__ p_red, const float* __restrict__ p_black,
                                                              const float* __restrict__ rr_red, const float* __restrict__ rr_black,
                                                              const uint8_t* __restrict__ m_red, const uint8_t* __restrict__ m_black,
                                                              RBLevel g, float* __restrict__ rc, int cx, int cy, int cz,
                                                              float hh, float inv_hh) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y * blockDim.y + threadIdx.y;
    const int Z = blockIdx.z;
    if (X >= cx || Y >= cy) return;
    float v[2][2][2];
#pragma unroll
    for (int dz = 0; dz < (DIM == 3 ? 2 : 1); ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int x = 2 * X + dx, y = 2 * Y + dy, z = DIM == 3 ? 2 * Z + dz : 0;
                float res = 0.f;
                const int c = (x + y + z) & 1;
                const int i = rb_index(x, y, z, g);
                const uint8_t m = (c ? m_black : m_red)[i];
                if (m & M_FLUID) {
                    const float p_sum = rb_psum<DIM>(c ? p_red : p_black, x, y, z, m, g);
                    const float f_sum = (float)__popc(m & 0x7E);
                    const float lap = p_sum - f_sum * __ldg((c ? p_black : p_red) + i);
                    res = __ldg((c ? rr_black : rr_red) + i) - (POW2 ? lap * inv_hh : lap / hh);
                }
                v[dz][dy][dx] = res;
            }
    float out;
    if constexpr (DIM == 3) {
        const float bottom = v[0][0][0] + v[1][0][0] + v[0][0][1] + v[1][0][1];
        const float top = v[0][1][0] + v[1][1][0] + v[0][1][1] + v[1][1][1];
        out = (bottom + top) / 8.f;
    } else {
        out = (v[0][0][0] + v[0][0][1] + v[0][1][0] + v[0][1][1]) / 4.f;
    }
    rc[idx3(X, Y, Z, cx, cy)] = out;
}

// prolong_pressure.comp:39-51 into the colour-split level 0
template <int DIM>
__global__ void __launch_bounds__(256) k_rb_prolong(float* __restrict__ p_red, float* __restrict__ p_black, RBLevel g,
                                                    const float* __restrict__ pc, int cx, int cy, int cz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx) return;
    const int ax = g.nx, ay = g.ny, az = g.nz;
    const float tx = (((float)x + 0.5f) / (float)ax) * (float)cx - 0.5f;
    const float ty = (((float)y + 0.5f) / (float)ay) * (float)cy - 0.5f;
    const float fx = floorf(tx), fy = floorf(ty);
    const int x0 = (int)fx, y0 = (int)fy;
    const float wx = tx - fx, wy = ty - fy;
    const int xa = min(max(x0, 0), cx - 1), xb = min(max(x0 + 1, 0), cx - 1);
    const int ya = min(max(y0, 0), cy - 1), yb = min(max(y0 + 1, 0), cy - 1);
    float s;
    if constexpr (DIM == 2) {
        s = lerp_(lerp_(__ldg(pc + idx3(xa, ya, 0, cx, cy)), __ldg(pc + idx3(xb, ya, 0, cx, cy)), wx),
                  lerp_(__ldg(pc + idx3(xa, yb, 0, cx, cy)), __ldg(pc + idx3(xb, yb, 0, cx, cy)), wx), wy);
    } else {
        const float tz = (((float)z + 0.5f) / (float)az) * (float)cz - 0.5f;
        const float fz = floorf(tz);
        const int z0 = (int)fz;
        const float wz = tz - fz;
        const int za = min(max(z0, 0), cz - 1), zb = min(max(z0 + 1, 0), cz - 1);
        const float c0 = lerp_(lerp_(__ldg(pc + idx3(xa, ya, za, cx, cy)), __ldg(pc + idx3(xb, ya, za, cx, cy)), wx),
                               lerp_(__ldg(pc + idx3(xa, yb, za, cx, cy)), __ldg(pc + idx3(xb, yb, za, cx, cy)), wx), wy);
        const float c1 = lerp_(lerp_(__ldg(pc + idx3(xa, ya, zb, cx, cy)), __ldg(pc + idx3(xb, ya, zb, cx, cy)), wx),
                               lerp_(__ldg(pc + idx3(xa, yb, zb, cx, cy)), __ldg(pc + idx3(xb, yb, zb, cx, cy)), wx), wy);
        s = lerp_(c0, c1, wz);
    }
    float* dst = ((x + y + z) & 1) ? p_black : p_red;
    const int i = rb_index(x, y, z, g);
    dst[i] = dst[i] + s;
}

// ------------------------------------------------------------------ host
// 256-thread blocks over rows of length n: n threads (rounded up to a warp)
// along x, the rest of the block on successive rows
static void row_launch(int n, int rows, int planes, dim3& b, dim3& g) {
    int bx = ((n + 31) / 32) * 32;
    if (bx > 256) bx = 256;
    const int by = 256 / bx;
    b = dim3(bx, by, 1);
    g = dim3((n + bx - 1) / bx, (rows + by - 1) / by, planes);
}

static RBLevel rb_level(const ss_sim* s) {
    RBLevel g;
    g.nx = s->lv[0].n[0]; g.ny = s->lv[0].n[1]; g.nz = s->lv[0].n[2];
    g.half = g.nx / 2;
    return g;
}

bool rb_supported(const ss_sim* s, int quirks) {
    return s->rhs_s && s->rb_mask && s->levels > 1 && (s->nx % 2) == 0 && (s->enclosed || !quirks);
}

int launch_rb_convert(ss_sim* s, bool split, cudaStream_t st) {
    const RBLevel g = rb_level(s);
    dim3 b(128), gr((g.nx + 127) / 128, g.ny, g.nz);
    float* red = s->p_alt[0];
    float* black = s->p_alt[0] + s->ncell / 2;
    if (split) k_rb_convert<true><<<gr, b, 0, st>>>(s->p[0], red, black, g);
    else k_rb_convert<false><<<gr, b, 0, st>>>(s->p[0], red, black, g);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_rb_convert");
}

int launch_rb_split_mask(ss_sim* s, cudaStream_t st) {
    const RBLevel g = rb_level(s);
    dim3 b(128), gr((g.nx + 127) / 128, g.ny, g.nz);
    k_rb_split_any<uint8_t><<<gr, b, 0, st>>>(s->fmask, s->rb_mask, s->rb_mask + s->ncell / 2, g);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_rb_split_any");
}

int launch_rb_sweep(ss_sim* s, int iterations, cudaStream_t st) {
    const RBLevel g = rb_level(s);
    const size_t h = s->ncell / 2;
    float* p[2] = {s->p_alt[0], s->p_alt[0] + h};
    const float* rhs[2] = {s->rhs_s, s->rhs_s + h};
    const uint8_t* mask[2] = {s->rb_mask, s->rb_mask + h};
    dim3 b, gr;
    row_launch(g.half, g.ny, g.nz, b, gr);
    for (int it = 0; it < iterations; ++it)
        for (int c = 0; c < 2; ++c) {
            if (s->dim == 3) k_rb_smooth<3><<<gr, b, 0, st>>>(p[c], p[1 - c], rhs[c], mask[c], g, c);
            else k_rb_smooth<2><<<gr, b, 0, st>>>(p[c], p[1 - c], rhs[c], mask[c], g, c);
        }
    s->nlaunch += 2 * iterations;
    return check_cuda(cudaGetLastError(), "k_rb_smooth");
}

static bool pow2f(float v) {
    if (!(v > 0.f) || !isfinite(v)) return false;
    int e;
    return frexpf(v, &e) == 0.5f && v >= 1.1754944e-38f && v <= 1e30f;
}

int launch_rb_residual_restrict(ss_sim* s, cudaStream_t st) {
    const RBLevel g = rb_level(s);
    const size_t h = s->ncell / 2;
    const int cx = s->lv[1].n[0], cy = s->lv[1].n[1], cz = s->lv[1].n[2];
    const float hh = s->lv[0].hh;
    const bool p2 = pow2f(hh);
    dim3 b, gr;
    row_launch(cx, cy, cz, b, gr);
    const float* pr = s->p_alt[0];
    const float* pb = pr + h;
    const float* rr = s->rhs_r;
    if (s->dim == 3) {
        if (p2) k_rb_residual_restrict<3, true><<<gr, b, 0, st>>>(pr, pb, rr, rr + h, s->rb_mask, s->rb_mask + h, g, s->r[1], cx, cy, cz, hh, 1.f / hh);
        else k_rb_residual_restrict<3, false><<<gr, b, 0, st>>>(pr, pb, rr, rr + h, s->rb_mask, s->rb_mask + h, g, s->r[1], cx, cy, cz, hh, 0.f);
    } else {
        if (p2) k_rb_residual_restrict<2, true><<<gr, b, 0, st>>>(pr, pb, rr, rr + h, s->rb_mask, s->rb_mask + h, g, s->r[1], cx, cy, cz, hh, 1.f / hh);
        else k_rb_residual_restrict<2, false><<<gr, b, 0, st>>>(pr, pb, rr, rr + h, s->rb_mask, s->rb_mask + h, g, s->r[1], cx, cy, cz, hh, 0.f);
    }
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_rb_residual_restrict");
}

int launch_rb_prolong(ss_sim* s, cudaStream_t st) {
    const RBLevel g = rb_level(s);
    const size_t h = s->ncell / 2;
    const int cx = s->lv[1].n[0], cy = s->lv[1].n[1], cz = s->lv[1].n[2];
    dim3 b(128), gr((g.nx + 127) / 128, g.ny, g.nz);
    if (s->dim == 3) k_rb_prolong<3><<<gr, b, 0, st>>>(s->p_alt[0], s->p_alt[0] + h, g, s->p[1], cx, cy, cz);
    else k_rb_prolong<2><<<gr, b, 0, st>>>(s->p_alt[0], s->p_alt[0] + h, g, s->p[1], cx, cy, cz);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_rb_prolong");
}

}  // namespace ss
