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
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

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
    pdl_entry();
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
// T: storage of the coarse level; for the mixed-precision correction solve
// (T = FP16 / BF16) the restricted value is multiplied by a power-of-two
// scale before it is rounded, which keeps it in the normal range.
template <int DIM, bool POW2, typename T = float>
__global__ void __launch_bounds__(256) k_rb_residual_restrict(const float* __restrict__ p_red, const float* __restrict__ p_black,
                                                              const float* __restrict__ rr_red, const float* __restrict__ rr_black,
                                                              const uint8_t* __restrict__ m_red, const uint8_t* __restrict__ m_black,
                                                              RBLevel g, T* __restrict__ rc, int cx, int cy, int cz,
                                                              float hh, float inv_hh, const float* __restrict__ scale) {
    pdl_entry();
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
    if constexpr (!std::is_same<T, float>::value) out = out * scale[0];
    rc[idx3(X, Y, Z, cx, cy)] = st<T>(out);
}

// prolong_pressure.comp:39-51 into the colour-split level 0
template <int DIM, typename T = float>
__global__ void __launch_bounds__(256) k_rb_prolong(float* __restrict__ p_red, float* __restrict__ p_black, RBLevel g,
                                                    const T* __restrict__ pc, int cx, int cy, int cz,
                                                    const float* __restrict__ scale) {
    pdl_entry();
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
        s = lerp_(lerp_(ld(pc[idx3(xa, ya, 0, cx, cy)]), ld(pc[idx3(xb, ya, 0, cx, cy)]), wx),
                  lerp_(ld(pc[idx3(xa, yb, 0, cx, cy)]), ld(pc[idx3(xb, yb, 0, cx, cy)]), wx), wy);
    } else {
        const float tz = (((float)z + 0.5f) / (float)az) * (float)cz - 0.5f;
        const float fz = floorf(tz);
        const int z0 = (int)fz;
        const float wz = tz - fz;
        const int za = min(max(z0, 0), cz - 1), zb = min(max(z0 + 1, 0), cz - 1);
        const float c0 = lerp_(lerp_(ld(pc[idx3(xa, ya, za, cx, cy)]), ld(pc[idx3(xb, ya, za, cx, cy)]), wx),
                               lerp_(ld(pc[idx3(xa, yb, za, cx, cy)]), ld(pc[idx3(xb, yb, za, cx, cy)]), wx), wy);
        const float c1 = lerp_(lerp_(ld(pc[idx3(xa, ya, zb, cx, cy)]), ld(pc[idx3(xb, ya, zb, cx, cy)]), wx),
                               lerp_(ld(pc[idx3(xa, yb, zb, cx, cy)]), ld(pc[idx3(xb, yb, zb, cx, cy)]), wx), wy);
        s = lerp_(c0, c1, wz);
    }
    if constexpr (!std::is_same<T, float>::value) s = s * scale[1];
    float* dst = ((x + y + z) & 1) ? p_black : p_red;
    const int i = rb_index(x, y, z, g);
    dst[i] = dst[i] + s;
}

// ------------------------------------------------------------------ 4 cells per thread
// With nx % 8 == 0 every colour row holds a whole number of float4 quads, so
// a thread takes four consecutive same-colour cells of a row: one float4 of
// each neighbouring row of the other colour, one of its own row plus one
// scalar for the row-end neighbour, a float4 of right-hand sides and the four
// mask bytes in one word.  Same values as the one-cell kernels above: the
// neighbour sum keeps the order +y, -y, +x, -x, +z, -z and selects 0 for a
// non-fluid or out-of-grid neighbour.

// A thread marches up `planes` z planes of its row: the other colour's row in
// its own plane is the previous plane's front row and the back row is the
// previous plane's own row (both kept in registers), and the loads of plane
// z+1 are issued before plane z is computed.
struct RbPlane {
    uint32_t m4;
    float4 rhs, pt, pb, pf;
    float extra;
};

// ZERO: every non-fluid cell of the other colour holds +0 (the mixed solve's
// correction: it starts at 0 and its prolongation zeroes non-fluid cells), so
// a neighbour needs no select - a +0 term in the same place of the sum is
// the value the select gives.
// INIT: the first half-sweep from a zero pressure.  Every neighbour is +0, so
// the neighbour sum is +0 and the other colour is not read; the kernel writes
// all of its own colour (+0 where the cell is not updated) and +0 over the
// other colour (zo) - the values a clear of both arrays followed by the plain
// half-sweep leaves.
template <int DIM, bool ZERO = false, bool INIT = false>
__global__ void __launch_bounds__(256) k_rb_smooth4(float* __restrict__ pc, const float* __restrict__ po,
                                                    const float* __restrict__ rhs_c, const uint8_t* __restrict__ mask_c,
                                                    RBLevel g, int colour, int planes, float* __restrict__ zo) {
    pdl_entry();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (q >= (g.half >> 2) || y >= g.ny) return;
    const int zb = blockIdx.z * planes, ze = min(zb + planes, g.nz);
    const int xh0 = q << 2;
    const int pl = g.ny * g.half;
    const bool up = y + 1 < g.ny, dn = y > 0;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    // every load of a plane is issued before the first one is waited for (no
    // early exit on an all-solid quad)
    auto load = [&](int z, RbPlane& P) {
        const int i = (z * g.ny + y) * g.half + xh0;
        const int par = (y + z + colour) & 1;   // x = 2*xh + par
        P.m4 = __ldg(reinterpret_cast<const uint32_t*>(mask_c + i));
        P.rhs = ldg4(rhs_c + i);
        if constexpr (INIT) return;
        P.pt = up ? ldg4(po + i + g.half) : zero;
        P.pb = dn ? ldg4(po + i - g.half) : zero;
        P.pf = (DIM == 3 && z + 1 < g.nz) ? ldg4(po + i + pl) : zero;
        // row-end neighbour: left of the first cell (par 0) or right of the last (par 1)
        P.extra = par == 0 ? (xh0 > 0 ? __ldg(po + i - 1) : 0.f) : (xh0 + 4 < g.half ? __ldg(po + i + 4) : 0.f);
    };
    const int i0 = (zb * g.ny + y) * g.half + xh0;
    float4 pm = zero, pk = zero;
    RbPlane cur, nxt;
    cur.pt = cur.pb = cur.pf = zero;
    cur.extra = 0.f;
    if constexpr (!INIT) {
        pm = ldg4(po + i0);
        pk = (DIM == 3 && zb > 0) ? ldg4(po + i0 - pl) : zero;
    }
    load(zb, cur);
    nxt = cur;
    for (int z = zb; z < ze; ++z) {
        if (z + 1 < ze) load(z + 1, nxt);
        const int i = (z * g.ny + y) * g.half + xh0;
        const int par = (y + z + colour) & 1;
        float out[4];
        bool wr[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t m = (cur.m4 >> (8 * k)) & 0xFFu;
            const int fs = __popc(m & 0x7Eu);
            wr[k] = (m & M_FLUID) && fs != 0;
            const float left = par ? f4(pm, k) : (k ? f4(pm, k - 1) : cur.extra);
            const float right = par ? (k < 3 ? f4(pm, k + 1) : cur.extra) : f4(pm, k);
            float sum;
            if constexpr (INIT) {
                sum = 0.f;
            } else if constexpr (ZERO) {
                sum = f4(cur.pt, k) + f4(cur.pb, k);
                sum = sum + right;
                sum = sum + left;
                if constexpr (DIM == 3) {
                    sum = sum + f4(cur.pf, k);
                    sum = sum + f4(pk, k);
                }
            } else {
                sum = ((m & M_TOP) ? f4(cur.pt, k) : 0.f) + ((m & M_BOTTOM) ? f4(cur.pb, k) : 0.f);
                sum = sum + ((m & M_RIGHT) ? right : 0.f);
                sum = sum + ((m & M_LEFT) ? left : 0.f);
                if constexpr (DIM == 3) {
                    sum = sum + ((m & M_FRONT) ? f4(cur.pf, k) : 0.f);
                    sum = sum + ((m & M_BACK) ? f4(pk, k) : 0.f);
                }
            }
            out[k] = wr[k] ? div_by_count(sum - f4(cur.rhs, k), fs) : 0.f;
        }
        if (INIT) {
            *reinterpret_cast<float4*>(pc + i) = make_float4(out[0], out[1], out[2], out[3]);
            *reinterpret_cast<float4*>(zo + i) = zero;
        } else if (wr[0] && wr[1] && wr[2] && wr[3]) {
            *reinterpret_cast<float4*>(pc + i) = make_float4(out[0], out[1], out[2], out[3]);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (wr[k]) pc[i + k] = out[k];
        }
        pk = pm;
        pm = cur.pf;
        cur = nxt;
    }
}

// Residual of the fine cells under four consecutive coarse cells of a row,
// restricted: per fine row the even-x cells sit in one colour array and the
// odd-x cells in the other, both at the coarse x index.
template <int DIM, bool POW2, typename T = float, bool ZERO = false>
__global__ void __launch_bounds__(256, 3) k_rb_residual_restrict4(const float* __restrict__ p_red, const float* __restrict__ p_black,
                                                               const float* __restrict__ rr_red, const float* __restrict__ rr_black,
                                                               const uint8_t* __restrict__ m_red, const uint8_t* __restrict__ m_black,
                                                               RBLevel g, T* __restrict__ rc, int cx, int cy,
                                                               float hh, float inv_hh, const float* __restrict__ scale,
                                                               T* __restrict__ pz) {
    pdl_entry();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y * blockDim.y + threadIdx.y;
    const int Z = blockIdx.z;
    if (q >= (cx >> 2) || Y >= cy) return;
    const int X0 = q << 2;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    const int pl = g.ny * g.half;
    float v[2][2][2][4];   // [dz][dy][dx][k]
#pragma unroll
    for (int dz = 0; dz < (DIM == 3 ? 2 : 1); ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            const int y = 2 * Y + dy, z = DIM == 3 ? 2 * Z + dz : 0;
            const int c0 = (y + z) & 1;   // colour of the even-x cells of this row
            const float* A0 = c0 ? p_black : p_red;
            const float* A1 = c0 ? p_red : p_black;
            const int i = (z * g.ny + y) * g.half + X0;
            // own row: even cells in A0, odd cells in A1; neighbouring rows swap
            const float4 e_m = ldg4(A0 + i), o_m = ldg4(A1 + i);
            const bool up = y + 1 < g.ny, dn = y > 0;
            const float4 e_t = up ? ldg4(A1 + i + g.half) : zero, o_t = up ? ldg4(A0 + i + g.half) : zero;
            const float4 e_b = dn ? ldg4(A1 + i - g.half) : zero, o_b = dn ? ldg4(A0 + i - g.half) : zero;
            float4 e_f = zero, o_f = zero, e_k = zero, o_k = zero;
            if constexpr (DIM == 3) {
                if (z + 1 < g.nz) { e_f = ldg4(A1 + i + pl); o_f = ldg4(A0 + i + pl); }
                if (z > 0) { e_k = ldg4(A1 + i - pl); o_k = ldg4(A0 + i - pl); }
            }
            const float o_left = X0 > 0 ? __ldg(A1 + i - 1) : 0.f;            // x = 2*X0 - 1
            const float e_right = X0 + 4 < g.half ? __ldg(A0 + i + 4) : 0.f;   // x = 2*X0 + 8
            const uint32_t me = __ldg(reinterpret_cast<const uint32_t*>((c0 ? m_black : m_red) + i));
            const uint32_t mo = __ldg(reinterpret_cast<const uint32_t*>((c0 ? m_red : m_black) + i));
            const float4 re = ldg4((c0 ? rr_black : rr_red) + i);
            const float4 ro = ldg4((c0 ? rr_red : rr_black) + i);
#pragma unroll
            for (int dx = 0; dx < 2; ++dx)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint32_t m = ((dx ? mo : me) >> (8 * k)) & 0xFFu;
                    float res = 0.f;
                    if (m & M_FLUID) {
                        float top, bot, left, right, front = 0.f, back = 0.f, own, rr;
                        if (dx == 0) {
                            top = f4(e_t, k); bot = f4(e_b, k);
                            left = k ? f4(o_m, k - 1) : o_left;
                            right = f4(o_m, k);
                            if constexpr (DIM == 3) { front = f4(e_f, k); back = f4(e_k, k); }
                            own = f4(e_m, k); rr = f4(re, k);
                        } else {
                            top = f4(o_t, k); bot = f4(o_b, k);
                            left = f4(e_m, k);
                            right = k < 3 ? f4(e_m, k + 1) : e_right;
                            if constexpr (DIM == 3) { front = f4(o_f, k); back = f4(o_k, k); }
                            own = f4(o_m, k); rr = f4(ro, k);
                        }
                        float sum;
                        if constexpr (ZERO) {   // non-fluid neighbours hold +0
                            sum = top + bot;
                            sum = sum + right;
                            sum = sum + left;
                            if constexpr (DIM == 3) {
                                sum = sum + front;
                                sum = sum + back;
                            }
                        } else {
                            sum = ((m & M_TOP) ? top : 0.f) + ((m & M_BOTTOM) ? bot : 0.f);
                            sum = sum + ((m & M_RIGHT) ? right : 0.f);
                            sum = sum + ((m & M_LEFT) ? left : 0.f);
                            if constexpr (DIM == 3) {
                                sum = sum + ((m & M_FRONT) ? front : 0.f);
                                sum = sum + ((m & M_BACK) ? back : 0.f);
                            }
                        }
                        const float f_sum = (float)__popc(m & 0x7Eu);
                        const float lap = sum - f_sum * own;
                        res = rr - (POW2 ? lap * inv_hh : lap / hh);
                    }
                    v[dz][dy][dx][k] = res;
                }
        }
    float out[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if constexpr (DIM == 3) {
            const float bottom = v[0][0][0][k] + v[1][0][0][k] + v[0][0][1][k] + v[1][0][1][k];
            const float top = v[0][1][0][k] + v[1][1][0][k] + v[0][1][1][k] + v[1][1][1][k];
            out[k] = (bottom + top) / 8.f;
        } else {
            out[k] = (v[0][0][0][k] + v[0][0][1][k] + v[0][1][0][k] + v[0][1][1][k]) / 4.f;
        }
    }
    T* dst = rc + (Z * cy + Y) * cx + X0;
    if constexpr (std::is_same<T, float>::value) {
        *reinterpret_cast<float4*>(dst) = make_float4(out[0], out[1], out[2], out[3]);
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) dst[k] = st<T>(out[k] * scale[0]);
    }
    // the coarse level's initial guess (+0), in place of a separate clear
    if (pz) {
        T* zp = pz + (Z * cy + Y) * cx + X0;
#pragma unroll
        for (int k = 0; k < 4; ++k) zp[k] = st<T>(0.f);
    }
}

// prolong_pressure.comp:39-51 for the fine cells under four consecutive
// coarse cells of a row; interpolation weights come from per-axis tables
// computed with the same float expression as k_rb_prolong (whose lower
// coarse index is x/2 - 1 + (x & 1), checked on the host when the tables are
// made).
// ZERO: non-fluid cells get +0 instead (the mixed solve's correction there
// is never read; the select-free operators above rely on it being +0)
template <int DIM, typename T = float, bool ZERO = false>
__global__ void __launch_bounds__(256) k_rb_prolong4(float* __restrict__ p_red, float* __restrict__ p_black, RBLevel g,
                                                     const T* __restrict__ pc, int cx, int cy, int cz,
                                                     const float* __restrict__ pw, const float* __restrict__ scale,
                                                     const uint8_t* __restrict__ m_red = nullptr,
                                                     const uint8_t* __restrict__ m_black = nullptr) {
    pdl_entry();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y * blockDim.y + threadIdx.y;
    const int Z = blockIdx.z;
    if (q >= (cx >> 2) || Y >= cy) return;
    const int X0 = q << 2;
    const float* wxt = pw;
    const float* wyt = pw + g.nx;
    const float* wzt = pw + g.nx + g.ny;
    const int Ys[3] = {max(Y - 1, 0), Y, min(Y + 1, cy - 1)};
    const int Zs[3] = {max(Z - 1, 0), Z, min(Z + 1, cz - 1)};
    const int xl = max(X0 - 1, 0), xr = min(X0 + 4, cx - 1);
    float wx[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) wx[j] = __ldg(wxt + 2 * X0 + j);
#pragma unroll
    for (int ez = 0; ez < (DIM == 3 ? 2 : 1); ++ez) {
        const int z = DIM == 3 ? 2 * Z + ez : 0;
        const float wz = DIM == 3 ? __ldg(wzt + z) : 0.f;
        float R[2][3][6];   // [plane za/zb][row Y-1..Y+1][x X0-1..X0+4]
#pragma unroll
        for (int pz = 0; pz < (DIM == 3 ? 2 : 1); ++pz)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int base = ((DIM == 3 ? Zs[ez + pz] : 0) * cy + Ys[r]) * cx;
                if constexpr (std::is_same<T, float>::value) {
                    const float4 c = ldg4(pc + base + X0);
                    R[pz][r][1] = c.x; R[pz][r][2] = c.y; R[pz][r][3] = c.z; R[pz][r][4] = c.w;
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k) R[pz][r][1 + k] = ld(pc[base + X0 + k]);
                }
                R[pz][r][0] = ld(pc[base + xl]);
                R[pz][r][5] = ld(pc[base + xr]);
            }
#pragma unroll
        for (int ey = 0; ey < 2; ++ey) {
            const int y = 2 * Y + ey;
            const float wy = __ldg(wyt + y);
            float se[4], so[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int lo = k + e, hi = k + e + 1;
                    const float w = wx[2 * k + e];
                    float sv = lerp_(lerp_(R[0][ey][lo], R[0][ey][hi], w), lerp_(R[0][ey + 1][lo], R[0][ey + 1][hi], w), wy);
                    if constexpr (DIM == 3) {
                        const float c1 = lerp_(lerp_(R[1][ey][lo], R[1][ey][hi], w), lerp_(R[1][ey + 1][lo], R[1][ey + 1][hi], w), wy);
                        sv = lerp_(sv, c1, wz);
                    }
                    if constexpr (!std::is_same<T, float>::value) sv = sv * scale[1];
                    (e ? so : se)[k] = sv;
                }
            const int c0 = (y + z) & 1;
            float* E = c0 ? p_black : p_red;
            float* O = c0 ? p_red : p_black;
            const int i = (z * g.ny + y) * g.half + X0;
            float4 a = *reinterpret_cast<const float4*>(E + i);
            a.x = a.x + se[0]; a.y = a.y + se[1]; a.z = a.z + se[2]; a.w = a.w + se[3];
            float4 b = *reinterpret_cast<const float4*>(O + i);
            b.x = b.x + so[0]; b.y = b.y + so[1]; b.z = b.z + so[2]; b.w = b.w + so[3];
            if constexpr (ZERO) {
                const uint32_t me = __ldg(reinterpret_cast<const uint32_t*>((c0 ? m_black : m_red) + i));
                const uint32_t mo = __ldg(reinterpret_cast<const uint32_t*>((c0 ? m_red : m_black) + i));
                a.x = (me & 0x1u) ? a.x : 0.f; a.y = (me & 0x100u) ? a.y : 0.f;
                a.z = (me & 0x10000u) ? a.z : 0.f; a.w = (me & 0x1000000u) ? a.w : 0.f;
                b.x = (mo & 0x1u) ? b.x : 0.f; b.y = (mo & 0x100u) ? b.y : 0.f;
                b.z = (mo & 0x10000u) ? b.z : 0.f; b.w = (mo & 0x1000000u) ? b.w : 0.f;
            }
            *reinterpret_cast<float4*>(E + i) = a;
            *reinterpret_cast<float4*>(O + i) = b;
        }
    }
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

int launch_rb_sweep(ss_sim* s, int iterations, cudaStream_t st, bool zero, bool from_zero) {
    const RBLevel g = rb_level(s);
    const size_t h = s->ncell / 2;
    float* p[2] = {s->p_alt[0], s->p_alt[0] + h};
    const float* rhs[2] = {s->rhs_s, s->rhs_s + h};
    const uint8_t* mask[2] = {s->rb_mask, s->rb_mask + h};
    dim3 b, gr;
    row_launch(s->rb_vec ? g.half / 4 : g.half, g.ny, g.nz, b, gr);
    // z planes per thread of the four-cell kernel: about three waves of
    // four 256-thread blocks per SM
    int planes = 1;
    if (s->rb_vec && s->dim == 3) {
        const long long per_plane = (long long)gr.x * gr.y;
        planes = (int)std::max(1LL, std::min(16LL, per_plane * g.nz / (148LL * 4 * 3)));
    }
    dim3 gr4(gr.x, gr.y, (g.nz + planes - 1) / planes);
    // from a zero pressure: the first red half-sweep of the four-cell kernel
    // clears the black array itself; otherwise both arrays are cleared first
    const bool init = from_zero && s->rb_vec && iterations > 0;
    if (from_zero && !init) {
        const cudaError_t e = cudaMemsetAsync(s->p_alt[0], 0, s->ncell * sizeof(float), st);
        if (e != cudaSuccess) return check_cuda(e, "clear level-0 pressure");
    }
    for (int it = 0; it < iterations; ++it)
        for (int c = 0; c < 2; ++c) {
            if (init && it == 0 && c == 0) {
                if (s->dim == 3) {
                    if (zero) launch_k(s->pdl, gr4, b, 0, st, k_rb_smooth4<3, true, true>, p[c], p[1 - c], rhs[c], mask[c], g, c, planes, p[1 - c]);
                    else launch_k(s->pdl, gr4, b, 0, st, k_rb_smooth4<3, false, true>, p[c], p[1 - c], rhs[c], mask[c], g, c, planes, p[1 - c]);
                } else {
                    launch_k(s->pdl, gr4, b, 0, st, k_rb_smooth4<2, false, true>, p[c], p[1 - c], rhs[c], mask[c], g, c, planes, p[1 - c]);
                }
            } else if (s->rb_vec) {
                if (s->dim == 3) {
                    if (zero) launch_k(s->pdl, gr4, b, 0, st, k_rb_smooth4<3, true>, p[c], p[1 - c], rhs[c], mask[c], g, c, planes, nullptr);
                    else launch_k(s->pdl, gr4, b, 0, st, k_rb_smooth4<3>, p[c], p[1 - c], rhs[c], mask[c], g, c, planes, nullptr);
                } else {
                    if (zero) launch_k(s->pdl, gr4, b, 0, st, k_rb_smooth4<2, true>, p[c], p[1 - c], rhs[c], mask[c], g, c, planes, nullptr);
                    else launch_k(s->pdl, gr4, b, 0, st, k_rb_smooth4<2>, p[c], p[1 - c], rhs[c], mask[c], g, c, planes, nullptr);
                }
            } else {
                if (s->dim == 3) launch_k(s->pdl, gr, b, 0, st, k_rb_smooth<3>, p[c], p[1 - c], rhs[c], mask[c], g, c);
                else launch_k(s->pdl, gr, b, 0, st, k_rb_smooth<2>, p[c], p[1 - c], rhs[c], mask[c], g, c);
            }
        }
    s->nlaunch += 2 * iterations;
    return check_cuda(cudaGetLastError(), "k_rb_smooth");
}

static bool pow2f(float v) {
    if (!(v > 0.f) || !isfinite(v)) return false;
    int e;
    return frexpf(v, &e) == 0.5f && v >= 1.1754944e-38f && v <= 1e30f;
}

// pz: also set the next level's pressure (its initial guess) to +0
template <typename T>
static int rb_residual_restrict_t(ss_sim* s, T* rc, const float* scale, cudaStream_t st, bool zero = false,
                                  T* pz = nullptr) {
    const RBLevel g = rb_level(s);
    const size_t h = s->ncell / 2;
    const int cx = s->lv[1].n[0], cy = s->lv[1].n[1], cz = s->lv[1].n[2];
    const float hh = s->lv[0].hh;
    const bool p2 = pow2f(hh);
    const float ih = p2 ? 1.f / hh : 0.f;
    dim3 b, gr;
    const float* pr = s->p_alt[0];
    const float* pb = pr + h;
    const float* rr = s->rhs_r_is_s ? s->rhs_s : s->rhs_r;
    const uint8_t* mr = s->rb_mask;
    const uint8_t* mb = s->rb_mask + h;
    if (s->rb_vec) {
        row_launch(cx / 4, cy, cz, b, gr);
        if (s->dim == 3 && zero) {
            if (p2) launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict4<3, true, T, true>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, hh, ih, scale, pz);
            else launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict4<3, false, T, true>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, hh, ih, scale, pz);
        } else if (s->dim == 3) {
            if (p2) launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict4<3, true, T>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, hh, ih, scale, pz);
            else launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict4<3, false, T>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, hh, ih, scale, pz);
        } else {
            if (p2) launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict4<2, true, T>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, hh, ih, scale, pz);
            else launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict4<2, false, T>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, hh, ih, scale, pz);
        }
        s->nlaunch += 1;
        return check_cuda(cudaGetLastError(), "k_rb_residual_restrict4");
    }
    if (pz) {
        const cudaError_t e = cudaMemsetAsync(pz, 0, (size_t)cx * cy * cz * sizeof(T), st);
        if (e != cudaSuccess) return check_cuda(e, "clear coarse p");
    }
    row_launch(cx, cy, cz, b, gr);
    if (s->dim == 3) {
        if (p2) launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict<3, true, T>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, cz, hh, ih, scale);
        else launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict<3, false, T>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, cz, hh, ih, scale);
    } else {
        if (p2) launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict<2, true, T>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, cz, hh, ih, scale);
        else launch_k(s->pdl, gr, b, 0, st, k_rb_residual_restrict<2, false, T>, pr, pb, rr, rr + h, mr, mb, g, rc, cx, cy, cz, hh, ih, scale);
    }
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_rb_residual_restrict");
}

template <typename T>
static int rb_prolong_t(ss_sim* s, const T* pc, const float* scale, cudaStream_t st, bool zero = false) {
    const RBLevel g = rb_level(s);
    const size_t h = s->ncell / 2;
    const int cx = s->lv[1].n[0], cy = s->lv[1].n[1], cz = s->lv[1].n[2];
    if (s->rb_prolong_vec) {
        dim3 b, gr;
        row_launch(cx / 4, cy, cz, b, gr);
        if (s->dim == 3 && zero)
            launch_k(s->pdl, gr, b, 0, st, k_rb_prolong4<3, T, true>, s->p_alt[0], s->p_alt[0] + h, g, pc, cx, cy, cz, s->rb_pw,
                     scale, s->rb_mask, s->rb_mask + h);
        else if (s->dim == 3)
            launch_k(s->pdl, gr, b, 0, st, k_rb_prolong4<3, T>, s->p_alt[0], s->p_alt[0] + h, g, pc, cx, cy, cz, s->rb_pw,
                     scale, nullptr, nullptr);
        else
            launch_k(s->pdl, gr, b, 0, st, k_rb_prolong4<2, T>, s->p_alt[0], s->p_alt[0] + h, g, pc, cx, cy, cz, s->rb_pw,
                     scale, nullptr, nullptr);
        s->nlaunch += 1;
        return check_cuda(cudaGetLastError(), "k_rb_prolong4");
    }
    dim3 b(128), gr((g.nx + 127) / 128, g.ny, g.nz);
    if (s->dim == 3) launch_k(s->pdl, gr, b, 0, st, k_rb_prolong<3, T>, s->p_alt[0], s->p_alt[0] + h, g, pc, cx, cy, cz, scale);
    else launch_k(s->pdl, gr, b, 0, st, k_rb_prolong<2, T>, s->p_alt[0], s->p_alt[0] + h, g, pc, cx, cy, cz, scale);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_rb_prolong");
}

int launch_rb_residual_restrict(ss_sim* s, cudaStream_t st) { return rb_residual_restrict_t<float>(s, s->r[1], nullptr, st); }

int launch_rb_prolong(ss_sim* s, cudaStream_t st) { return rb_prolong_t<float>(s, s->p[1], nullptr, st); }

// The correction solve's level 0 may take the select-free operators when
// its prolongation zeroes non-fluid cells (the four-cells-a-thread forms of
// all three operators, 3D).
bool rb_zero_form(const ss_sim* s) { return s->dim == 3 && s->rb_vec && s->rb_prolong_vec; }

int launch_rb_residual_restrict_mixed(ss_sim* s, int prec, cudaStream_t st) {
    const bool z = rb_zero_form(s);
    if (prec == SS_PREC_MIXED)
        return rb_residual_restrict_t<__half>(s, (__half*)s->cr[1], s->d_scale, st, z, (__half*)s->cp[1]);
    return rb_residual_restrict_t<__nv_bfloat16>(s, (__nv_bfloat16*)s->cr[1], s->d_scale, st, z,
                                                 (__nv_bfloat16*)s->cp[1]);
}

int launch_rb_prolong_mixed(ss_sim* s, int prec, cudaStream_t st) {
    const bool z = rb_zero_form(s);
    if (prec == SS_PREC_MIXED) return rb_prolong_t<__half>(s, (const __half*)s->cp[1], s->d_scale, st, z);
    return rb_prolong_t<__nv_bfloat16>(s, (const __nv_bfloat16*)s->cp[1], s->d_scale, st, z);
}

// Per-axis weight of the fine cell's coarse interpolation, the float
// expression of k_rb_prolong; returns false when the lower coarse index does
// not follow x/2 - 1 + (x & 1) (clamped) on this axis.
static bool prolong_axis_table(int n, int c, float* w) {
    if (n != 2 * c || c < 1) return false;
    for (int x = 0; x < n; ++x) {
        volatile float a = (float)x + 0.5f;
        volatile float b = a / (float)n;
        volatile float t = b * (float)c;
        volatile float tx = t - 0.5f;
        const float fx = floorf(tx);
        if ((int)fx != x / 2 - 1 + (x & 1)) return false;
        volatile float wv = tx - fx;
        w[x] = wv;
    }
    return true;
}

int rb_init_vector_paths(ss_sim* s, cudaStream_t st) {
    s->rb_vec = (s->nx % 8) == 0 ? 1 : 0;
    s->rb_prolong_vec = 0;
    if (!s->rb_vec) return SS_OK;
    const int nx = s->lv[0].n[0], ny = s->lv[0].n[1], nz = s->lv[0].n[2];
    const int cx = s->lv[1].n[0], cy = s->lv[1].n[1], cz = s->lv[1].n[2];
    std::vector<float> w((size_t)nx + ny + nz, 0.f);
    bool ok = prolong_axis_table(nx, cx, w.data()) && prolong_axis_table(ny, cy, w.data() + nx);
    if (s->dim == 3) ok = ok && prolong_axis_table(nz, cz, w.data() + nx + ny);
    if (!ok) return SS_OK;
    int rc = check_cuda(cudaMalloc((void**)&s->rb_pw, w.size() * sizeof(float)), "cudaMalloc");
    if (rc) return rc;
    rc = check_cuda(cudaMemcpyAsync(s->rb_pw, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, st), "weights upload");
    if (rc) return rc;
    rc = check_cuda(cudaStreamSynchronize(st), "weights upload");
    if (!rc) s->rb_prolong_vec = 1;
    return rc;
}

}  // namespace ss
