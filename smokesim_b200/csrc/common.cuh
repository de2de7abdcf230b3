// common.cuh - device helpers shared by the smoke-step kernels.
//
// Layout: every field is a structure-of-arrays FP32 array, x fastest.  Cell
// arrays are nx*ny*nz; the MAC face arrays are one longer on their own axis.
// The level-0 solid map is one byte per cell (bit 0: this cell is solid,
// bits 1-6: the +y,-y,+x,-x,+z,-z neighbour is solid, out of grid = fluid).
//
// All arithmetic is written so that, compiled with -fmad=false and IEEE
// division / square root, each cell rounds exactly like the CPU oracle:
// same operation order, no contraction.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#define SS_HD __host__ __device__ __forceinline__
#define SS_D __device__ __forceinline__

namespace ss {

enum : uint8_t {
    F_SOLID = 1u << 0,
    F_TOP = 1u << 1,     // +y
    F_BOTTOM = 1u << 2,  // -y
    F_RIGHT = 1u << 3,   // +x
    F_LEFT = 1u << 4,    // -x
    F_FRONT = 1u << 5,   // +z
    F_BACK = 1u << 6,    // -z
};

struct Grid {
    int nx, ny, nz;   // cells (nz = 1 in 2D)
};

SS_HD int idx3(int x, int y, int z, int ax, int ay) { return (z * ay + y) * ax + x; }

SS_D float lerp_(float a, float b, float t) { return a * (1.f - t) + b * t; }

SS_D float clampt(float t, float lo, float hi) { return fminf(fmaxf(t, lo), hi); }

SS_D float fetch_b(const float* __restrict__ a, int ax, int ay, int az, int x, int y, int z, float border) {
    if (x < 0 || y < 0 || z < 0 || x >= ax || y >= ay || z >= az) return border;
    return __ldg(a + idx3(x, y, z, ax, ay));
}

// GL_LINEAR + CLAMP_TO_BORDER at texel-space coordinate (texel centres at integers).
template <int DIM>
SS_D float sample_border(const float* __restrict__ a, int ax, int ay, int az, float tx, float ty, float tz,
                         float border) {
    tx = clampt(tx, -2.f, (float)(ax + 1));
    ty = clampt(ty, -2.f, (float)(ay + 1));
    float fx = floorf(tx), fy = floorf(ty);
    int x0 = (int)fx, y0 = (int)fy;
    float wx = tx - fx, wy = ty - fy;
    if constexpr (DIM == 2) {
        float c00 = fetch_b(a, ax, ay, 1, x0, y0, 0, border), c10 = fetch_b(a, ax, ay, 1, x0 + 1, y0, 0, border);
        float c01 = fetch_b(a, ax, ay, 1, x0, y0 + 1, 0, border), c11 = fetch_b(a, ax, ay, 1, x0 + 1, y0 + 1, 0, border);
        return lerp_(lerp_(c00, c10, wx), lerp_(c01, c11, wx), wy);
    } else {
        tz = clampt(tz, -2.f, (float)(az + 1));
        float fz = floorf(tz);
        int z0 = (int)fz;
        float wz = tz - fz;
        float c000 = fetch_b(a, ax, ay, az, x0, y0, z0, border), c100 = fetch_b(a, ax, ay, az, x0 + 1, y0, z0, border);
        float c010 = fetch_b(a, ax, ay, az, x0, y0 + 1, z0, border), c110 = fetch_b(a, ax, ay, az, x0 + 1, y0 + 1, z0, border);
        float c001 = fetch_b(a, ax, ay, az, x0, y0, z0 + 1, border), c101 = fetch_b(a, ax, ay, az, x0 + 1, y0, z0 + 1, border);
        float c011 = fetch_b(a, ax, ay, az, x0, y0 + 1, z0 + 1, border), c111 = fetch_b(a, ax, ay, az, x0 + 1, y0 + 1, z0 + 1, border);
        float c0 = lerp_(lerp_(c000, c100, wx), lerp_(c010, c110, wx), wy);
        float c1 = lerp_(lerp_(c001, c101, wx), lerp_(c011, c111, wx), wy);
        return lerp_(c0, c1, wz);
    }
}

// Tap positions and weights of one border sample, shared by several channels.
struct Taps {
    int x0, y0, z0;
    float wx, wy, wz;
};

template <int DIM>
SS_D Taps make_taps(int ax, int ay, int az, float tx, float ty, float tz) {
    Taps t;
    tx = clampt(tx, -2.f, (float)(ax + 1));
    ty = clampt(ty, -2.f, (float)(ay + 1));
    float fx = floorf(tx), fy = floorf(ty);
    t.x0 = (int)fx; t.y0 = (int)fy;
    t.wx = tx - fx; t.wy = ty - fy;
    if constexpr (DIM == 3) {
        tz = clampt(tz, -2.f, (float)(az + 1));
        float fz = floorf(tz);
        t.z0 = (int)fz;
        t.wz = tz - fz;
    } else {
        t.z0 = 0; t.wz = 0.f;
    }
    return t;
}

template <int DIM>
SS_D float sample_taps(const float* __restrict__ a, int ax, int ay, int az, const Taps& t, float border) {
    const int x0 = t.x0, y0 = t.y0, z0 = t.z0;
    if constexpr (DIM == 2) {
        float c00 = fetch_b(a, ax, ay, 1, x0, y0, 0, border), c10 = fetch_b(a, ax, ay, 1, x0 + 1, y0, 0, border);
        float c01 = fetch_b(a, ax, ay, 1, x0, y0 + 1, 0, border), c11 = fetch_b(a, ax, ay, 1, x0 + 1, y0 + 1, 0, border);
        return lerp_(lerp_(c00, c10, t.wx), lerp_(c01, c11, t.wx), t.wy);
    } else {
        float c000 = fetch_b(a, ax, ay, az, x0, y0, z0, border), c100 = fetch_b(a, ax, ay, az, x0 + 1, y0, z0, border);
        float c010 = fetch_b(a, ax, ay, az, x0, y0 + 1, z0, border), c110 = fetch_b(a, ax, ay, az, x0 + 1, y0 + 1, z0, border);
        float c001 = fetch_b(a, ax, ay, az, x0, y0, z0 + 1, border), c101 = fetch_b(a, ax, ay, az, x0 + 1, y0, z0 + 1, border);
        float c011 = fetch_b(a, ax, ay, az, x0, y0 + 1, z0 + 1, border), c111 = fetch_b(a, ax, ay, az, x0 + 1, y0 + 1, z0 + 1, border);
        float c0 = lerp_(lerp_(c000, c100, t.wx), lerp_(c010, c110, t.wx), t.wy);
        float c1 = lerp_(lerp_(c001, c101, t.wx), lerp_(c011, c111, t.wx), t.wy);
        return lerp_(c0, c1, t.wz);
    }
}

// Velocity at grid-space point g (reference get_interpolated_velocity,
// shaders3d/compute/advect_vx.comp:33-46).
template <int DIM>
SS_D void interp_velocity(const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                          int nx, int ny, int nz, float gx, float gy, float gz, float out[3]) {
    if constexpr (DIM == 2) {
        out[0] = sample_border<2>(u, nx + 1, ny, 1, gx, gy - 0.5f, 0.f, 0.f);
        out[1] = sample_border<2>(v, nx, ny + 1, 1, gx - 0.5f, gy, 0.f, 0.f);
        out[2] = 0.f;
    } else {
        out[0] = sample_border<3>(u, nx + 1, ny, nz, gx, gy - 0.5f, gz - 0.5f, 0.f);
        out[1] = sample_border<3>(v, nx, ny + 1, nz, gx - 0.5f, gy, gz - 0.5f, 0.f);
        out[2] = sample_border<3>(w, nx, ny, nz + 1, gx - 0.5f, gy - 0.5f, gz, 0.f);
    }
}

SS_D float round_half(float x) { return __half2float(__float2half_rn(x)); }

}  // namespace ss
