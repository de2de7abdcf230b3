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
#include <cuda_bf16.h>
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

// Entry of a kernel that may be launched as a programmatic dependent (launch_k):
// wait until the grid before it on the stream has completed and its memory
// is visible, then allow the grid after it to be scheduled (it waits the same
// way).  No effect in a plain launch.
SS_D void pdl_entry() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

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


// ---------------------------------------------------------------------------
// Specialised forms of sample_border at the points the kernels actually use.
// At a MAC face or cell centre every texel-space coordinate is an integer or
// an integer + 1/2, so each linear weight is exactly 0 or 0.5.  A weight-0
// lerp a*(1-0) + b*0 equals a (for finite b), so skipping those taps gives the
// same value as the generic 8-tap form; the remaining lerps are kept in the
// generic x-then-y-then-z nesting.

// value of a[x,y,z] or the border when out of range
SS_D float at_b(const float* __restrict__ a, int ax, int ay, int az, int x, int y, int z) {
    return fetch_b(a, ax, ay, az, x, y, z, 0.f);
}

// Velocity at the x face (i, j+1/2, k+1/2)
template <int DIM>
SS_D void vel_at_xface(const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                       int nx, int ny, int nz, int i, int j, int k, float out[3]) {
    out[0] = __ldg(u + idx3(i, j, k, nx + 1, ny));
    // v at texel (i-1/2, j+1/2, k): x and y at 0.5
    out[1] = lerp_(lerp_(at_b(v, nx, ny + 1, nz, i - 1, j, k), at_b(v, nx, ny + 1, nz, i, j, k), 0.5f),
                   lerp_(at_b(v, nx, ny + 1, nz, i - 1, j + 1, k), at_b(v, nx, ny + 1, nz, i, j + 1, k), 0.5f), 0.5f);
    if constexpr (DIM == 3) {
        // w at texel (i-1/2, j, k+1/2): x and z at 0.5
        out[2] = lerp_(lerp_(at_b(w, nx, ny, nz + 1, i - 1, j, k), at_b(w, nx, ny, nz + 1, i, j, k), 0.5f),
                       lerp_(at_b(w, nx, ny, nz + 1, i - 1, j, k + 1), at_b(w, nx, ny, nz + 1, i, j, k + 1), 0.5f), 0.5f);
    } else {
        out[2] = 0.f;
    }
}

// Velocity at the y face (i+1/2, j, k+1/2)
template <int DIM>
SS_D void vel_at_yface(const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                       int nx, int ny, int nz, int i, int j, int k, float out[3]) {
    // u at texel (i+1/2, j-1/2, k)
    out[0] = lerp_(lerp_(at_b(u, nx + 1, ny, nz, i, j - 1, k), at_b(u, nx + 1, ny, nz, i + 1, j - 1, k), 0.5f),
                   lerp_(at_b(u, nx + 1, ny, nz, i, j, k), at_b(u, nx + 1, ny, nz, i + 1, j, k), 0.5f), 0.5f);
    out[1] = __ldg(v + idx3(i, j, k, nx, ny + 1));
    if constexpr (DIM == 3) {
        // w at texel (i, j-1/2, k+1/2): y and z at 0.5
        out[2] = lerp_(lerp_(at_b(w, nx, ny, nz + 1, i, j - 1, k), at_b(w, nx, ny, nz + 1, i, j, k), 0.5f),
                       lerp_(at_b(w, nx, ny, nz + 1, i, j - 1, k + 1), at_b(w, nx, ny, nz + 1, i, j, k + 1), 0.5f), 0.5f);
    } else {
        out[2] = 0.f;
    }
}

// Velocity at the z face (i+1/2, j+1/2, k)
SS_D void vel_at_zface(const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                       int nx, int ny, int nz, int i, int j, int k, float out[3]) {
    // u at texel (i+1/2, j, k-1/2): x and z at 0.5
    out[0] = lerp_(lerp_(at_b(u, nx + 1, ny, nz, i, j, k - 1), at_b(u, nx + 1, ny, nz, i + 1, j, k - 1), 0.5f),
                   lerp_(at_b(u, nx + 1, ny, nz, i, j, k), at_b(u, nx + 1, ny, nz, i + 1, j, k), 0.5f), 0.5f);
    // v at texel (i, j+1/2, k-1/2): y and z at 0.5
    out[1] = lerp_(lerp_(at_b(v, nx, ny + 1, nz, i, j, k - 1), at_b(v, nx, ny + 1, nz, i, j + 1, k - 1), 0.5f),
                   lerp_(at_b(v, nx, ny + 1, nz, i, j, k), at_b(v, nx, ny + 1, nz, i, j + 1, k), 0.5f), 0.5f);
    out[2] = __ldg(w + idx3(i, j, k, nx, ny));
}

// The same three face velocities for a face whose every tap is inside the
// arrays (1 <= i, j, k and i < nx, j < ny, k < nz): direct loads, no border
// checks - the values (and lerp order) of vel_at_*face.
template <int DIM>
SS_D void vel_at_face_interior(const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                               int nx, int ny, int nz, int comp, int i, int j, int k, float out[3]) {
    const int ux = nx + 1, vy = ny + 1;
    if (comp == 0) {
        out[0] = __ldg(u + idx3(i, j, k, ux, ny));
        const float* pv = v + idx3(i - 1, j, k, nx, vy);
        out[1] = lerp_(lerp_(__ldg(pv), __ldg(pv + 1), 0.5f), lerp_(__ldg(pv + nx), __ldg(pv + nx + 1), 0.5f), 0.5f);
        if constexpr (DIM == 3) {
            const float* pw = w + idx3(i - 1, j, k, nx, ny);
            const int pl = nx * ny;
            out[2] = lerp_(lerp_(__ldg(pw), __ldg(pw + 1), 0.5f), lerp_(__ldg(pw + pl), __ldg(pw + pl + 1), 0.5f), 0.5f);
        } else {
            out[2] = 0.f;
        }
    } else if (comp == 1) {
        const float* pu = u + idx3(i, j - 1, k, ux, ny);
        out[0] = lerp_(lerp_(__ldg(pu), __ldg(pu + 1), 0.5f), lerp_(__ldg(pu + ux), __ldg(pu + ux + 1), 0.5f), 0.5f);
        out[1] = __ldg(v + idx3(i, j, k, nx, vy));
        if constexpr (DIM == 3) {
            const float* pw = w + idx3(i, j - 1, k, nx, ny);
            const int pl = nx * ny;
            out[2] = lerp_(lerp_(__ldg(pw), __ldg(pw + nx), 0.5f), lerp_(__ldg(pw + pl), __ldg(pw + pl + nx), 0.5f), 0.5f);
        } else {
            out[2] = 0.f;
        }
    } else {
        const int plu = ux * ny, plv = nx * vy;
        const float* pu = u + idx3(i, j, k - 1, ux, ny);
        out[0] = lerp_(lerp_(__ldg(pu), __ldg(pu + 1), 0.5f), lerp_(__ldg(pu + plu), __ldg(pu + plu + 1), 0.5f), 0.5f);
        const float* pv = v + idx3(i, j, k - 1, nx, vy);
        out[1] = lerp_(lerp_(__ldg(pv), __ldg(pv + nx), 0.5f), lerp_(__ldg(pv + plv), __ldg(pv + plv + nx), 0.5f), 0.5f);
        out[2] = __ldg(w + idx3(i, j, k, nx, ny));
    }
}

// Velocity at the cell centre (i+1/2, j+1/2, k+1/2): each component is the
// mean of the cell's two faces on its axis.
template <int DIM>
SS_D void vel_at_centre(const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
                        int nx, int ny, int nz, int i, int j, int k, float out[3]) {
    out[0] = lerp_(__ldg(u + idx3(i, j, k, nx + 1, ny)), __ldg(u + idx3(i + 1, j, k, nx + 1, ny)), 0.5f);
    out[1] = lerp_(__ldg(v + idx3(i, j, k, nx, ny + 1)), __ldg(v + idx3(i, j + 1, k, nx, ny + 1)), 0.5f);
    if constexpr (DIM == 3) out[2] = lerp_(__ldg(w + idx3(i, j, k, nx, ny)), __ldg(w + idx3(i, j, k + 1, nx, ny)), 0.5f);
    else out[2] = 0.f;
}

// Border sample with a branch-free interior fast path: when all taps are in
// range one base address serves the 8 (4) loads.
// 0 <= v && v + 1 < n, as one unsigned comparison (v is a clamped tap index)
SS_D bool tap_pair_in(int v, int n) { return (unsigned)v < (unsigned)(n - 1); }

template <int DIM>
SS_D float sample_taps_fast(const float* __restrict__ a, int ax, int ay, int az, const Taps& t, float border) {
    const bool in = tap_pair_in(t.x0, ax) && tap_pair_in(t.y0, ay) && (DIM == 2 || tap_pair_in(t.z0, az));
    if (!in) return sample_taps<DIM>(a, ax, ay, az, t, border);
    const float* p = a + idx3(t.x0, t.y0, t.z0, ax, ay);
    const float c00 = __ldg(p), c10 = __ldg(p + 1), c01 = __ldg(p + ax), c11 = __ldg(p + ax + 1);
    if constexpr (DIM == 2) {
        return lerp_(lerp_(c00, c10, t.wx), lerp_(c01, c11, t.wx), t.wy);
    } else {
        const int pl = ax * ay;
        const float d00 = __ldg(p + pl), d10 = __ldg(p + pl + 1), d01 = __ldg(p + pl + ax), d11 = __ldg(p + pl + ax + 1);
        const float c0 = lerp_(lerp_(c00, c10, t.wx), lerp_(c01, c11, t.wx), t.wy);
        const float c1 = lerp_(lerp_(d00, d10, t.wx), lerp_(d01, d11, t.wx), t.wy);
        return lerp_(c0, c1, t.wz);
    }
}

SS_D float round_half(float x) { return __half2float(__float2half_rn(x)); }

// Storage types of the coarse multigrid levels: FP32, or FP16 / BF16 for the
// corrections of the mixed-precision solve.  Arithmetic is FP32 throughout;
// ld converts a stored value to float, st rounds to nearest even on store and
// rnd<T> gives the float value that storing as T would keep.
SS_D float ld(float v) { return v; }
SS_D float ld(__half v) { return __half2float(v); }
SS_D float ld(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename T> SS_D T st(float v);
template <> SS_D float st<float>(float v) { return v; }
template <> SS_D __half st<__half>(float v) { return __float2half_rn(v); }
template <> SS_D __nv_bfloat16 st<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <typename T> SS_D float rnd(float v) { return ld(st<T>(v)); }

// Sum of n per-block partials by one block's threads, each
// thread keeping eight independent accumulators so its L2 loads are in
// flight together; the order depends only on n and the thread count.
SS_D double fold_sum(const double* p, unsigned int n, unsigned int tid, unsigned int nt) {
    double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    unsigned int i = tid;
    for (; i + 7 * nt < n; i += 8 * nt) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] += __ldcg(p + i + k * nt);
    }
    for (; i < n; i += nt) a[0] += __ldcg(p + i);
    return ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
}
// a float4 through the read-only path, and lane k of a float4
SS_D float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
SS_D float f4(const float4& v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

// a / f for an integer count f in 1..6, bit-identical to the IEEE quotient
// for every finite a: q0 = a*RN(1/f) followed by one residual correction with
// fused multiply-adds - the FMA-based correctly rounded division of P.
// Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990, with the reciprocal of a small
// integer as its start value - verified exhaustively against IEEE division
// over every finite float a for f = 1..6 (tests/division_check.c).  A zero a
// is returned as it is (the correction would turn -0 into +0).  For f = 6 it
// divides a/2 by 3, exact except where a/2 is subnormal: |a| < 2^-120 (zeros
// included) takes the IEEE path.  An infinite a gives NaN.
SS_D float div_by_count(float a, int f) {
    if (f == 6) {
        // the f = 3 steps below on a/2, written out so the interior cells'
        // path carries no selection of the reciprocal
        if (fabsf(a) < 7.52316385e-37f) return a / 6.f;
        const float h = a * 0.5f;
        const float q0 = __fmul_rn(h, 1.0f / 3.0f);
        const float r = __fmaf_rn(-3.0f, q0, h);
        return __fmaf_rn(r, 1.0f / 3.0f, q0);
    }
    if (a == 0.f) return a;
    const float y = f == 1 ? 1.f : f == 2 ? 0.5f : f == 3 ? (1.0f / 3.0f) : f == 4 ? 0.25f : (1.0f / 5.0f);
    const float q0 = __fmul_rn(a, y);
    const float r = __fmaf_rn(-(float)f, q0, a);
    return __fmaf_rn(r, y, q0);
}

// Fluid mask byte of a level-0 cell: bit 0 the cell is fluid, bits 1-6 the
// +y,-y,+x,-x,+z,-z neighbour is fluid (out of grid: fluid on an open grid,
// solid on an enclosed one).  Zero - the TMA fill outside the grid - reads as
// "not fluid", so tile kernels need no bounds checks.
enum : uint8_t {
    M_FLUID = 1u << 0,
    M_TOP = 1u << 1,
    M_BOTTOM = 1u << 2,
    M_RIGHT = 1u << 3,
    M_LEFT = 1u << 4,
    M_FRONT = 1u << 5,
    M_BACK = 1u << 6,
};

}  // namespace ss
