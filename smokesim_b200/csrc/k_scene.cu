// k_scene.cu - solid map rasterisation and field initialisation.
#include "common.cuh"
#include "ss_internal.h"

namespace ss {

// init_solid_map (shaders3d/compute/init_solid_map.comp:34-48) followed by
// update_solid_map (update_solid_map.comp:46-83): wall shell when enclosed;
// spheres (last one wins) and then boxes on cells with 2 <= idx <= n-2; every
// other cell fluid.  Velocities are stored FP16-rounded like the reference's
// RGBA16F solid image.
template <int DIM>
__global__ void k_rasterize(uint8_t* __restrict__ solid, float* __restrict__ sv0, float* __restrict__ sv1,
                            float* __restrict__ sv2, int nx, int ny, int nz, int enclosed,
                            const ss_obstacle* __restrict__ ob, int no, const ss_box* __restrict__ bx, int nb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const int c = idx3(x, y, z, nx, ny);
    const bool shell = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || (DIM == 3 && (z == 0 || z == nz - 1));
    const bool invalid = x <= 1 || y <= 1 || x >= nx - 1 || y >= ny - 1 || (DIM == 3 && (z <= 1 || z >= nz - 1));
    uint8_t s = 0;
    float v[3] = {0.f, 0.f, 0.f};
    if (invalid) {
        s = (enclosed && shell) ? 1 : 0;
    } else {
        for (int i = 0; i < no; ++i) {
            const ss_obstacle& o = ob[i];
            const float dx = (float)x - o.pos[0], dy = (float)y - o.pos[1];
            float d2 = dx * dx + dy * dy;
            if constexpr (DIM == 3) { const float dz = (float)z - o.pos[2]; d2 = d2 + dz * dz; }
            if (sqrtf(d2) < o.radius) {
                const float m = 1.f - o.anchored;
                s = 1;
                v[0] = o.velocity[0] * m; v[1] = o.velocity[1] * m; v[2] = DIM == 3 ? o.velocity[2] * m : 0.f;
            }
        }
        for (int i = 0; i < nb; ++i) {
            const ss_box& b = bx[i];
            bool in = (float)x >= b.lo[0] && (float)x < b.hi[0] && (float)y >= b.lo[1] && (float)y < b.hi[1];
            if constexpr (DIM == 3) in = in && (float)z >= b.lo[2] && (float)z < b.hi[2];
            if (in) {
                const float m = 1.f - b.anchored;
                s = 1;
                v[0] = b.velocity[0] * m; v[1] = b.velocity[1] * m; v[2] = DIM == 3 ? b.velocity[2] * m : 0.f;
            }
        }
    }
    solid[c] = s;
    if (sv0) {
        sv0[c] = round_half(v[0]);
        sv1[c] = round_half(v[1]);
        if (sv2) sv2[c] = round_half(v[2]);
    }
}

// flag byte: bit 0 own solid, bits 1-6 neighbours (+y,-y,+x,-x,+z,-z), out of grid = fluid
template <int DIM>
__global__ void k_flags(const uint8_t* __restrict__ solid, uint8_t* __restrict__ flags, uint8_t* __restrict__ fmask,
                        int nx, int ny, int nz, int enclosed) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const int c = idx3(x, y, z, nx, ny);
    uint8_t f = solid[c] ? F_SOLID : 0;
    if (y + 1 < ny && solid[c + nx]) f |= F_TOP;
    if (y > 0 && solid[c - nx]) f |= F_BOTTOM;
    if (x + 1 < nx && solid[c + 1]) f |= F_RIGHT;
    if (x > 0 && solid[c - 1]) f |= F_LEFT;
    if constexpr (DIM == 3) {
        if (z + 1 < nz && solid[c + nx * ny]) f |= F_FRONT;
        if (z > 0 && solid[c - nx * ny]) f |= F_BACK;
    }
    flags[c] = f;
    if (fmask) {
        const uint8_t oob = enclosed ? 0 : 1;   // out-of-grid neighbour fluid on an open grid
        uint8_t m = solid[c] ? 0 : M_FLUID;
        m |= (y + 1 < ny ? !solid[c + nx] : oob) ? M_TOP : 0;
        m |= (y > 0 ? !solid[c - nx] : oob) ? M_BOTTOM : 0;
        m |= (x + 1 < nx ? !solid[c + 1] : oob) ? M_RIGHT : 0;
        m |= (x > 0 ? !solid[c - 1] : oob) ? M_LEFT : 0;
        if constexpr (DIM == 3) {
            m |= (z + 1 < nz ? !solid[c + nx * ny] : oob) ? M_FRONT : 0;
            m |= (z > 0 ? !solid[c - nx * ny] : oob) ? M_BACK : 0;
        }
        fmask[c] = m;
    }
}

static inline dim3 grid_for(int ax, int ay, int az, dim3 b) {
    return dim3((ax + b.x - 1) / b.x, (ay + b.y - 1) / b.y, (az + b.z - 1) / b.z);
}

int launch_rasterize(ss_sim* s, cudaStream_t st) {
    dim3 b(32, 8, 1);
    dim3 g = grid_for(s->nx, s->ny, s->nz, b);
    float* sv0 = s->svel_active ? s->svel[0] : nullptr;
    float* sv1 = s->svel_active ? s->svel[1] : nullptr;
    float* sv2 = (s->svel_active && s->dim == 3) ? s->svel[2] : nullptr;
    if (s->dim == 3)
        k_rasterize<3><<<g, b, 0, st>>>(s->solid, sv0, sv1, sv2, s->nx, s->ny, s->nz, s->enclosed, s->d_ob,
                                        (int)s->ob.size(), s->d_bx, (int)s->bx.size());
    else
        k_rasterize<2><<<g, b, 0, st>>>(s->solid, sv0, sv1, sv2, s->nx, s->ny, s->nz, s->enclosed, s->d_ob,
                                        (int)s->ob.size(), s->d_bx, (int)s->bx.size());
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_rasterize");
}

int launch_flags(ss_sim* s, cudaStream_t st) {
    dim3 b(32, 8, 1);
    dim3 g = grid_for(s->nx, s->ny, s->nz, b);
    if (s->dim == 3) k_flags<3><<<g, b, 0, st>>>(s->solid, s->flags, s->fmask, s->nx, s->ny, s->nz, s->enclosed);
    else k_flags<2><<<g, b, 0, st>>>(s->solid, s->flags, s->fmask, s->nx, s->ny, s->nz, s->enclosed);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_flags");
}

__global__ void k_fill(float* __restrict__ a, size_t n, float v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) a[i] = v;
}

int launch_fill(float* a, size_t n, float v, cudaStream_t st) {
    if (n == 0) return SS_OK;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_fill<<<blocks, 256, 0, st>>>(a, n, v);
    return check_cuda(cudaGetLastError(), "k_fill");
}

}  // namespace ss
