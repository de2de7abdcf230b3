// k_mg.cu - multigrid pressure projection kernels.
//
// Reference: the recursive V-cycle of common/physics/grid.c:173-266 over the
// pressure / residual / solid pyramid of 3d/grid3d.c:45-68, with the shaders
// of shaders{2,3}d/compute/pressure_solve/.  Level 0 reads the solid map as a
// flag byte and its right-hand side from the precomputed divergence (the
// reference recomputes it from the velocities in every sweep); coarse levels
// read the FP16-rounded solid fraction alpha (the reference stores the solid
// pyramid as RGBA16F images).
#include <algorithm>

#include <cooperative_groups.h>

#include "common.cuh"
#include "ss_internal.h"

namespace cg = cooperative_groups;

namespace ss {

#define TRY_CUDA_MG(x, what)                              \
    do {                                                  \
        const int _rc = check_cuda((x), what);            \
        if (_rc != SS_OK) return _rc;                     \
    } while (0)


// T: storage type of p and r (float, or __half / __nv_bfloat16 on the coarse
// levels of the mixed-precision solve)
template <typename T>
struct MGArgsT {
    T* __restrict__ p;
    T* __restrict__ r;              // level right-hand side / residual (L >= 1)
    const float* __restrict__ alpha;  // L >= 1
    const uint8_t* __restrict__ flags;  // L == 0
    const float* __restrict__ div0;   // L == 0, smoother rule
    const float* __restrict__ div0r;  // L == 0, residual rule
    int nx, ny, nz;
    float oobA;     // solid fraction read for out-of-grid neighbours (0 = open, 1 = wall)
    float hh;       // h_L^2
    float rho_h;    // rho * h   (L == 0 smoother)
    float dt;
    float rho;
    float dt_h;     // dt * h    (L == 0 residual)
};
using MGArgs = MGArgsT<float>;

// Out-of-grid rule: ref_quirks keeps the reference's smoother (open, p = 0) /
// residual (wall) mismatch; the corrected mode uses the physical rule of the
// grid (wall when enclosed, open otherwise) in both operators.
static float smooth_oob(const ss_sim* s, int quirks) { return quirks ? 0.f : (s->enclosed ? 1.f : 0.f); }
static float resid_oob(const ss_sim* s, int quirks) { return quirks ? 1.f : (s->enclosed ? 1.f : 0.f); }

static MGArgs mg_args(ss_sim* s, const StepConsts& c, int L, float oobA) {
    MGArgs a;
    a.oobA = oobA;
    a.p = s->p[L];
    a.r = s->r[L];
    a.alpha = L > 0 ? s->alpha[L] : nullptr;
    a.flags = s->flags;
    a.div0 = oobA != 0.f ? s->div0r : s->div0;   // level-0 right-hand side under the chosen rule
    a.div0r = a.div0;
    a.nx = s->lv[L].n[0]; a.ny = s->lv[L].n[1]; a.nz = s->lv[L].n[2];
    a.hh = s->lv[L].hh;
    a.rho_h = c.rho_h;
    a.dt = c.dt;
    a.rho = c.rho;
    a.dt_h = c.dt_h;
    return a;
}

// ------------------------------------------------------------------ smoother
// A level value as float; CG reads through L2 only (ld.global.cg), for
// arrays that other blocks of the same launch may have written since this SM
// last cached them (L1 is not coherent across SMs).
template <bool CG, typename T>
SS_D float ldv(const T* p) {
    if constexpr (CG) return ld(__ldcg(p));
    else return ld(*p);
}

// smooth.comp:79-136 (2D :74-123): red-black Gauss-Seidel in place; solid
// cells and cells without fluid neighbours are skipped; out of grid = fluid
// with p = 0.
// R: the type whose rounding every stored pressure gets (== T for global
// arrays; the shared-memory bottom solve keeps float storage rounded as R).
template <int DIM, bool L0, typename T = float, typename R = T, bool CG = false>
SS_D void smooth_cell(const MGArgsT<T>& a, int x, int y, int z) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int c = idx3(x, y, z, nx, ny);
    float f_top, f_bottom, f_right, f_left, f_front = 0.f, f_back = 0.f;
    float r_c = 0.f;
    float p_top, p_bottom, p_right, p_left, p_front = 0.f, p_back = 0.f;
    auto load_p = [&]() {
        const T* P = a.p;
        p_top = y + 1 < ny ? ldv<CG>(P + c + nx) : 0.f;
        p_bottom = y > 0 ? ldv<CG>(P + c - nx) : 0.f;
        p_right = x + 1 < nx ? ldv<CG>(P + c + 1) : 0.f;
        p_left = x > 0 ? ldv<CG>(P + c - 1) : 0.f;
        if constexpr (DIM == 3) {
            p_front = z + 1 < nz ? ldv<CG>(P + c + nx * ny) : 0.f;
            p_back = z > 0 ? ldv<CG>(P + c - nx * ny) : 0.f;
        }
    };
    if constexpr (L0) {
        const uint8_t fl = a.flags[c];
        if (fl & F_SOLID) return;
        const float fo = 1.f - a.oobA;
        f_top = (fl & F_TOP) ? 0.f : (y + 1 < ny ? 1.f : fo);
        f_bottom = (fl & F_BOTTOM) ? 0.f : (y > 0 ? 1.f : fo);
        f_right = (fl & F_RIGHT) ? 0.f : (x + 1 < nx ? 1.f : fo);
        f_left = (fl & F_LEFT) ? 0.f : (x > 0 ? 1.f : fo);
        if constexpr (DIM == 3) {
            f_front = (fl & F_FRONT) ? 0.f : (z + 1 < nz ? 1.f : fo);
            f_back = (fl & F_BACK) ? 0.f : (z > 0 ? 1.f : fo);
        }
    } else {
        // every load of the cell is issued before the solid test, so one
        // memory latency covers the fraction, pressure and residual reads
        const float a_c = a.alpha[c];
        const float a_t = y + 1 < ny ? a.alpha[c + nx] : a.oobA;
        const float a_b = y > 0 ? a.alpha[c - nx] : a.oobA;
        const float a_r = x + 1 < nx ? a.alpha[c + 1] : a.oobA;
        const float a_l = x > 0 ? a.alpha[c - 1] : a.oobA;
        float a_f = 0.f, a_k = 0.f;
        if constexpr (DIM == 3) {
            a_f = z + 1 < nz ? a.alpha[c + nx * ny] : a.oobA;
            a_k = z > 0 ? a.alpha[c - nx * ny] : a.oobA;
        }
        r_c = ldv<CG>(a.r + c);
        // the neighbours' pressures too: with CG they come from L2, and
        // issuing them here keeps the cell to one memory round trip
        load_p();
        if (a_c >= 1.f) return;
        f_top = 1.f - a_t;
        f_bottom = 1.f - a_b;
        f_right = 1.f - a_r;
        f_left = 1.f - a_l;
        if constexpr (DIM == 3) {
            f_front = 1.f - a_f;
            f_back = 1.f - a_k;
        }
    }
    if constexpr (L0) load_p();
    float f_sum = f_top + f_bottom + f_right + f_left;
    if constexpr (DIM == 3) f_sum = f_sum + f_front + f_back;
    if (f_sum == 0.f) return;
    float p_sum = p_top * f_top + p_bottom * f_bottom;
    p_sum = p_sum + p_right * f_right;
    p_sum = p_sum + p_left * f_left;
    if constexpr (DIM == 3) {
        p_sum = p_sum + p_front * f_front;
        p_sum = p_sum + p_back * f_back;
    }
    float pn;
    if constexpr (L0) pn = (p_sum - a.rho_h * a.div0[c] / a.dt) / f_sum;
    else pn = (p_sum - r_c * a.hh) / f_sum;
    a.p[c] = st<T>(rnd<R>(pn));
}

template <int DIM, bool L0, typename T = float>
__global__ void __launch_bounds__(256) k_smooth(MGArgsT<T> a, int parity) {
    pdl_entry();
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    const int x = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((y + z + parity) & 1);
    if (x >= a.nx || y >= a.ny || z >= a.nz) return;
    smooth_cell<DIM, L0, T>(a, x, y, z);
}

static inline dim3 grid_for(int ax, int ay, int az, dim3 b) {
    return dim3((ax + b.x - 1) / b.x, (ay + b.y - 1) / b.y, (az + b.z - 1) / b.z);
}

int launch_smooth(ss_sim* s, const StepConsts& c, int L, int iterations, int quirks, cudaStream_t st) {
    MGArgs a = mg_args(s, c, L, smooth_oob(s, quirks));
    dim3 b(32, 8, 1);
    dim3 g = grid_for((a.nx + 1) / 2, a.ny, a.nz, b);
    for (int it = 0; it < 2 * iterations; ++it) {
        const int parity = it & 1;
        if (s->dim == 3) {
            if (L == 0) launch_k(s->pdl, g, b, 0, st, k_smooth<3, true>, a, parity);
            else launch_k(s->pdl, g, b, 0, st, k_smooth<3, false>, a, parity);
        } else {
            if (L == 0) launch_k(s->pdl, g, b, 0, st, k_smooth<2, true>, a, parity);
            else launch_k(s->pdl, g, b, 0, st, k_smooth<2, false>, a, parity);
        }
    }
    s->nlaunch += 2 * iterations;
    return check_cuda(cudaGetLastError(), "k_smooth");
}

// ------------------------------------------------------------------ residual
// compute_residual.comp:77-130 (2D :72-117): r = b - (sum_f p_nb - f_sum p)/h^2,
// out of grid = solid; level 0 takes b = rho*div/(dt*h).
template <int DIM, bool L0, typename T = float, bool CG = false>
SS_D float residual_cell(const MGArgsT<T>& a, int x, int y, int z) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int c = idx3(x, y, z, nx, ny);
    float f_top, f_bottom, f_right, f_left, f_front = 0.f, f_back = 0.f;
    float p_top, p_bottom, p_right, p_left, p_front = 0.f, p_back = 0.f, p_c, old;
    const T* P = a.p;
    auto load_p = [&]() {
        p_top = y + 1 < ny ? ldv<CG>(P + c + nx) : 0.f;
        p_bottom = y > 0 ? ldv<CG>(P + c - nx) : 0.f;
        p_right = x + 1 < nx ? ldv<CG>(P + c + 1) : 0.f;
        p_left = x > 0 ? ldv<CG>(P + c - 1) : 0.f;
        if constexpr (DIM == 3) {
            p_front = z + 1 < nz ? ldv<CG>(P + c + nx * ny) : 0.f;
            p_back = z > 0 ? ldv<CG>(P + c - nx * ny) : 0.f;
        }
        p_c = ldv<CG>(P + c);
    };
    if constexpr (L0) {
        const uint8_t fl = a.flags[c];
        if (fl & F_SOLID) return 0.f;
        const float fo = 1.f - a.oobA;
        f_top = (fl & F_TOP) ? 0.f : (y + 1 < ny ? 1.f : fo);
        f_bottom = (fl & F_BOTTOM) ? 0.f : (y > 0 ? 1.f : fo);
        f_right = (fl & F_RIGHT) ? 0.f : (x + 1 < nx ? 1.f : fo);
        f_left = (fl & F_LEFT) ? 0.f : (x > 0 ? 1.f : fo);
        if constexpr (DIM == 3) {
            f_front = (fl & F_FRONT) ? 0.f : (z + 1 < nz ? 1.f : fo);
            f_back = (fl & F_BACK) ? 0.f : (z > 0 ? 1.f : fo);
        }
        load_p();
        old = a.rho * a.div0r[c] / a.dt_h;
    } else {
        // every load of the cell (fractions, pressures, right-hand side) is
        // issued before the solid test: one memory round trip a cell
        const float a_c = a.alpha[c];
        const float a_t = y + 1 < ny ? a.alpha[c + nx] : a.oobA;
        const float a_b = y > 0 ? a.alpha[c - nx] : a.oobA;
        const float a_r = x + 1 < nx ? a.alpha[c + 1] : a.oobA;
        const float a_l = x > 0 ? a.alpha[c - 1] : a.oobA;
        float a_f = 0.f, a_k = 0.f;
        if constexpr (DIM == 3) {
            a_f = z + 1 < nz ? a.alpha[c + nx * ny] : a.oobA;
            a_k = z > 0 ? a.alpha[c - nx * ny] : a.oobA;
        }
        load_p();
        old = ldv<CG>(a.r + c);
        if (a_c >= 1.f) return 0.f;
        f_top = 1.f - a_t;
        f_bottom = 1.f - a_b;
        f_right = 1.f - a_r;
        f_left = 1.f - a_l;
        if constexpr (DIM == 3) {
            f_front = 1.f - a_f;
            f_back = 1.f - a_k;
        }
    }
    float p_sum = p_top * f_top + p_bottom * f_bottom;
    p_sum = p_sum + p_right * f_right;
    p_sum = p_sum + p_left * f_left;
    float f_sum = f_top + f_bottom + f_right + f_left;
    if constexpr (DIM == 3) {
        p_sum = p_sum + p_front * f_front;
        p_sum = p_sum + p_back * f_back;
        f_sum = f_sum + f_front + f_back;
    }
    return old - (p_sum - f_sum * p_c) / a.hh;
}

// One thread per coarse cell: residual of its 2^DIM children (written in place
// when WRITE_FINE, the reference's in-place residual), then restrict_residual
// (restrict_residual.comp:40-64, 2D :40-59) into the next level when
// WRITE_COARSE.  The grid also covers the fine cells left over by odd sizes.
template <int DIM, bool L0, bool WRITE_FINE, bool WRITE_COARSE, typename T = float, bool CG = false>
SS_D void residual_restrict_cell(const MGArgsT<T>& a, T* __restrict__ rc, int cx, int cy, int cz, int X, int Y, int Z,
                                 T* __restrict__ pz = nullptr) {
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int x0 = 2 * X, y0 = 2 * Y, z0 = DIM == 3 ? 2 * Z : 0;
    if (x0 >= nx || y0 >= ny || z0 >= nz) return;
    float v[2][2][2];  // [dz][dy][dx]
#pragma unroll
    for (int dz = 0; dz < (DIM == 3 ? 2 : 1); ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int x = x0 + dx, y = y0 + dy, z = z0 + dz;
                float res = 0.f;
                if (x < nx && y < ny && z < nz) {
                    res = residual_cell<DIM, L0, T, CG>(a, x, y, z);
                    if constexpr (WRITE_FINE) {
                        a.r[idx3(x, y, z, nx, ny)] = st<T>(res);
                        res = rnd<T>(res);
                    }
                }
                v[dz][dy][dx] = res;
            }
    if constexpr (WRITE_COARSE) {
        if (X < cx && Y < cy && Z < cz) {
            float out;
            if constexpr (DIM == 3) {
                const float bottom = v[0][0][0] + v[1][0][0] + v[0][0][1] + v[1][0][1];
                const float top = v[0][1][0] + v[1][1][0] + v[0][1][1] + v[1][1][1];
                out = (bottom + top) / 8.f;
            } else {
                out = (v[0][0][0] + v[0][0][1] + v[0][1][0] + v[0][1][1]) / 4.f;
            }
            rc[idx3(X, Y, Z, cx, cy)] = st<T>(out);
            if (pz) pz[idx3(X, Y, Z, cx, cy)] = st<T>(0.f);   // the coarse initial guess
        }
    }
}

// pz: also set the next level's pressure (its initial guess) to +0
template <int DIM, bool L0, bool WRITE_FINE, bool WRITE_COARSE, typename T = float>
__global__ void __launch_bounds__(256) k_residual_restrict(MGArgsT<T> a, T* __restrict__ rc, int cx, int cy, int cz,
                                                           T* __restrict__ pz) {
    pdl_entry();
    residual_restrict_cell<DIM, L0, WRITE_FINE, WRITE_COARSE, T>(a, rc, cx, cy, cz, blockIdx.x * blockDim.x + threadIdx.x,
                                                                 blockIdx.y * blockDim.y + threadIdx.y,
                                                                 blockIdx.z * blockDim.z + threadIdx.z, pz);
}

template <int DIM, bool L0>
static void launch_rr(bool pdl, const MGArgs& a, float* rc, int cx, int cy, int cz, bool wf, bool wc, dim3 g, dim3 b,
                      cudaStream_t st) {
    if (wf && wc) launch_k(pdl, g, b, 0, st, k_residual_restrict<DIM, L0, true, true>, a, rc, cx, cy, cz, nullptr);
    else if (wf) launch_k(pdl, g, b, 0, st, k_residual_restrict<DIM, L0, true, false>, a, rc, cx, cy, cz, nullptr);
    else launch_k(pdl, g, b, 0, st, k_residual_restrict<DIM, L0, false, true>, a, rc, cx, cy, cz, nullptr);
}

int launch_residual(ss_sim* s, const StepConsts& c, int L, bool write_fine, bool write_coarse, int quirks,
                    cudaStream_t st) {
    if (!write_fine && !write_coarse) return SS_OK;
    if (write_coarse && L + 1 >= s->levels) return set_error(SS_E_INVALID, "residual restriction below the coarsest level");
    MGArgs a = mg_args(s, c, L, resid_oob(s, quirks));
    const int cx = write_coarse ? s->lv[L + 1].n[0] : 0;
    const int cy = write_coarse ? s->lv[L + 1].n[1] : 0;
    const int cz = write_coarse ? s->lv[L + 1].n[2] : 0;
    float* rc = write_coarse ? s->r[L + 1] : nullptr;
    dim3 b(32, 8, 1);
    dim3 g = grid_for((a.nx + 1) / 2, (a.ny + 1) / 2, s->dim == 3 ? (a.nz + 1) / 2 : 1, b);
    if (s->dim == 3) {
        if (L == 0) launch_rr<3, true>(s->pdl != 0, a, rc, cx, cy, cz, write_fine, write_coarse, g, b, st);
        else launch_rr<3, false>(s->pdl != 0, a, rc, cx, cy, cz, write_fine, write_coarse, g, b, st);
    } else {
        if (L == 0) launch_rr<2, true>(s->pdl != 0, a, rc, cx, cy, cz, write_fine, write_coarse, g, b, st);
        else launch_rr<2, false>(s->pdl != 0, a, rc, cx, cy, cz, write_fine, write_coarse, g, b, st);
    }
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_residual_restrict");
}

// restrict_residual alone (reads the in-place residual of level L)
template <int DIM>
__global__ void k_restrict(const float* __restrict__ rf, int fx, int fy, float* __restrict__ rc, int cx, int cy, int cz) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y * blockDim.y + threadIdx.y;
    const int Z = blockIdx.z * blockDim.z + threadIdx.z;
    if (X >= cx || Y >= cy || Z >= cz) return;
    const int x = 2 * X, y = 2 * Y, z = 2 * Z;
    float out;
    if constexpr (DIM == 3) {
        const float bottom = rf[idx3(x, y, z, fx, fy)] + rf[idx3(x, y, z + 1, fx, fy)] + rf[idx3(x + 1, y, z, fx, fy)] +
                             rf[idx3(x + 1, y, z + 1, fx, fy)];
        const float top = rf[idx3(x, y + 1, z, fx, fy)] + rf[idx3(x, y + 1, z + 1, fx, fy)] +
                          rf[idx3(x + 1, y + 1, z, fx, fy)] + rf[idx3(x + 1, y + 1, z + 1, fx, fy)];
        out = (bottom + top) / 8.f;
    } else {
        out = (rf[idx3(x, y, 0, fx, fy)] + rf[idx3(x + 1, y, 0, fx, fy)] + rf[idx3(x, y + 1, 0, fx, fy)] +
               rf[idx3(x + 1, y + 1, 0, fx, fy)]) / 4.f;
    }
    rc[idx3(X, Y, Z, cx, cy)] = out;
}

int launch_restrict(ss_sim* s, int L, cudaStream_t st) {
    if (L + 1 >= s->levels) return set_error(SS_E_INVALID, "restriction below the coarsest level");
    const int* f = s->lv[L].n;
    const int* cc = s->lv[L + 1].n;
    dim3 b(32, 8, 1);
    dim3 g = grid_for(cc[0], cc[1], cc[2], b);
    if (s->dim == 3) k_restrict<3><<<g, b, 0, st>>>(s->r[L], f[0], f[1], s->r[L + 1], cc[0], cc[1], cc[2]);
    else k_restrict<2><<<g, b, 0, st>>>(s->r[L], f[0], f[1], s->r[L + 1], cc[0], cc[1], cc[2]);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_restrict");
}

// --------------------------------------------------------------- prolongation
// prolong_pressure.comp:39-51: p_L += GL_LINEAR, CLAMP_TO_EDGE sample of
// p_{L+1} at the fine cell centre, on every cell.
template <int DIM, typename T = float, bool CG = false>
SS_D void prolong_cell(T* __restrict__ p, int ax, int ay, int az, const T* __restrict__ pc, int cx, int cy, int cz,
                       int x, int y, int z) {
    if (x >= ax || y >= ay || z >= az) return;
    const float tx = (((float)x + 0.5f) / (float)ax) * (float)cx - 0.5f;
    const float ty = (((float)y + 0.5f) / (float)ay) * (float)cy - 0.5f;
    const float fx = floorf(tx), fy = floorf(ty);
    const int x0 = (int)fx, y0 = (int)fy;
    const float wx = tx - fx, wy = ty - fy;
    const int xa = min(max(x0, 0), cx - 1), xb = min(max(x0 + 1, 0), cx - 1);
    const int ya = min(max(y0, 0), cy - 1), yb = min(max(y0 + 1, 0), cy - 1);
    float s;
    if constexpr (DIM == 2) {
        s = lerp_(lerp_(ldv<CG>(&pc[idx3(xa, ya, 0, cx, cy)]), ldv<CG>(&pc[idx3(xb, ya, 0, cx, cy)]), wx),
                  lerp_(ldv<CG>(&pc[idx3(xa, yb, 0, cx, cy)]), ldv<CG>(&pc[idx3(xb, yb, 0, cx, cy)]), wx), wy);
    } else {
        const float tz = (((float)z + 0.5f) / (float)az) * (float)cz - 0.5f;
        const float fz = floorf(tz);
        const int z0 = (int)fz;
        const float wz = tz - fz;
        const int za = min(max(z0, 0), cz - 1), zb = min(max(z0 + 1, 0), cz - 1);
        const float c0 = lerp_(lerp_(ldv<CG>(&pc[idx3(xa, ya, za, cx, cy)]), ldv<CG>(&pc[idx3(xb, ya, za, cx, cy)]), wx),
                               lerp_(ldv<CG>(&pc[idx3(xa, yb, za, cx, cy)]), ldv<CG>(&pc[idx3(xb, yb, za, cx, cy)]), wx), wy);
        const float c1 = lerp_(lerp_(ldv<CG>(&pc[idx3(xa, ya, zb, cx, cy)]), ldv<CG>(&pc[idx3(xb, ya, zb, cx, cy)]), wx),
                               lerp_(ldv<CG>(&pc[idx3(xa, yb, zb, cx, cy)]), ldv<CG>(&pc[idx3(xb, yb, zb, cx, cy)]), wx), wy);
        s = lerp_(c0, c1, wz);
    }
    const int i = idx3(x, y, z, ax, ay);
    p[i] = st<T>(ldv<CG>(p + i) + s);
}

template <int DIM, typename T = float>
__global__ void __launch_bounds__(256) k_prolong(T* __restrict__ p, int ax, int ay, int az,
                                                 const T* __restrict__ pc, int cx, int cy, int cz) {
    pdl_entry();
    prolong_cell<DIM, T>(p, ax, ay, az, pc, cx, cy, cz, blockIdx.x * blockDim.x + threadIdx.x,
                         blockIdx.y * blockDim.y + threadIdx.y, blockIdx.z * blockDim.z + threadIdx.z);
}

int launch_prolong(ss_sim* s, int L, cudaStream_t st) {
    const int next = L + 1 < s->levels ? L + 1 : s->levels - 1;
    const int* f = s->lv[L].n;
    const int* cc = s->lv[next].n;
    dim3 b(32, 8, 1);
    dim3 g = grid_for(f[0], f[1], f[2], b);
    if (s->dim == 3) launch_k(s->pdl, g, b, 0, st, k_prolong<3>, s->p[L], f[0], f[1], f[2], s->p[next], cc[0], cc[1], cc[2]);
    else launch_k(s->pdl, g, b, 0, st, k_prolong<2>, s->p[L], f[0], f[1], f[2], s->p[next], cc[0], cc[1], cc[2]);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_prolong");
}

// -------------------------------------------------------------- solid pyramid
// restrict_solid.comp:53-78 (2D :53-73): mean of the children, zeroed below
// 0.5, stored as FP16.  Only the alpha channel feeds the coarse operators.
template <int DIM, bool FROM_FLAGS>
__global__ void k_restrict_alpha(const uint8_t* __restrict__ flags, const float* __restrict__ af, int fx, int fy,
                                 float* __restrict__ ac, int cx, int cy, int cz) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y * blockDim.y + threadIdx.y;
    const int Z = blockIdx.z * blockDim.z + threadIdx.z;
    if (X >= cx || Y >= cy || Z >= cz) return;
    const int x = 2 * X, y = 2 * Y, z = 2 * Z;
    auto A = [&](int i, int j, int k) -> float {
        const int q = idx3(i, j, k, fx, fy);
        if constexpr (FROM_FLAGS) return (flags[q] & F_SOLID) ? 1.f : 0.f;
        else return af[q];
    };
    float m;
    if constexpr (DIM == 3) {
        const float b = A(x, y, z) + A(x, y, z + 1) + A(x + 1, y, z) + A(x + 1, y, z + 1);
        const float t = A(x, y + 1, z) + A(x, y + 1, z + 1) + A(x + 1, y + 1, z) + A(x + 1, y + 1, z + 1);
        m = (b + t) / 8.f;
    } else {
        m = (A(x, y, 0) + A(x + 1, y, 0) + A(x, y + 1, 0) + A(x + 1, y + 1, 0)) / 4.f;
    }
    const float keep = m >= 0.5f ? 1.f : 0.f;
    ac[idx3(X, Y, Z, cx, cy)] = round_half(m * keep);
}

int launch_solid_pyramid(ss_sim* s, cudaStream_t st) {
    dim3 b(32, 8, 1);
    for (int L = 0; L + 1 < s->levels; ++L) {
        const int* f = s->lv[L].n;
        const int* cc = s->lv[L + 1].n;
        dim3 g = grid_for(cc[0], cc[1], cc[2], b);
        if (s->dim == 3) {
            if (L == 0) k_restrict_alpha<3, true><<<g, b, 0, st>>>(s->flags, nullptr, f[0], f[1], s->alpha[1], cc[0], cc[1], cc[2]);
            else k_restrict_alpha<3, false><<<g, b, 0, st>>>(nullptr, s->alpha[L], f[0], f[1], s->alpha[L + 1], cc[0], cc[1], cc[2]);
        } else {
            if (L == 0) k_restrict_alpha<2, true><<<g, b, 0, st>>>(s->flags, nullptr, f[0], f[1], s->alpha[1], cc[0], cc[1], cc[2]);
            else k_restrict_alpha<2, false><<<g, b, 0, st>>>(nullptr, s->alpha[L], f[0], f[1], s->alpha[L + 1], cc[0], cc[1], cc[2]);
        }
    }
    s->pyramid_dirty = 0;
    s->cmat_dirty = 1;
    s->nlaunch += s->levels - 1;
    return check_cuda(cudaGetLastError(), "k_restrict_alpha");
}

// ------------------------------------------------- projected residual (FP64)
// R = div - (dt/(rho h)) (sum_f p_nb - f_sum p) over fluid cells, evaluated in
// FP64 from the FP32 state: the divergence the projection would leave.
SS_D double block_sum_d(double v) {
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

template <int DIM>
__global__ void __launch_bounds__(256) k_projected_residual(const float* __restrict__ p, const float* __restrict__ div0,
                                                            const uint8_t* __restrict__ flags, int nx, int ny, int nz,
                                                            double k, double* __restrict__ partial) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    double acc = 0.0;
    if (x < nx && y < ny && z < nz) {
        const int c = idx3(x, y, z, nx, ny);
        const uint8_t fl = flags[c];
        if (!(fl & F_SOLID)) {
            double psum = 0.0, fsum = 0.0;
            auto nb = [&](bool in, uint8_t bit, int off) {
                const double f = in ? ((fl & bit) ? 0.0 : 1.0) : 1.0;
                const double pn = in ? (double)p[c + off] : 0.0;
                psum += f * pn;
                fsum += f;
            };
            nb(y + 1 < ny, F_TOP, nx);
            nb(y > 0, F_BOTTOM, -nx);
            nb(x + 1 < nx, F_RIGHT, 1);
            nb(x > 0, F_LEFT, -1);
            if constexpr (DIM == 3) {
                nb(z + 1 < nz, F_FRONT, nx * ny);
                nb(z > 0, F_BACK, -nx * ny);
            }
            const double rr = (double)div0[c] - k * (psum - fsum * (double)p[c]);
            acc = rr * rr;
        }
    }
    const double bs = block_sum_d(acc);
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0)
        partial[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = bs;
}

int launch_projected_residual_norm(ss_sim* s, const StepConsts& c, int slot, cudaStream_t st) {
    dim3 b(32, 8, 1);
    dim3 g = grid_for(s->nx, s->ny, s->nz, b);
    const double k = (double)c.dt / ((double)c.rho * (double)s->h);
    if (s->dim == 3) k_projected_residual<3><<<g, b, 0, st>>>(s->p[0], s->div0, s->flags, s->nx, s->ny, s->nz, k, s->red.partial);
    else k_projected_residual<2><<<g, b, 0, st>>>(s->p[0], s->div0, s->flags, s->nx, s->ny, s->nz, k, s->red.partial);
    s->nlaunch += 1;
    int rc = check_cuda(cudaGetLastError(), "k_projected_residual");
    if (rc) return rc;
    return launch_reduce_final(s, (int)(g.x * g.y * g.z), slot, st);
}


// ------------------------------------------------------------- bottom solver
// The lower part of the V-cycle (levels Lb..coarsest) in ONE thread block with
// every array resident in shared memory.  It runs the same per-cell
// operations as the per-level kernels above (smooth_cell, residual_cell, the
// restriction sum order, the prolongation formula), so the result is
// bit-identical to launching them level by level - without the
// 2*(n_pre+n_post)+2 launches per level and 2*n_coarse launches on the
// coarsest level, which are pure launch latency at these sizes.
struct BottomLevel {
    int n[3];
    int off;        // offset of the level in the shared arrays
    float hh;
};
template <typename T>
struct BottomArgsT {
    int nlev;
    BottomLevel lv[SS_MAX_LEVELS];
    T* p[SS_MAX_LEVELS];
    T* r[SS_MAX_LEVELS];
    const float* alpha[SS_MAX_LEVELS];
    int total;
    int n_pre, n_post, n_coarse, quirks;
    float oob_smooth, oob_resid;
    const float* cmat;   // coarsest level by its response matrix (mixed solve), or null: sweeps
    float* cpart;        // the product's slice sums (kProductLanes floats)
};

template <typename T>
SS_D MGArgs bottom_level(const BottomArgsT<T>& b, float* sp, float* sr, float* sa, int l, float oobA) {
    MGArgs a;
    a.p = sp + b.lv[l].off;
    a.r = sr + b.lv[l].off;
    a.alpha = sa + b.lv[l].off;
    a.flags = nullptr;
    a.div0 = nullptr;
    a.div0r = nullptr;
    a.nx = b.lv[l].n[0];
    a.ny = b.lv[l].n[1];
    a.nz = b.lv[l].n[2];
    a.oobA = oobA;
    a.hh = b.lv[l].hh;
    a.rho_h = 0.f;
    a.dt = 1.f;
    a.rho = 1.f;
    a.dt_h = 1.f;
    return a;
}

// Red-black sweeps of one small level.  Each thread's cells (at most
// kBottomCells) and their colours are decoded once, outside the sweep loop;
// a level small enough for two cells per thread of fewer warps runs on those
// warps only, synchronised by a named barrier.
constexpr int kBottomCells = 4;

// A level of at most two cells per active thread (the coarsest level, which
// takes n_coarse sweeps): each thread keeps its cells' neighbour weights,
// diagonal and r*h^2 term in registers for all the sweeps - the arithmetic
// of smooth_cell, minus its per-sweep solid-fraction loads.
template <int DIM, typename R>
SS_D void bottom_smooth_cached(const MGArgs& a, int iterations, int nt) {
    const int n = a.nx * a.ny * a.nz;
    const int nx = a.nx, ny = a.ny, nz = a.nz, pl = nx * ny;
    int ci[2], col[2], inr[2];
    bool act[2];
    float f[2][6], rhh[2], fs[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int c = threadIdx.x + k * nt;
        act[k] = c < n;
        ci[k] = c;
        col[k] = 0;
        inr[k] = 0;
        rhh[k] = 0.f;
        fs[k] = 1.f;
#pragma unroll
        for (int d = 0; d < 6; ++d) f[k][d] = 0.f;
        if (!act[k]) continue;
        const int x = c % nx, t = c / nx, y = t % ny, z = t / ny;
        col[k] = (x + y + z) & 1;
        if (a.alpha[c] >= 1.f) { act[k] = false; continue; }
        inr[k] = (y + 1 < ny ? 1 : 0) | (y > 0 ? 2 : 0) | (x + 1 < nx ? 4 : 0) | (x > 0 ? 8 : 0) |
                 (z + 1 < nz ? 16 : 0) | (z > 0 ? 32 : 0);
        f[k][0] = 1.f - (y + 1 < ny ? a.alpha[c + nx] : a.oobA);
        f[k][1] = 1.f - (y > 0 ? a.alpha[c - nx] : a.oobA);
        f[k][2] = 1.f - (x + 1 < nx ? a.alpha[c + 1] : a.oobA);
        f[k][3] = 1.f - (x > 0 ? a.alpha[c - 1] : a.oobA);
        if constexpr (DIM == 3) {
            f[k][4] = 1.f - (z + 1 < nz ? a.alpha[c + pl] : a.oobA);
            f[k][5] = 1.f - (z > 0 ? a.alpha[c - pl] : a.oobA);
        }
        float f_sum = f[k][0] + f[k][1] + f[k][2] + f[k][3];
        if constexpr (DIM == 3) f_sum = f_sum + f[k][4] + f[k][5];
        if (f_sum == 0.f) { act[k] = false; continue; }
        fs[k] = f_sum;
        rhh[k] = ld(a.r[c]) * a.hh;
    }
    const float* P = a.p;
    for (int it = 0; it < 2 * iterations; ++it) {
        const int parity = it & 1;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (!act[k] || col[k] != parity) continue;
            const int c = ci[k], m = inr[k];
            const float p_top = (m & 1) ? P[c + nx] : 0.f;
            const float p_bottom = (m & 2) ? P[c - nx] : 0.f;
            const float p_right = (m & 4) ? P[c + 1] : 0.f;
            const float p_left = (m & 8) ? P[c - 1] : 0.f;
            float p_sum = p_top * f[k][0] + p_bottom * f[k][1];
            p_sum = p_sum + p_right * f[k][2];
            p_sum = p_sum + p_left * f[k][3];
            if constexpr (DIM == 3) {
                const float p_front = (m & 16) ? P[c + pl] : 0.f;
                const float p_back = (m & 32) ? P[c - pl] : 0.f;
                p_sum = p_sum + p_front * f[k][4];
                p_sum = p_sum + p_back * f[k][5];
            }
            a.p[c] = rnd<R>((p_sum - rhh[k]) / fs[k]);
        }
        if (nt == (int)blockDim.x) __syncthreads();
        else asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
    }
}

template <int DIM, typename R>
SS_D void bottom_smooth(const MGArgs& a, int iterations) {
    const int n = a.nx * a.ny * a.nz;
    int nt = blockDim.x;
    // the fewest threads that still give every cell its own thread (the
    // coarsest 8^3 level: 512); measured faster than two cells a thread
    while (nt > 128 && (n + nt / 2 - 1) / (nt / 2) <= 1) nt /= 2;
    if ((n + nt - 1) / nt <= 2) {
        if ((int)threadIdx.x < nt) bottom_smooth_cached<DIM, R>(a, iterations, nt);
        __syncthreads();
        return;
    }
    if ((int)threadIdx.x < nt) {
        int cx[kBottomCells], cy[kBottomCells], cz[kBottomCells], col[kBottomCells];
        int k = 0;
        for (int c = threadIdx.x; c < n && k < kBottomCells; c += nt, ++k) {
            cx[k] = c % a.nx;
            const int t = c / a.nx;
            cy[k] = t % a.ny;
            cz[k] = t / a.ny;
            col[k] = (cx[k] + cy[k] + cz[k]) & 1;
        }
        const bool fits = (n + nt - 1) / nt <= kBottomCells;
        for (int it = 0; it < 2 * iterations; ++it) {
            const int parity = it & 1;
            if (fits) {
                for (int q = 0; q < k; ++q)
                    if (col[q] == parity) smooth_cell<DIM, false, float, R>(a, cx[q], cy[q], cz[q]);
            } else {
                for (int c = threadIdx.x; c < n; c += nt) {
                    const int x = c % a.nx, t = c / a.nx, y = t % a.ny, z = t / a.ny;
                    if (((x + y + z) & 1) != parity) continue;
                    smooth_cell<DIM, false, float, R>(a, x, y, z);
                }
            }
            if (nt == (int)blockDim.x) __syncthreads();
            else asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
        }
    }
    __syncthreads();
}

// T: storage type of the global level arrays; R: rounding of every value the
// solve stores (T, or float for the FP32 solve).
// Part of p_j = sum_i E[i n + j] r_i over i in [i0, i1), where E[i n + j] =
// dp_j / dr_i of the coarsest level's n_coarse sweeps from p = 0
// (k_coarse_response, layout 1): eight partial sums taken round-robin
// ((i - i0) mod 8), added pairwise, so the oracle can repeat the order.  Two
// rounds of eight independent loads are in flight per step (the matrix
// streams from L2).
// r: the level's right-hand side (shared-memory floats in the one-block
// bottom solve, the level's global array with CG in the cluster form).
template <bool CG = false, typename RT>
SS_D float coarse_product(const float* __restrict__ E, const RT* r, int n, int j, int i0, int i1) {
    float a[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float* e = E + j;
    int i = i0;
    for (; i + 16 <= i1; i += 16) {
        float v[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = __ldg(e + (size_t)(i + k) * n);
#pragma unroll
        for (int k = 0; k < 16; ++k) a[k & 7] += v[k] * ldv<CG>(r + i + k);
    }
#pragma unroll
    for (int k = 0; k < 16; ++k)
        if (i + k < i1) a[k & 7] += __ldg(e + (size_t)(i + k) * n) * ldv<CG>(r + i + k);
    return ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
}

// Slices of i per coarse value in the matrix product: the largest power of
// two (at most 32) with parts * n <= kProductLanes, a cluster's threads - so
// the cluster form takes one slice (at most 16 terms at 8^3) per thread.  The
// one-block bottom solve walks the same (slice, value) items in turns of its
// 1024 threads, so both give the same sums in the same order.
SS_D int coarse_parts(int n) {
    int parts = 1;
    while (parts < 32 && parts * 2 * n <= kProductLanes) parts *= 2;
    return parts;
}

// p_j = sum_i E[i n + j] r_i for every j of the coarsest level, in two phases
// separated by a barrier of the caller's.  Phase 1: item t is slice
// q = t / n of value j = t % n (adjacent lanes read adjacent j of a row of E,
// coalesced); its sum goes to part[q n + j].  Phase 2: value j folds its
// slices as a tree, v[q] += v[q + o] for o = parts/2 .. 1, rounds the result
// as R and stores it as PT.  `part` holds parts * n <= kProductLanes floats.
template <bool CG, typename RT>
SS_D void coarse_matrix_partials(const float* __restrict__ E, const RT* r, float* part, int n, int tid,
                                 int nthreads) {
    const int parts = coarse_parts(n), chunk = (n + parts - 1) / parts;
    for (int t = tid; t < parts * n; t += nthreads) {
        const int q = t / n, j = t % n;
        part[t] = coarse_product<CG>(E, r, n, j, q * chunk, min(n, (q + 1) * chunk));
    }
}

template <bool CG, typename R, typename PT>
SS_D void coarse_matrix_fold(const float* part, PT* p, int n, int tid, int nthreads) {
    const int parts = coarse_parts(n);
    for (int j = tid; j < n; j += nthreads) {
        float v[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) v[q] = q < parts ? ldv<CG>(part + q * n + j) : 0.f;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1)
            if (o < parts) {
#pragma unroll
                for (int q = 0; q < o; ++q) v[q] = v[q] + v[q + o];
            }
        p[j] = st<PT>(rnd<R>(v[0]));
    }
}

template <int DIM, typename T, typename R>
__global__ void __launch_bounds__(1024) k_bottom(BottomArgsT<T> b) {
    pdl_entry();
    extern __shared__ float sm[];
    float* sp = sm;
    float* sr = sm + b.total;
    float* sa = sm + 2 * b.total;
    for (int l = 0; l < b.nlev; ++l) {
        const int n = b.lv[l].n[0] * b.lv[l].n[1] * b.lv[l].n[2];
        const int o = b.lv[l].off;
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            sp[o + c] = ld(b.p[l][c]);
            sr[o + c] = ld(b.r[l][c]);
            sa[o + c] = b.alpha[l][c];
        }
    }
    __syncthreads();
    // down: pre-smoothing, residual (in place only with the reference's rule) + restriction, clear next p
    for (int l = 0; l + 1 < b.nlev; ++l) {
        const MGArgs a = bottom_level(b, sp, sr, sa, l, b.oob_smooth);
        bottom_smooth<DIM, R>(a, b.n_pre);
        const MGArgs ar = bottom_level(b, sp, sr, sa, l, b.oob_resid);
        const int cx = b.lv[l + 1].n[0], cy = b.lv[l + 1].n[1], cz = b.lv[l + 1].n[2];
        const int hx = (a.nx + 1) / 2, hy = (a.ny + 1) / 2, hz = DIM == 3 ? (a.nz + 1) / 2 : 1;
        float* rc = sr + b.lv[l + 1].off;
        for (int q = threadIdx.x; q < hx * hy * hz; q += blockDim.x) {
            const int X = q % hx, t = q / hx, Y = t % hy, Z = t / hy;
            const int x0 = 2 * X, y0 = 2 * Y, z0 = DIM == 3 ? 2 * Z : 0;
            float v[2][2][2];
            for (int dz = 0; dz < (DIM == 3 ? 2 : 1); ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx) {
                        const int x = x0 + dx, y = y0 + dy, z = z0 + dz;
                        float res = 0.f;
                        if (x < a.nx && y < a.ny && z < a.nz) {
                            res = residual_cell<DIM, false>(ar, x, y, z);
                            if (b.quirks) {
                                res = rnd<R>(res);
                                ar.r[idx3(x, y, z, a.nx, a.ny)] = res;
                            }
                        }
                        v[dz][dy][dx] = res;
                    }
            if (X < cx && Y < cy && Z < cz) {
                float out;
                if constexpr (DIM == 3) {
                    const float bottom = v[0][0][0] + v[1][0][0] + v[0][0][1] + v[1][0][1];
                    const float top = v[0][1][0] + v[1][1][0] + v[0][1][1] + v[1][1][1];
                    out = (bottom + top) / 8.f;
                } else {
                    out = (v[0][0][0] + v[0][0][1] + v[0][1][0] + v[0][1][1]) / 4.f;
                }
                rc[idx3(X, Y, Z, cx, cy)] = rnd<R>(out);
            }
        }
        float* pc = sp + b.lv[l + 1].off;
        for (int c = threadIdx.x; c < cx * cy * cz; c += blockDim.x) pc[c] = 0.f;
        __syncthreads();
    }
    // coarsest level
    if (b.cmat) {
        // p = E r (coarse_matrix_apply), the stores rounded as R
        const MGArgs ac = bottom_level(b, sp, sr, sa, b.nlev - 1, b.oob_smooth);
        const int n = ac.nx * ac.ny * ac.nz;
        coarse_matrix_partials<false>(b.cmat, ac.r, b.cpart, n, (int)threadIdx.x, (int)blockDim.x);
        __syncthreads();
        coarse_matrix_fold<false, R>(b.cpart, ac.p, n, (int)threadIdx.x, (int)blockDim.x);
        __syncthreads();
    } else {
        bottom_smooth<DIM, R>(bottom_level(b, sp, sr, sa, b.nlev - 1, b.oob_smooth), b.n_coarse);
    }
    // up: prolongation + post-smoothing
    for (int l = b.nlev - 2; l >= 0; --l) {
        const MGArgs a = bottom_level(b, sp, sr, sa, l, b.oob_smooth);
        const int cx = b.lv[l + 1].n[0], cy = b.lv[l + 1].n[1], cz = b.lv[l + 1].n[2];
        const float* pc = sp + b.lv[l + 1].off;
        const int ax = a.nx, ay = a.ny, az = a.nz;
        for (int c = threadIdx.x; c < ax * ay * az; c += blockDim.x) {
            const int x = c % ax, t = c / ax, y = t % ay, z = t / ay;
            const float tx = (((float)x + 0.5f) / (float)ax) * (float)cx - 0.5f;
            const float ty = (((float)y + 0.5f) / (float)ay) * (float)cy - 0.5f;
            const float fx = floorf(tx), fy = floorf(ty);
            const int x0 = (int)fx, y0 = (int)fy;
            const float wx = tx - fx, wy = ty - fy;
            const int xa = min(max(x0, 0), cx - 1), xb = min(max(x0 + 1, 0), cx - 1);
            const int ya = min(max(y0, 0), cy - 1), yb = min(max(y0 + 1, 0), cy - 1);
            float sv;
            if constexpr (DIM == 2) {
                sv = lerp_(lerp_(pc[idx3(xa, ya, 0, cx, cy)], pc[idx3(xb, ya, 0, cx, cy)], wx),
                           lerp_(pc[idx3(xa, yb, 0, cx, cy)], pc[idx3(xb, yb, 0, cx, cy)], wx), wy);
            } else {
                const float tz = (((float)z + 0.5f) / (float)az) * (float)cz - 0.5f;
                const float fz = floorf(tz);
                const int z0 = (int)fz;
                const float wz = tz - fz;
                const int za = min(max(z0, 0), cz - 1), zb = min(max(z0 + 1, 0), cz - 1);
                const float c0 = lerp_(lerp_(pc[idx3(xa, ya, za, cx, cy)], pc[idx3(xb, ya, za, cx, cy)], wx),
                                       lerp_(pc[idx3(xa, yb, za, cx, cy)], pc[idx3(xb, yb, za, cx, cy)], wx), wy);
                const float c1 = lerp_(lerp_(pc[idx3(xa, ya, zb, cx, cy)], pc[idx3(xb, ya, zb, cx, cy)], wx),
                                       lerp_(pc[idx3(xa, yb, zb, cx, cy)], pc[idx3(xb, yb, zb, cx, cy)], wx), wy);
                sv = lerp_(c0, c1, wz);
            }
            a.p[c] = rnd<R>(a.p[c] + sv);
        }
        __syncthreads();
        bottom_smooth<DIM, R>(a, b.n_post);
    }
    // write back every level (pressure and, with the in-place rule, residual)
    for (int l = 0; l < b.nlev; ++l) {
        const int n = b.lv[l].n[0] * b.lv[l].n[1] * b.lv[l].n[2];
        const int o = b.lv[l].off;
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            b.p[l][c] = st<T>(sp[o + c]);
            b.r[l][c] = st<T>(sr[o + c]);
        }
    }
}

// ------------------------------------------------ coarse levels in one cluster
// The mixed solve's levels from cluster_from (the first of at most
// kClusterCells cells) down to the coarsest and back up, in ONE launch of one
// thread-block cluster of up to 16 CTAs x 1024 threads.  Every phase - a red
// or black half-sweep of a level, a residual + restriction (which also sets
// the next level's pressure to +0), a prolongation, the coarsest level's
// matrix product - is spread over all the cluster's threads, and a cluster
// barrier (barrier.cluster, release / acquire; about 0.3 us on B200) separates
// it from the next, in place of a launch per phase.  The arrays stay in global
// memory (L2-resident at these sizes): every value another CTA of the launch
// may have written is read with ld.global.cg (L1 is not coherent across SMs),
// the fixed solid fractions through L1.  The per-cell operations are those of
// the per-level kernels, so the result is the same, bit for bit, as launching
// them level by level.
constexpr int kClusterCells = 32768;
constexpr int kClusterThreads = 1024;

template <typename T>
struct ClusterArgsT {
    int nlev;
    int n[SS_MAX_LEVELS][3];
    float hh[SS_MAX_LEVELS];
    T* p[SS_MAX_LEVELS];
    T* r[SS_MAX_LEVELS];
    const float* alpha[SS_MAX_LEVELS];
    int n_pre, n_post, n_coarse;
    float oob_smooth, oob_resid;
    const float* cmat;   // coarsest level by its response matrix, or null: sweeps
    float* cpart;        // the product's slice sums (kProductLanes floats)
    float* fine;         // a level's residuals (kClusterCells floats)
};

// restrict_residual of coarse cell (X, Y, Z) from the fine residuals of the
// previous phase, in residual_restrict_cell's sum order (fine cells outside
// the grid count 0)
template <int DIM>
SS_D float cluster_restrict(const float* fine, int nx, int ny, int nz, int X, int Y, int Z) {
    float v[2][2][2];   // [dz][dy][dx]
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int x = 2 * X + dx, y = 2 * Y + dy, z = DIM == 3 ? 2 * Z + dz : 0;
                v[dz][dy][dx] = (x < nx && y < ny && z < nz && (DIM == 3 || dz == 0))
                                    ? __ldcg(fine + idx3(x, y, z, nx, ny)) : 0.f;
            }
    if constexpr (DIM == 3) {
        const float bottom = v[0][0][0] + v[1][0][0] + v[0][0][1] + v[1][0][1];
        const float top = v[0][1][0] + v[1][1][0] + v[0][1][1] + v[1][1][1];
        return (bottom + top) / 8.f;
    } else {
        return (v[0][0][0] + v[0][0][1] + v[0][1][0] + v[0][1][1]) / 4.f;
    }
}

template <typename T>
SS_D MGArgsT<T> cluster_level(const ClusterArgsT<T>& b, int l, float oobA) {
    MGArgsT<T> a;
    a.p = b.p[l];
    a.r = b.r[l];
    a.alpha = b.alpha[l];
    a.flags = nullptr;
    a.div0 = nullptr;
    a.div0r = nullptr;
    a.nx = b.n[l][0];
    a.ny = b.n[l][1];
    a.nz = b.n[l][2];
    a.oobA = oobA;
    a.hh = b.hh[l];
    a.rho_h = 0.f;
    a.dt = 1.f;
    a.rho = 1.f;
    a.dt_h = 1.f;
    return a;
}

// `iterations` red-black sweeps of one level, cell (x, y, z) of each colour
// as k_smooth numbers them, a cluster barrier after every half-sweep
template <int DIM, typename T>
SS_D void cluster_sweeps(const MGArgsT<T>& a, int iterations, int tid, int nthreads, cg::cluster_group& cl) {
    const int hx = (a.nx + 1) / 2, m = hx * a.ny * a.nz;
    for (int it = 0; it < 2 * iterations; ++it) {
        const int parity = it & 1;
        for (int i = tid; i < m; i += nthreads) {
            const int xi = i % hx, t = i / hx, y = t % a.ny, z = t / a.ny;
            const int x = 2 * xi + ((y + z + parity) & 1);
            if (x < a.nx) smooth_cell<DIM, false, T, T, true>(a, x, y, z);
        }
        cl.sync();
    }
}

template <int DIM, typename T>
__global__ void __launch_bounds__(kClusterThreads, 1) k_coarse_cluster(ClusterArgsT<T> b) {
    pdl_entry();
    cg::cluster_group cl = cg::this_cluster();
    const int nthreads = (int)(cl.num_blocks() * blockDim.x);
    const int tid = (int)(cl.block_rank() * blockDim.x + threadIdx.x);
    // down: pre-smoothing, residual + restriction (next level's p cleared)
    for (int l = 0; l + 1 < b.nlev; ++l) {
        cluster_sweeps<DIM, T>(cluster_level(b, l, b.oob_smooth), b.n_pre, tid, nthreads, cl);
        // residual of every fine cell (one a thread), then the restriction
        // from those values; the next level's p is cleared beside it
        const MGArgsT<T> ar = cluster_level(b, l, b.oob_resid);
        const int nf = ar.nx * ar.ny * ar.nz;
        for (int c = tid; c < nf; c += nthreads) {
            const int x = c % ar.nx, t = c / ar.nx, y = t % ar.ny, z = t / ar.ny;
            b.fine[c] = residual_cell<DIM, false, T, true>(ar, x, y, z);
        }
        cl.sync();
        const int cx = b.n[l + 1][0], cy = b.n[l + 1][1], cz = b.n[l + 1][2];
        for (int q = tid; q < cx * cy * cz; q += nthreads) {
            const int X = q % cx, t = q / cx, Y = t % cy, Z = t / cy;
            b.r[l + 1][q] = st<T>(cluster_restrict<DIM>(b.fine, ar.nx, ar.ny, ar.nz, X, Y, Z));
            b.p[l + 1][q] = st<T>(0.f);
        }
        cl.sync();
    }
    // coarsest level
    const int lc = b.nlev - 1;
    if (b.cmat) {
        const int n = b.n[lc][0] * b.n[lc][1] * b.n[lc][2];
        coarse_matrix_partials<true>(b.cmat, b.r[lc], b.cpart, n, tid, nthreads);
        cl.sync();
        coarse_matrix_fold<true, T>(b.cpart, b.p[lc], n, tid, nthreads);
        cl.sync();
    } else {
        cluster_sweeps<DIM, T>(cluster_level(b, lc, b.oob_smooth), b.n_coarse, tid, nthreads, cl);
    }
    // up: prolongation + post-smoothing
    for (int l = b.nlev - 2; l >= 0; --l) {
        const int ax = b.n[l][0], ay = b.n[l][1], az = b.n[l][2];
        for (int c = tid; c < ax * ay * az; c += nthreads) {
            const int x = c % ax, t = c / ax, y = t % ay, z = t / ay;
            prolong_cell<DIM, T, true>(b.p[l], ax, ay, az, b.p[l + 1], b.n[l + 1][0], b.n[l + 1][1], b.n[l + 1][2], x,
                                       y, z);
        }
        cl.sync();
        cluster_sweeps<DIM, T>(cluster_level(b, l, b.oob_smooth), b.n_post, tid, nthreads, cl);
    }
}

int bottom_start(const ss_sim* s) {
    // finest level >= 1 from which the rest of the pyramid fits the block's shared memory
    long long cum = 0;
    int start = s->levels;
    for (int l = s->levels - 1; l >= 1; --l) {
        const long long n = (long long)s->lv[l].n[0] * s->lv[l].n[1] * s->lv[l].n[2];
        if ((cum + n) * 12 > kBottomSmemBytes) break;
        cum += n;
        start = l;
    }
    return start;
}

template <typename T, typename R>
static int launch_bottom_t(ss_sim* s, const ss_mg_schedule& mg, int L, T* const* p, T* const* r, cudaStream_t st) {
    BottomArgsT<T> b{};
    b.nlev = s->levels - L;
    int off = 0;
    for (int l = 0; l < b.nlev; ++l) {
        const ss::Level& lv = s->lv[L + l];
        b.lv[l].n[0] = lv.n[0]; b.lv[l].n[1] = lv.n[1]; b.lv[l].n[2] = lv.n[2];
        b.lv[l].off = off;
        b.lv[l].hh = lv.hh;
        b.p[l] = p[L + l];
        b.r[l] = r[L + l];
        b.alpha[l] = s->alpha[L + l];
        off += lv.n[0] * lv.n[1] * lv.n[2];
    }
    b.total = off;
    b.n_pre = mg.n_pre; b.n_post = mg.n_post; b.n_coarse = mg.n_coarse;
    b.quirks = mg.ref_quirks ? 1 : 0;
    b.oob_smooth = smooth_oob(s, mg.ref_quirks);
    b.oob_resid = resid_oob(s, mg.ref_quirks);
    b.cmat = sizeof(T) == 2 ? s->cmat : nullptr;   // the mixed solve's coarse storage
    b.cpart = s->cmat_part;
    const size_t smem = (size_t)3 * off * sizeof(float);
    if (smem > (size_t)kBottomSmemBytes) return set_error(SS_E_INVALID, "bottom levels exceed shared memory");
    // the attribute is per function; setting it on every launch is cheap
    cudaError_t e = s->dim == 3
        ? cudaFuncSetAttribute(k_bottom<3, T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBottomSmemBytes)
        : cudaFuncSetAttribute(k_bottom<2, T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBottomSmemBytes);
    if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute(k_bottom)");
    if (s->dim == 3) launch_k(s->pdl, 1, 1024, smem, st, k_bottom<3, T, R>, b);
    else launch_k(s->pdl, 1, 1024, smem, st, k_bottom<2, T, R>, b);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_bottom");
}

int launch_bottom(ss_sim* s, const ss_mg_schedule& mg, int L, cudaStream_t st) {
    return launch_bottom_t<float, float>(s, mg, L, s->p, s->r, st);
}

// Response of the coarsest level's smoothing to unit right-hand sides: block
// i runs the bottom solve's `iters` red-black iterations from p = 0 with
// r = e_i (corrected out-of-grid rule, FP32 stores) and writes the result p
// as D[j * n + i] = dp_j / dr_i (layout 0: the adjoint applies D^T, reading
// consecutive i) or D[i * n + j] (layout 1: the mixed solve's bottom applies
// D, reading consecutive j).  With `state`, blocks do nothing unless
// state[1] (set by k_coarse_check) asks for a rebuild.
template <int DIM>
__global__ void __launch_bounds__(1024) k_coarse_response(BottomLevel lv, const float* __restrict__ alpha, float oobA,
                                                          int iters, float* __restrict__ D, int layout,
                                                          const int* __restrict__ state) {
    if (state && state[1] == 0) return;
    extern __shared__ float sm[];
    const int n = lv.n[0] * lv.n[1] * lv.n[2];
    float* sp = sm;
    float* sr = sm + n;
    float* sa = sm + 2 * n;
    const int i = blockIdx.x;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        sp[c] = 0.f;
        sr[c] = c == i ? 1.f : 0.f;
        sa[c] = alpha[c];
    }
    __syncthreads();
    MGArgs a;
    a.p = sp; a.r = sr; a.alpha = sa;
    a.flags = nullptr; a.div0 = nullptr; a.div0r = nullptr;
    a.nx = lv.n[0]; a.ny = lv.n[1]; a.nz = lv.n[2];
    a.oobA = oobA;
    a.hh = lv.hh;
    a.rho_h = 0.f; a.dt = 1.f; a.rho = 1.f; a.dt_h = 1.f;
    bottom_smooth<DIM, float>(a, iters);
    for (int c = threadIdx.x; c < n; c += blockDim.x) D[layout ? (size_t)i * n + c : (size_t)c * n + i] = sp[c];
}

// One block: state[1] = 1 when the coarsest level's solid fractions or the
// iteration count differ from the ones the matrix was built for (state[0];
// -1 before the first build), and the new ones are kept.
__global__ void __launch_bounds__(1024) k_coarse_check(const float* __restrict__ alpha, float* __restrict__ kept, int n,
                                                       int iters, int* __restrict__ state) {
    int diff = 0;
    for (int c = threadIdx.x; c < n; c += blockDim.x) diff |= alpha[c] != kept[c];
    diff = __syncthreads_or(diff) || state[0] != iters;
    for (int c = threadIdx.x; c < n; c += blockDim.x) kept[c] = alpha[c];
    if (threadIdx.x == 0) {
        state[0] = iters;
        state[1] = diff;
    }
}

static int launch_response(ss_sim* s, int iters, float* D, int layout, const int* state, cudaStream_t st) {
    const ss::Level& lv = s->lv[s->levels - 1];
    const int n = lv.n[0] * lv.n[1] * lv.n[2];
    if (n > kCoarseResponseMax) return set_error(SS_E_INVALID, "coarsest level too large for its response matrix");
    BottomLevel b{};
    b.n[0] = lv.n[0]; b.n[1] = lv.n[1]; b.n[2] = lv.n[2];
    b.off = 0;
    b.hh = lv.hh;
    const size_t smem = (size_t)3 * n * sizeof(float);
    const float* alpha = s->alpha[s->levels - 1];
    if (s->dim == 3) k_coarse_response<3><<<n, 1024, smem, st>>>(b, alpha, smooth_oob(s, 0), iters, D, layout, state);
    else k_coarse_response<2><<<n, 1024, smem, st>>>(b, alpha, smooth_oob(s, 0), iters, D, layout, state);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_coarse_response");
}

int launch_coarse_response(ss_sim* s, int iters, float* D, cudaStream_t st) {
    return launch_response(s, iters, D, 0, nullptr, st);
}

// The mixed solve's coarsest-level matrix, rebuilt where the solid pyramid
// or the coarse iteration count changed since it was built.
int update_coarse_matrix(ss_sim* s, const ss_mg_schedule& mg, cudaStream_t st) {
    if (!s->cmat) return SS_OK;
    if (!s->cmat_dirty && s->cmat_iters == mg.n_coarse) return SS_OK;
    const ss::Level& lv = s->lv[s->levels - 1];
    const int n = lv.n[0] * lv.n[1] * lv.n[2];
    k_coarse_check<<<1, 1024, 0, st>>>(s->alpha[s->levels - 1], s->cmat_alpha, n, mg.n_coarse, s->cmat_state);
    s->nlaunch += 1;
    int rc = check_cuda(cudaGetLastError(), "k_coarse_check");
    if (rc == SS_OK) rc = launch_response(s, mg.n_coarse, s->cmat, 1, s->cmat_state, st);
    if (rc != SS_OK) return rc;
    s->cmat_dirty = 0;
    s->cmat_iters = mg.n_coarse;
    return SS_OK;
}

// ---------------------------------------------------- coarse-storage variants
// The coarse levels of the mixed-precision correction solve: the same
// operators as above (out-of-grid rule of the corrected mode) on FP16 or BF16
// arrays; prec is SS_PREC_MIXED (FP16) or SS_PREC_MIXED_BF16.
template <typename T>
static MGArgsT<T> mg_args_t(ss_sim* s, const StepConsts& c, int L, float oobA, T* p, T* r) {
    const MGArgs f = mg_args(s, c, L, oobA);
    MGArgsT<T> a;
    a.p = p; a.r = r;
    a.alpha = f.alpha; a.flags = f.flags; a.div0 = f.div0; a.div0r = f.div0r;
    a.nx = f.nx; a.ny = f.ny; a.nz = f.nz;
    a.oobA = f.oobA; a.hh = f.hh; a.rho_h = f.rho_h; a.dt = f.dt; a.rho = f.rho; a.dt_h = f.dt_h;
    return a;
}

template <typename T>
static int coarse_smooth_t(ss_sim* s, const StepConsts& c, int L, int iterations, T* p, T* r, cudaStream_t st) {
    MGArgsT<T> a = mg_args_t<T>(s, c, L, smooth_oob(s, 0), p, r);
    dim3 b(32, 8, 1);
    dim3 g = grid_for((a.nx + 1) / 2, a.ny, a.nz, b);
    for (int it = 0; it < 2 * iterations; ++it) {
        if (s->dim == 3) launch_k(s->pdl, g, b, 0, st, k_smooth<3, false, T>, a, it & 1);
        else launch_k(s->pdl, g, b, 0, st, k_smooth<2, false, T>, a, it & 1);
    }
    s->nlaunch += 2 * iterations;
    return check_cuda(cudaGetLastError(), "k_smooth (coarse storage)");
}

template <typename T>
static int coarse_residual_restrict_t(ss_sim* s, const StepConsts& c, int L, T* p, T* r, T* rc, T* pz, cudaStream_t st) {
    MGArgsT<T> a = mg_args_t<T>(s, c, L, resid_oob(s, 0), p, r);
    const int cx = s->lv[L + 1].n[0], cy = s->lv[L + 1].n[1], cz = s->lv[L + 1].n[2];
    dim3 b(32, 8, 1);
    dim3 g = grid_for((a.nx + 1) / 2, (a.ny + 1) / 2, s->dim == 3 ? (a.nz + 1) / 2 : 1, b);
    if (s->dim == 3) launch_k(s->pdl, g, b, 0, st, k_residual_restrict<3, false, false, true, T>, a, rc, cx, cy, cz, pz);
    else launch_k(s->pdl, g, b, 0, st, k_residual_restrict<2, false, false, true, T>, a, rc, cx, cy, cz, pz);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_residual_restrict (coarse storage)");
}

template <typename T>
static int coarse_prolong_t(ss_sim* s, int L, T* p, const T* pc, cudaStream_t st) {
    const int* f = s->lv[L].n;
    const int* cc = s->lv[L + 1].n;
    dim3 b(32, 8, 1);
    dim3 g = grid_for(f[0], f[1], f[2], b);
    if (s->dim == 3) launch_k(s->pdl, g, b, 0, st, k_prolong<3, T>, p, f[0], f[1], f[2], pc, cc[0], cc[1], cc[2]);
    else launch_k(s->pdl, g, b, 0, st, k_prolong<2, T>, p, f[0], f[1], f[2], pc, cc[0], cc[1], cc[2]);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_prolong (coarse storage)");
}

int coarse_smooth(ss_sim* s, const StepConsts& c, int L, int iterations, int prec, cudaStream_t st) {
    if (prec == SS_PREC_MIXED) return coarse_smooth_t<__half>(s, c, L, iterations, (__half*)s->cp[L], (__half*)s->cr[L], st);
    return coarse_smooth_t<__nv_bfloat16>(s, c, L, iterations, (__nv_bfloat16*)s->cp[L], (__nv_bfloat16*)s->cr[L], st);
}

int coarse_residual_restrict(ss_sim* s, const StepConsts& c, int L, int prec, cudaStream_t st) {
    if (prec == SS_PREC_MIXED)
        return coarse_residual_restrict_t<__half>(s, c, L, (__half*)s->cp[L], (__half*)s->cr[L], (__half*)s->cr[L + 1],
                                                  (__half*)s->cp[L + 1], st);
    return coarse_residual_restrict_t<__nv_bfloat16>(s, c, L, (__nv_bfloat16*)s->cp[L], (__nv_bfloat16*)s->cr[L],
                                                      (__nv_bfloat16*)s->cr[L + 1], (__nv_bfloat16*)s->cp[L + 1], st);
}

int coarse_prolong(ss_sim* s, int L, int prec, cudaStream_t st) {
    if (prec == SS_PREC_MIXED) return coarse_prolong_t<__half>(s, L, (__half*)s->cp[L], (const __half*)s->cp[L + 1], st);
    return coarse_prolong_t<__nv_bfloat16>(s, L, (__nv_bfloat16*)s->cp[L], (const __nv_bfloat16*)s->cp[L + 1], st);
}

// ---------------------------------------------- coarse levels in one cluster
// The first level >= 1 of at most kClusterCells cells (0: none).
int coarse_cluster_from(const ss_sim* s) {
    for (int l = 1; l < s->levels; ++l)
        if ((long long)s->lv[l].n[0] * s->lv[l].n[1] * s->lv[l].n[2] <= kClusterCells) return l;
    return 0;
}

template <int DIM, typename T>
static cudaError_t cluster_config(int ctas, cudaLaunchConfig_t* cfg, cudaLaunchAttribute* at, int* active) {
    cudaError_t e = cudaFuncSetAttribute(k_coarse_cluster<DIM, T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    *cfg = cudaLaunchConfig_t{};
    cfg->gridDim = dim3(ctas);
    cfg->blockDim = dim3(kClusterThreads);
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg->attrs = at;
    cfg->numAttrs = 1;
    return active ? cudaOccupancyMaxActiveClusters(active, k_coarse_cluster<DIM, T>, cfg) : cudaSuccess;
}

// Cluster size for this device: 16 CTAs when the GPU can place such a
// cluster (non-portable size), else 8, else 0 (the per-level launches).
// Called outside any stream capture.
int coarse_cluster_setup(ss_sim* s) {
    if (s->cluster_ctas >= 0) return SS_OK;
    s->cluster_ctas = 0;
    if (!s->use_cluster || !s->cluster_from) return SS_OK;
    if (!s->cluster_fine) {
        const cudaError_t e = cudaMalloc((void**)&s->cluster_fine, kClusterCells * sizeof(float));
        if (e != cudaSuccess) return check_cuda(e, "cudaMalloc(cluster residuals)");
    }
    for (int ctas : {16, 8}) {
        cudaLaunchConfig_t cfg;
        cudaLaunchAttribute at[1];
        int active = 0, a2 = 0;
        cudaError_t e = s->dim == 3 ? cluster_config<3, __half>(ctas, &cfg, at, &active)
                                    : cluster_config<2, __half>(ctas, &cfg, at, &active);
        if (e == cudaSuccess)
            e = s->dim == 3 ? cluster_config<3, __nv_bfloat16>(ctas, &cfg, at, &a2)
                            : cluster_config<2, __nv_bfloat16>(ctas, &cfg, at, &a2);
        if (e != cudaSuccess) {
            cudaGetLastError();   // an unsupported size is not an error of the solve
            continue;
        }
        if (active >= 1 && a2 >= 1) {
            s->cluster_ctas = ctas;
            break;
        }
    }
    return SS_OK;
}

template <int DIM, typename T>
static int launch_cluster_t(ss_sim* s, const ss_mg_schedule& mg, int L, T* const* p, T* const* r, cudaStream_t st) {
    ClusterArgsT<T> b{};
    b.nlev = s->levels - L;
    for (int l = 0; l < b.nlev; ++l) {
        const ss::Level& lv = s->lv[L + l];
        b.n[l][0] = lv.n[0]; b.n[l][1] = lv.n[1]; b.n[l][2] = lv.n[2];
        b.hh[l] = lv.hh;
        b.p[l] = p[L + l];
        b.r[l] = r[L + l];
        b.alpha[l] = s->alpha[L + l];
    }
    b.n_pre = mg.n_pre; b.n_post = mg.n_post; b.n_coarse = mg.n_coarse;
    b.oob_smooth = smooth_oob(s, 0);
    b.oob_resid = resid_oob(s, 0);
    b.cmat = s->cmat;
    b.cpart = s->cmat_part;
    b.fine = s->cluster_fine;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[2];
    cudaError_t e = cluster_config<DIM, T>(s->cluster_ctas, &cfg, at, nullptr);
    if (e != cudaSuccess) return check_cuda(e, "cluster attributes");
    cfg.stream = st;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.numAttrs = s->pdl ? 2 : 1;
    e = cudaLaunchKernelEx(&cfg, k_coarse_cluster<DIM, T>, b);
    s->nlaunch += 1;
    return check_cuda(e, "k_coarse_cluster");
}

int coarse_cluster(ss_sim* s, const ss_mg_schedule& mg, int L, int prec, cudaStream_t st) {
    if (prec == SS_PREC_MIXED) {
        __half* const* p = (__half* const*)s->cp;
        __half* const* r = (__half* const*)s->cr;
        return s->dim == 3 ? launch_cluster_t<3, __half>(s, mg, L, p, r, st) : launch_cluster_t<2, __half>(s, mg, L, p, r, st);
    }
    __nv_bfloat16* const* p = (__nv_bfloat16* const*)s->cp;
    __nv_bfloat16* const* r = (__nv_bfloat16* const*)s->cr;
    return s->dim == 3 ? launch_cluster_t<3, __nv_bfloat16>(s, mg, L, p, r, st)
                       : launch_cluster_t<2, __nv_bfloat16>(s, mg, L, p, r, st);
}

int coarse_bottom(ss_sim* s, const ss_mg_schedule& mg, int L, int prec, cudaStream_t st) {
    if (prec == SS_PREC_MIXED)
        return launch_bottom_t<__half, __half>(s, mg, L, (__half* const*)s->cp, (__half* const*)s->cr, st);
    return launch_bottom_t<__nv_bfloat16, __nv_bfloat16>(s, mg, L, (__nv_bfloat16* const*)s->cp,
                                                         (__nv_bfloat16* const*)s->cr, st);
}

}  // namespace ss
