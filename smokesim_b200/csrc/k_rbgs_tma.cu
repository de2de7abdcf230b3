// k_rbgs_tma.cu - the tiled red-black sweep of k_rbgs.cu with its tile fetched
// by the Tensor Memory Accelerator.
//
// One elected thread issues three cp.async.bulk.tensor loads (pressure,
// right-hand side, solid flags or solid fraction) of the 16^3 tile plus its
// halo into shared memory; completion is counted in bytes on an mbarrier.
// The hardware fills out-of-grid texels with zeros, which is the pressure the
// operators assume outside the grid.  TMA requires the innermost box
// coordinate times the element size to be a multiple of 16 bytes, so the
// boxes start at x0-4 (floats, 24 wide) and x0-16 (bytes, 48 wide) instead of
// x0-H, and the row pitch of the level must be a multiple of 16 bytes
// (nx % 16 == 0); other levels use the per-thread loads of k_rbgs.cu.
// The arithmetic per cell is the same as k_rbgs_tile's (bit-identical).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <math.h>

#include <vector>

#include "common.cuh"
#include "ss_internal.h"
#include "tma.cuh"

namespace ss {

struct TmaArgs {
    float* __restrict__ p_out;
    const float* __restrict__ rhs_r;   // RESID at L0: rho*div/(dt*h) under the residual's rule (global)
    float* __restrict__ r_out;         // RESID with the in-place rule (L>0)
    float* __restrict__ rc;            // RESID: coarse right-hand side
    int* __restrict__ err;             // set when a barrier wait gives up
    int nx, ny, nz;
    int cx, cy, cz;
    float oob_smooth, oob_resid;
    float hh, inv_hh;                  // h^2 and, when h^2 is a power of two, its exact reciprocal
};

// Box geometry: pressure (and alpha) with the full halo H; the right-hand side
// and the flag bytes only out to ring H-1, the cells a half-sweep updates.
template <bool L0, bool RESID>
struct TmaGeom {
    static constexpr int T = 16;
    static constexpr int H = RESID ? 3 : 2;
    static constexpr int BX = 24;                 // float boxes start at x0 - 4
    static constexpr int FX = 48;                 // byte boxes start at x0 - 16
    static constexpr int PY = T + 2 * H;          // pressure / alpha box
    static constexpr int RY = T + 2 * (H - 1);    // rhs / flags box
    static constexpr int PB = BX * PY * PY * 4;
    static constexpr int RB = BX * RY * RY * 4;
    static constexpr int FB = L0 ? FX * RY * RY : PB;
    static constexpr int AL(int b) { return (b + 1023) / 1024 * 1024; }
    static constexpr int SMEM = AL(PB) + AL(RB) + AL(FB) + 1024;
};

template <bool L0, bool RESID, bool POW2>
__global__ void __launch_bounds__(256) k_rbgs_tma(const __grid_constant__ CUtensorMap tm_p,
                                                  const __grid_constant__ CUtensorMap tm_r,
                                                  const __grid_constant__ CUtensorMap tm_f, TmaArgs a) {
    using G = TmaGeom<L0, RESID>;
    constexpr int T = G::T, H = G::H, BX = G::BX, FX = G::FX, PY = G::PY, RY = G::RY;
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar;
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    float* sp = reinterpret_cast<float*>(base);
    float* sr = reinterpret_cast<float*>(base + G::AL(G::PB));
    unsigned char* sfb = base + G::AL(G::PB) + G::AL(G::RB);
    const uint8_t* sf = reinterpret_cast<const uint8_t*>(sfb);
    const float* sa = reinterpret_cast<const float*>(sfb);

    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int X0 = blockIdx.x * T, Y0 = blockIdx.y * T, Z0 = blockIdx.z * T;
    const int bx0 = X0 - 4, py0 = Y0 - H, pz0 = Z0 - H;          // pressure / alpha box
    const int ry0 = Y0 - (H - 1), rz0 = Z0 - (H - 1);            // rhs / flag box
    const int fx0 = X0 - 16;

    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, (uint32_t)(G::PB + G::RB + G::FB));
        tma_load_3d(sp, &tm_p, bx0, py0, pz0, &bar);
        tma_load_3d(sr, &tm_r, bx0, ry0, rz0, &bar);
        if constexpr (L0) tma_load_3d(sfb, &tm_f, fx0, ry0, rz0, &bar);
        else tma_load_3d(sfb, &tm_f, bx0, py0, pz0, &bar);
    }
    if (!wait_tile(&bar, 0, a.err)) return;

    // ---- red then black half-sweep; one thread per (x pair, y) column, marching in z
#pragma unroll
    for (int colour = 0; colour < 2; ++colour) {
        const int R = H - 1 - colour;
        const int S = T + 2 * R;
        const int half = S / 2;
        for (int col = threadIdx.x; col < half * S; col += blockDim.x) {
            const int xh = col % half, ys = col / half;
            const int y = Y0 - R + ys;
            if (y < 0 || y >= ny) continue;
            const int xs = X0 - R + 2 * xh;
            int z = Z0 - R;
            int lp = ((z - pz0) * PY + (y - py0)) * BX + (xs - bx0);
            int lr = ((z - rz0) * RY + (y - ry0)) * BX + (xs - bx0);
            int lf = ((z - rz0) * RY + (y - ry0)) * FX + (xs - fx0);
            for (int k = 0; k < S; ++k, ++z, lp += BX * PY, lr += BX * RY, lf += FX * RY) {
                const int dx = ((xs + y + z) & 1) != colour ? 1 : 0;
                const int x = xs + dx;
                if (x < 0 || z < 0 || x >= nx || z >= nz) continue;
                const int l = lp + dx;
                float f_top, f_bottom, f_right, f_left, f_front, f_back;
                if constexpr (L0) {
                    const uint8_t fl = sf[lf + dx];
                    if (fl & F_SOLID) continue;
                    const float fo = 1.f - a.oob_smooth;
                    f_top = (fl & F_TOP) ? 0.f : (y + 1 < ny ? 1.f : fo);
                    f_bottom = (fl & F_BOTTOM) ? 0.f : (y > 0 ? 1.f : fo);
                    f_right = (fl & F_RIGHT) ? 0.f : (x + 1 < nx ? 1.f : fo);
                    f_left = (fl & F_LEFT) ? 0.f : (x > 0 ? 1.f : fo);
                    f_front = (fl & F_FRONT) ? 0.f : (z + 1 < nz ? 1.f : fo);
                    f_back = (fl & F_BACK) ? 0.f : (z > 0 ? 1.f : fo);
                } else {
                    if (sa[l] >= 1.f) continue;
                    f_top = 1.f - (y + 1 < ny ? sa[l + BX] : a.oob_smooth);
                    f_bottom = 1.f - (y > 0 ? sa[l - BX] : a.oob_smooth);
                    f_right = 1.f - (x + 1 < nx ? sa[l + 1] : a.oob_smooth);
                    f_left = 1.f - (x > 0 ? sa[l - 1] : a.oob_smooth);
                    f_front = 1.f - (z + 1 < nz ? sa[l + BX * PY] : a.oob_smooth);
                    f_back = 1.f - (z > 0 ? sa[l - BX * PY] : a.oob_smooth);
                }
                float f_sum = f_top + f_bottom + f_right + f_left;
                f_sum = f_sum + f_front + f_back;
                if (f_sum == 0.f) continue;
                // out-of-grid pressure is 0: the TMA fill
                float p_sum = sp[l + BX] * f_top + sp[l - BX] * f_bottom;
                p_sum = p_sum + sp[l + 1] * f_right;
                p_sum = p_sum + sp[l - 1] * f_left;
                p_sum = p_sum + sp[l + BX * PY] * f_front;
                p_sum = p_sum + sp[l - BX * PY] * f_back;
                // L0: the rhs box holds rho*h*div/dt, precomputed with the same operations
                float rhs = sr[lr + dx];
                if constexpr (!L0) rhs = rhs * a.hh;   // (p_sum - r*h^2) / f_sum
                sp[l] = (p_sum - rhs) / f_sum;
            }
        }
        __syncthreads();
    }

    // ---- write the interior (rows of 16 floats)
    for (int q = threadIdx.x; q < T * T * T; q += blockDim.x) {
        const int ix = q & (T - 1), iy = (q / T) & (T - 1), iz = q / (T * T);
        const int x = X0 + ix, y = Y0 + iy, z = Z0 + iz;
        if (x >= nx || y >= ny || z >= nz) continue;
        a.p_out[idx3(x, y, z, nx, ny)] = sp[((z - pz0) * PY + (y - py0)) * BX + (x - bx0)];
    }

    // ---- residual of the interior, restricted to the coarse level
    if constexpr (RESID) {
        constexpr int hq = T / 2;
        for (int q = threadIdx.x; q < hq * hq * hq; q += blockDim.x) {
            const int X = blockIdx.x * hq + (q & (hq - 1));
            const int Y = blockIdx.y * hq + ((q / hq) & (hq - 1));
            const int Z = blockIdx.z * hq + q / (hq * hq);
            float v[2][2][2];
#pragma unroll
            for (int dz = 0; dz < 2; ++dz)
#pragma unroll
                for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                    for (int dxx = 0; dxx < 2; ++dxx) {
                        const int x = 2 * X + dxx, y = 2 * Y + dy, z = 2 * Z + dz;
                        float res = 0.f;
                        if (x < nx && y < ny && z < nz) {
                            const int l = ((z - pz0) * PY + (y - py0)) * BX + (x - bx0);
                            const int lr = ((z - rz0) * RY + (y - ry0)) * BX + (x - bx0);
                            bool solid;
                            float f_top, f_bottom, f_right, f_left, f_front, f_back;
                            if constexpr (L0) {
                                const uint8_t fl = sf[((z - rz0) * RY + (y - ry0)) * FX + (x - fx0)];
                                solid = fl & F_SOLID;
                                const float fo = 1.f - a.oob_resid;
                                f_top = (fl & F_TOP) ? 0.f : (y + 1 < ny ? 1.f : fo);
                                f_bottom = (fl & F_BOTTOM) ? 0.f : (y > 0 ? 1.f : fo);
                                f_right = (fl & F_RIGHT) ? 0.f : (x + 1 < nx ? 1.f : fo);
                                f_left = (fl & F_LEFT) ? 0.f : (x > 0 ? 1.f : fo);
                                f_front = (fl & F_FRONT) ? 0.f : (z + 1 < nz ? 1.f : fo);
                                f_back = (fl & F_BACK) ? 0.f : (z > 0 ? 1.f : fo);
                            } else {
                                solid = sa[l] >= 1.f;
                                f_top = 1.f - (y + 1 < ny ? sa[l + BX] : a.oob_resid);
                                f_bottom = 1.f - (y > 0 ? sa[l - BX] : a.oob_resid);
                                f_right = 1.f - (x + 1 < nx ? sa[l + 1] : a.oob_resid);
                                f_left = 1.f - (x > 0 ? sa[l - 1] : a.oob_resid);
                                f_front = 1.f - (z + 1 < nz ? sa[l + BX * PY] : a.oob_resid);
                                f_back = 1.f - (z > 0 ? sa[l - BX * PY] : a.oob_resid);
                            }
                            if (!solid) {
                                float p_sum = sp[l + BX] * f_top + sp[l - BX] * f_bottom;
                                p_sum = p_sum + sp[l + 1] * f_right;
                                p_sum = p_sum + sp[l - 1] * f_left;
                                float f_sum = f_top + f_bottom + f_right + f_left;
                                p_sum = p_sum + sp[l + BX * PY] * f_front;
                                p_sum = p_sum + sp[l - BX * PY] * f_back;
                                f_sum = f_sum + f_front + f_back;
                                float old;
                                if constexpr (L0) old = __ldg(a.rhs_r + idx3(x, y, z, nx, ny));
                                else old = sr[lr];
                                const float lap = p_sum - f_sum * sp[l];
                                res = old - (POW2 ? lap * a.inv_hh : lap / a.hh);
                            }
                            if (a.r_out) a.r_out[idx3(x, y, z, nx, ny)] = res;
                        }
                        v[dz][dy][dxx] = res;
                    }
            if (X < a.cx && Y < a.cy && Z < a.cz) {
                const float bottom = v[0][0][0] + v[1][0][0] + v[0][0][1] + v[1][0][1];
                const float top = v[0][1][0] + v[1][1][0] + v[0][1][1] + v[1][1][1];
                a.rc[idx3(X, Y, Z, a.cx, a.cy)] = (bottom + top) / 8.f;
            }
        }
    }
}

// ------------------------------------------------------------------ host
PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 3D tiled tensor map of an x-fastest array; cached per (address, box).
int tma_tensor_map(ss_sim* s, const void* ptr, bool bytes, const int dims[3], const int box[3], CUtensorMap* out) {
    for (const auto& e : s->tmaps) {
        if (e.ptr == ptr && e.bytes == bytes && e.box[0] == box[0] && e.box[1] == box[1] && e.box[2] == box[2] &&
            e.dims[0] == dims[0] && e.dims[1] == dims[1] && e.dims[2] == dims[2]) {
            *out = e.map;
            return SS_OK;
        }
    }
    auto fn = tma_encode_fn();
    if (!fn) return set_error(SS_E_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    const int es = bytes ? 1 : 4;
    cuuint64_t gdim[3] = {(cuuint64_t)dims[0], (cuuint64_t)dims[1], (cuuint64_t)dims[2]};
    cuuint64_t gstride[2] = {(cuuint64_t)dims[0] * es, (cuuint64_t)dims[0] * dims[1] * es};
    cuuint32_t bdim[3] = {(cuuint32_t)box[0], (cuuint32_t)box[1], (cuuint32_t)box[2]};
    cuuint32_t estr[3] = {1, 1, 1};
    TensorMapEntry e;
    CUresult r = fn(&e.map, bytes ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                    const_cast<void*>(ptr), gdim, gstride, bdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(SS_E_CUDA, "cuTensorMapEncodeTiled failed");
    e.ptr = ptr;
    e.bytes = bytes;
    for (int d = 0; d < 3; ++d) { e.dims[d] = dims[d]; e.box[d] = box[d]; }
    s->tmaps.push_back(e);
    *out = e.map;
    return SS_OK;
}

bool tma_sweep_supported(const ss_sim* s, int L) {
    // 16-byte row pitch for the flag bytes and whole 16^3 tiles' alignment rules
    return s->dim == 3 && s->use_tma && (s->lv[L].n[0] % 16) == 0 && tma_encode_fn() != nullptr;
}

template <bool L0, bool RESID, bool POW2>
static int launch_tma_t(ss_sim* s, const CUtensorMap& tp, const CUtensorMap& tr, const CUtensorMap& tf,
                        const TmaArgs& a, cudaStream_t st) {
    using G = TmaGeom<L0, RESID>;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_rbgs_tma<L0, RESID, POW2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             G::SMEM);
        if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute(k_rbgs_tma)");
        attr = true;
    }
    dim3 g((a.nx + 15) / 16, (a.ny + 15) / 16, (a.nz + 15) / 16);
    k_rbgs_tma<L0, RESID, POW2><<<g, 256, G::SMEM, st>>>(tp, tr, tf, a);
    return check_cuda(cudaGetLastError(), "k_rbgs_tma");
}

template <bool L0, bool RESID>
static int launch_tma_p(ss_sim* s, bool pow2, const CUtensorMap& tp, const CUtensorMap& tr, const CUtensorMap& tf,
                        const TmaArgs& a, cudaStream_t st) {
    return pow2 ? launch_tma_t<L0, RESID, true>(s, tp, tr, tf, a, st) : launch_tma_t<L0, RESID, false>(s, tp, tr, tf, a, st);
}

static bool is_pow2_float(float v) {
    if (!(v > 0.f) || !isfinite(v)) return false;
    int e;
    return frexpf(v, &e) == 0.5f && v >= 1.1754944e-38f && v <= 1e30f;
}

int launch_rbgs_sweep_tma(ss_sim* s, const StepConsts& c, int L, int quirks, bool resid, cudaStream_t st) {
    (void)c;
    const int dims[3] = {s->lv[L].n[0], s->lv[L].n[1], s->lv[L].n[2]};
    const int H = resid ? 3 : 2;
    const int pbox[3] = {24, 16 + 2 * H, 16 + 2 * H};
    const int rbox[3] = {24, 16 + 2 * (H - 1), 16 + 2 * (H - 1)};
    const int fbox[3] = {48, 16 + 2 * (H - 1), 16 + 2 * (H - 1)};
    TmaArgs a{};
    a.nx = dims[0]; a.ny = dims[1]; a.nz = dims[2];
    a.oob_smooth = quirks ? 0.f : (s->enclosed ? 1.f : 0.f);
    a.oob_resid = quirks ? 1.f : (s->enclosed ? 1.f : 0.f);
    a.hh = s->lv[L].hh;
    const bool pow2 = is_pow2_float(a.hh);
    a.inv_hh = pow2 ? 1.f / a.hh : 0.f;
    a.err = s->d_err;
    s->err_armed = 1;   // its bounded waits may set the error word
    a.p_out = s->p_alt[L];
    if (L == 0) return set_error(SS_E_UNSUPPORTED, "level 0 runs on the colour-split arrays");
    const float* rhs = s->r[L];
    a.rhs_r = nullptr;
    if (resid) {
        if (L + 1 >= s->levels) return set_error(SS_E_INVALID, "no coarser level");
        a.cx = s->lv[L + 1].n[0]; a.cy = s->lv[L + 1].n[1]; a.cz = s->lv[L + 1].n[2];
        a.rc = s->r[L + 1];
    }
    const bool write_fine = resid && quirks && L > 0;
    a.r_out = write_fine ? s->r_alt[L] : nullptr;
    CUtensorMap tp, tr, tf;
    int rc = tma_tensor_map(s, s->p[L], false, dims, pbox, &tp);
    if (!rc) rc = tma_tensor_map(s, rhs, false, dims, rbox, &tr);
    if (!rc) rc = L == 0 ? tma_tensor_map(s, s->flags, true, dims, fbox, &tf) : tma_tensor_map(s, s->alpha[L], false, dims, pbox, &tf);
    if (rc) return rc;
    if (L == 0) rc = resid ? launch_tma_p<true, true>(s, pow2, tp, tr, tf, a, st) : launch_tma_p<true, false>(s, pow2, tp, tr, tf, a, st);
    else rc = resid ? launch_tma_p<false, true>(s, pow2, tp, tr, tf, a, st) : launch_tma_p<false, false>(s, pow2, tp, tr, tf, a, st);
    if (rc) return rc;
    s->nlaunch += 1;
    float* t = s->p[L]; s->p[L] = s->p_alt[L]; s->p_alt[L] = t;
    if (write_fine) { t = s->r[L]; s->r[L] = s->r_alt[L]; s->r_alt[L] = t; }
    return SS_OK;
}

}  // namespace ss
