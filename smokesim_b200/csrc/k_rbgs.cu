// k_rbgs.cu - one full red-black Gauss-Seidel sweep per launch, tiled in
// shared memory, with the neighbouring multigrid operations fused in.
//
// A thread block owns a TX x TY x TZ tile of the level and loads it with a
// halo of H cells (pressure, right-hand side, solid flags / fraction).  The
// red half-sweep then updates the red cells up to ring H-1, the black
// half-sweep the black cells up to ring H-2 - each half-sweep needs one more
// ring of the other colour - so the interior holds exactly the values of the
// reference's two dispatches (smooth.comp:79-136 with parity 0 then 1).  The
// pass reads p_in and writes p_out (separate buffers), so tiles never see a
// neighbour's new values through their halo.
//
// Fusions (each optional, bit-identical to the separate kernel):
//   PROLONG - the loaded pressure is p + prolong(p_coarse) (prolong_pressure.comp:39-51),
//             i.e. prolong_and_add is folded into the first post-smoothing sweep;
//   RESID   - after the sweep the residual of the interior (compute_residual.comp,
//             H = 3 so the last colour is valid one ring out) is restricted into
//             the coarse level (restrict_residual.comp) and, with the reference's
//             in-place rule, also written to r_out.
#include "common.cuh"
#include "ss_internal.h"

namespace ss {

struct TileArgs {
    const float* __restrict__ p_in;
    float* __restrict__ p_out;
    const float* __restrict__ rhs;       // L0: divergence (chosen boundary rule); L>0: r_L
    const uint8_t* __restrict__ flags;   // L0
    const float* __restrict__ alpha;     // L>0
    const float* __restrict__ pc;        // PROLONG: coarse pressure
    float* __restrict__ r_out;           // RESID with the in-place rule (L>0)
    float* __restrict__ rc;              // RESID: coarse right-hand side
    const float* __restrict__ rhs_r;     // RESID at L0: divergence under the residual's boundary rule
    int nx, ny, nz;
    int cx, cy, cz;                      // coarse level sizes
    float oob_smooth, oob_resid;         // solid fraction of out-of-grid neighbours
    float hh, rho_h, dt, rho, dt_h;
};

template <int DIM>
struct TileShape;
template <>
struct TileShape<3> {
    static constexpr int TX = 16, TY = 16, TZ = 16;
};
template <>
struct TileShape<2> {
    static constexpr int TX = 32, TY = 32, TZ = 1;
};

template <int DIM, bool L0, bool PROLONG, bool RESID>
__global__ void __launch_bounds__(256) k_rbgs_tile(TileArgs a) {
    constexpr int TX = TileShape<DIM>::TX, TY = TileShape<DIM>::TY, TZ = TileShape<DIM>::TZ;
    constexpr int H = RESID ? 3 : 2;
    constexpr int HZ = DIM == 3 ? H : 0;
    constexpr int LX = TX + 2 * H, LY = TY + 2 * H, LZ = TZ + 2 * HZ;
    constexpr int LN = LX * LY * LZ;
    extern __shared__ float smem[];
    float* sp = smem;
    float* sr = smem + LN;
    float* sa = smem + 2 * LN;                                  // L>0: alpha
    uint8_t* sf = reinterpret_cast<uint8_t*>(smem + 2 * LN);   // L0: flags

    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int gx0 = blockIdx.x * TX - H, gy0 = blockIdx.y * TY - H, gz0 = blockIdx.z * TZ - HZ;

    // ---- load the tile and its halo
    for (int q = threadIdx.x; q < LN; q += blockDim.x) {
        const int lx = q % LX, t = q / LX, ly = t % LY, lz = t / LY;
        const int x = gx0 + lx, y = gy0 + ly, z = gz0 + lz;
        const bool in = x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz;
        float pv = 0.f, rv = 0.f;
        if (in) {
            const int g = idx3(x, y, z, nx, ny);
            pv = __ldg(a.p_in + g);
            if constexpr (PROLONG) {
                const int cx = a.cx, cy = a.cy, cz = a.cz;
                const float tx = (((float)x + 0.5f) / (float)nx) * (float)cx - 0.5f;
                const float ty = (((float)y + 0.5f) / (float)ny) * (float)cy - 0.5f;
                const float fx = floorf(tx), fy = floorf(ty);
                const int x0 = (int)fx, y0 = (int)fy;
                const float wx = tx - fx, wy = ty - fy;
                const int xa = min(max(x0, 0), cx - 1), xb = min(max(x0 + 1, 0), cx - 1);
                const int ya = min(max(y0, 0), cy - 1), yb = min(max(y0 + 1, 0), cy - 1);
                const float* pc = a.pc;
                float s;
                if constexpr (DIM == 2) {
                    s = lerp_(lerp_(__ldg(pc + idx3(xa, ya, 0, cx, cy)), __ldg(pc + idx3(xb, ya, 0, cx, cy)), wx),
                              lerp_(__ldg(pc + idx3(xa, yb, 0, cx, cy)), __ldg(pc + idx3(xb, yb, 0, cx, cy)), wx), wy);
                } else {
                    const float tz = (((float)z + 0.5f) / (float)nz) * (float)cz - 0.5f;
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
                pv = pv + s;
            }
            rv = __ldg(a.rhs + g);
            if constexpr (L0) sf[q] = a.flags[g];
            else sa[q] = __ldg(a.alpha + g);
        } else {
            if constexpr (L0) sf[q] = 0;
            else sa[q] = 0.f;
        }
        sp[q] = pv;
        sr[q] = rv;
    }
    __syncthreads();

    // ---- red then black half-sweep on shrinking regions
#pragma unroll
    for (int colour = 0; colour < 2; ++colour) {
        const int R = H - 1 - colour;                 // ring reached by this half-sweep
        const int SX = TX + 2 * R, SY = TY + 2 * R, SZ = DIM == 3 ? TZ + 2 * R : 1;
        const int ox = H - R, oy = H - R, oz = DIM == 3 ? H - R : 0;
        const int half = SX / 2;
        for (int q = threadIdx.x; q < half * SY * SZ; q += blockDim.x) {
            const int xh = q % half, t = q / half, sy = t % SY, sz = t / SY;
            const int ly = oy + sy, lz = oz + sz;
            const int y = gy0 + ly, z = gz0 + lz;
            // x of this colour in the row: (x + y + z) & 1 == colour
            const int lx0 = ox + 2 * xh;
            const int x0 = gx0 + lx0;
            const int lx = lx0 + (((x0 + y + z) & 1) != colour ? 1 : 0);
            const int x = gx0 + lx;
            if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) continue;
            const int l = (lz * LY + ly) * LX + lx;
            float f_top, f_bottom, f_right, f_left, f_front = 0.f, f_back = 0.f;
            if constexpr (L0) {
                const uint8_t fl = sf[l];
                if (fl & F_SOLID) continue;
                const float fo = 1.f - a.oob_smooth;
                f_top = (fl & F_TOP) ? 0.f : (y + 1 < ny ? 1.f : fo);
                f_bottom = (fl & F_BOTTOM) ? 0.f : (y > 0 ? 1.f : fo);
                f_right = (fl & F_RIGHT) ? 0.f : (x + 1 < nx ? 1.f : fo);
                f_left = (fl & F_LEFT) ? 0.f : (x > 0 ? 1.f : fo);
                if constexpr (DIM == 3) {
                    f_front = (fl & F_FRONT) ? 0.f : (z + 1 < nz ? 1.f : fo);
                    f_back = (fl & F_BACK) ? 0.f : (z > 0 ? 1.f : fo);
                }
            } else {
                if (sa[l] >= 1.f) continue;
                f_top = 1.f - (y + 1 < ny ? sa[l + LX] : a.oob_smooth);
                f_bottom = 1.f - (y > 0 ? sa[l - LX] : a.oob_smooth);
                f_right = 1.f - (x + 1 < nx ? sa[l + 1] : a.oob_smooth);
                f_left = 1.f - (x > 0 ? sa[l - 1] : a.oob_smooth);
                if constexpr (DIM == 3) {
                    f_front = 1.f - (z + 1 < nz ? sa[l + LX * LY] : a.oob_smooth);
                    f_back = 1.f - (z > 0 ? sa[l - LX * LY] : a.oob_smooth);
                }
            }
            float f_sum = f_top + f_bottom + f_right + f_left;
            if constexpr (DIM == 3) f_sum = f_sum + f_front + f_back;
            if (f_sum == 0.f) continue;
            const float p_top = y + 1 < ny ? sp[l + LX] : 0.f;
            const float p_bottom = y > 0 ? sp[l - LX] : 0.f;
            const float p_right = x + 1 < nx ? sp[l + 1] : 0.f;
            const float p_left = x > 0 ? sp[l - 1] : 0.f;
            float p_sum = p_top * f_top + p_bottom * f_bottom;
            p_sum = p_sum + p_right * f_right;
            p_sum = p_sum + p_left * f_left;
            if constexpr (DIM == 3) {
                const float p_front = z + 1 < nz ? sp[l + LX * LY] : 0.f;
                const float p_back = z > 0 ? sp[l - LX * LY] : 0.f;
                p_sum = p_sum + p_front * f_front;
                p_sum = p_sum + p_back * f_back;
            }
            float pn;
            if constexpr (L0) pn = (p_sum - a.rho_h * sr[l] / a.dt) / f_sum;
            else pn = (p_sum - sr[l] * a.hh) / f_sum;
            sp[l] = pn;
        }
        __syncthreads();
    }

    // ---- write the interior
    for (int q = threadIdx.x; q < TX * TY * TZ; q += blockDim.x) {
        const int ix = q % TX, t = q / TX, iy = t % TY, iz = t / TY;
        const int x = gx0 + H + ix, y = gy0 + H + iy, z = gz0 + HZ + iz;
        if (x >= nx || y >= ny || z >= nz) continue;
        a.p_out[idx3(x, y, z, nx, ny)] = sp[((iz + HZ) * LY + (iy + H)) * LX + (ix + H)];
    }

    // ---- residual of the interior, restricted to the coarse level
    if constexpr (RESID) {
        const int hx = TX / 2, hy = TY / 2, hz = DIM == 3 ? TZ / 2 : 1;
        for (int q = threadIdx.x; q < hx * hy * hz; q += blockDim.x) {
            const int X = blockIdx.x * hx + q % hx;
            const int t = q / hx;
            const int Y = blockIdx.y * hy + t % hy;
            const int Z = DIM == 3 ? blockIdx.z * hz + t / hy : 0;
            float v[2][2][2];
#pragma unroll
            for (int dz = 0; dz < (DIM == 3 ? 2 : 1); ++dz)
#pragma unroll
                for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                    for (int dx = 0; dx < 2; ++dx) {
                        const int x = 2 * X + dx, y = 2 * Y + dy, z = DIM == 3 ? 2 * Z + dz : 0;
                        float res = 0.f;
                        if (x < nx && y < ny && z < nz) {
                            const int l = ((z - gz0) * LY + (y - gy0)) * LX + (x - gx0);
                            bool solid;
                            float f_top, f_bottom, f_right, f_left, f_front = 0.f, f_back = 0.f;
                            if constexpr (L0) {
                                const uint8_t fl = sf[l];
                                solid = fl & F_SOLID;
                                const float fo = 1.f - a.oob_resid;
                                f_top = (fl & F_TOP) ? 0.f : (y + 1 < ny ? 1.f : fo);
                                f_bottom = (fl & F_BOTTOM) ? 0.f : (y > 0 ? 1.f : fo);
                                f_right = (fl & F_RIGHT) ? 0.f : (x + 1 < nx ? 1.f : fo);
                                f_left = (fl & F_LEFT) ? 0.f : (x > 0 ? 1.f : fo);
                                if constexpr (DIM == 3) {
                                    f_front = (fl & F_FRONT) ? 0.f : (z + 1 < nz ? 1.f : fo);
                                    f_back = (fl & F_BACK) ? 0.f : (z > 0 ? 1.f : fo);
                                }
                            } else {
                                solid = sa[l] >= 1.f;
                                f_top = 1.f - (y + 1 < ny ? sa[l + LX] : a.oob_resid);
                                f_bottom = 1.f - (y > 0 ? sa[l - LX] : a.oob_resid);
                                f_right = 1.f - (x + 1 < nx ? sa[l + 1] : a.oob_resid);
                                f_left = 1.f - (x > 0 ? sa[l - 1] : a.oob_resid);
                                if constexpr (DIM == 3) {
                                    f_front = 1.f - (z + 1 < nz ? sa[l + LX * LY] : a.oob_resid);
                                    f_back = 1.f - (z > 0 ? sa[l - LX * LY] : a.oob_resid);
                                }
                            }
                            if (!solid) {
                                const float p_top = y + 1 < ny ? sp[l + LX] : 0.f;
                                const float p_bottom = y > 0 ? sp[l - LX] : 0.f;
                                const float p_right = x + 1 < nx ? sp[l + 1] : 0.f;
                                const float p_left = x > 0 ? sp[l - 1] : 0.f;
                                float p_sum = p_top * f_top + p_bottom * f_bottom;
                                p_sum = p_sum + p_right * f_right;
                                p_sum = p_sum + p_left * f_left;
                                float f_sum = f_top + f_bottom + f_right + f_left;
                                if constexpr (DIM == 3) {
                                    const float p_front = z + 1 < nz ? sp[l + LX * LY] : 0.f;
                                    const float p_back = z > 0 ? sp[l - LX * LY] : 0.f;
                                    p_sum = p_sum + p_front * f_front;
                                    p_sum = p_sum + p_back * f_back;
                                    f_sum = f_sum + f_front + f_back;
                                }
                                float old;
                                if constexpr (L0) old = a.rho * __ldg(a.rhs_r + idx3(x, y, z, nx, ny)) / a.dt_h;
                                else old = sr[l];
                                res = old - (p_sum - f_sum * sp[l]) / a.hh;
                            }
                            if (a.r_out) a.r_out[idx3(x, y, z, nx, ny)] = res;
                        }
                        v[dz][dy][dx] = res;
                    }
            if (X < a.cx && Y < a.cy && Z < a.cz) {
                float out;
                if constexpr (DIM == 3) {
                    const float bottom = v[0][0][0] + v[1][0][0] + v[0][0][1] + v[1][0][1];
                    const float top = v[0][1][0] + v[1][1][0] + v[0][1][1] + v[1][1][1];
                    out = (bottom + top) / 8.f;
                } else {
                    out = (v[0][0][0] + v[0][0][1] + v[0][1][0] + v[0][1][1]) / 4.f;
                }
                a.rc[idx3(X, Y, Z, a.cx, a.cy)] = out;
            }
        }
    }
}

template <int DIM, bool L0, bool PROLONG, bool RESID>
static int launch_tile_t(const TileArgs& a, cudaStream_t st) {
    constexpr int TX = TileShape<DIM>::TX, TY = TileShape<DIM>::TY, TZ = TileShape<DIM>::TZ;
    constexpr int H = RESID ? 3 : 2;
    constexpr int HZ = DIM == 3 ? H : 0;
    constexpr int LN = (TX + 2 * H) * (TY + 2 * H) * (TZ + 2 * HZ);
    const size_t smem = (size_t)LN * (L0 ? 9 : 12);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_rbgs_tile<DIM, L0, PROLONG, RESID>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute(k_rbgs_tile)");
        attr = true;
    }
    dim3 g((a.nx + TX - 1) / TX, (a.ny + TY - 1) / TY, DIM == 3 ? (a.nz + TZ - 1) / TZ : 1);
    k_rbgs_tile<DIM, L0, PROLONG, RESID><<<g, 256, smem, st>>>(a);
    return check_cuda(cudaGetLastError(), "k_rbgs_tile");
}

template <int DIM, bool L0>
static int launch_tile_d(const TileArgs& a, bool prolong, bool resid, cudaStream_t st) {
    if (prolong && resid) return launch_tile_t<DIM, L0, true, true>(a, st);
    if (prolong) return launch_tile_t<DIM, L0, true, false>(a, st);
    if (resid) return launch_tile_t<DIM, L0, false, true>(a, st);
    return launch_tile_t<DIM, L0, false, false>(a, st);
}

// One red-black sweep of level L in one launch; prolong: add the coarse
// correction first; resid: restrict the residual to level L+1 afterwards.
int launch_rbgs_sweep(ss_sim* s, const StepConsts& c, int L, int quirks, bool prolong, bool resid,
                      cudaStream_t st) {
    if (L > 0 && tma_sweep_supported(s, L)) {
        if (prolong) {
            int rc = launch_prolong(s, L, st);
            if (rc) return rc;
        }
        return launch_rbgs_sweep_tma(s, c, L, quirks, resid, st);
    }
    TileArgs a{};
    a.nx = s->lv[L].n[0]; a.ny = s->lv[L].n[1]; a.nz = s->lv[L].n[2];
    a.p_in = s->p[L];
    a.p_out = s->p_alt[L];
    a.oob_smooth = quirks ? 0.f : (s->enclosed ? 1.f : 0.f);
    a.oob_resid = quirks ? 1.f : (s->enclosed ? 1.f : 0.f);
    a.rhs = L == 0 ? (a.oob_smooth != 0.f ? s->div0r : s->div0) : s->r[L];
    a.rhs_r = L == 0 ? (a.oob_resid != 0.f ? s->div0r : s->div0) : nullptr;
    a.flags = s->flags;
    a.alpha = L > 0 ? s->alpha[L] : nullptr;
    a.hh = s->lv[L].hh;
    a.rho_h = c.rho_h; a.dt = c.dt; a.rho = c.rho; a.dt_h = c.dt_h;
    if (prolong || resid) {
        if (L + 1 >= s->levels) return set_error(SS_E_INVALID, "no coarser level");
        a.cx = s->lv[L + 1].n[0]; a.cy = s->lv[L + 1].n[1]; a.cz = s->lv[L + 1].n[2];
    }
    a.pc = prolong ? s->p[L + 1] : nullptr;
    a.rc = resid ? s->r[L + 1] : nullptr;
    const bool write_fine = resid && quirks && L > 0;
    a.r_out = write_fine ? s->r_alt[L] : nullptr;
    int rc;
    if (s->dim == 3) rc = L == 0 ? launch_tile_d<3, true>(a, prolong, resid, st) : launch_tile_d<3, false>(a, prolong, resid, st);
    else rc = L == 0 ? launch_tile_d<2, true>(a, prolong, resid, st) : launch_tile_d<2, false>(a, prolong, resid, st);
    if (rc) return rc;
    s->nlaunch += 1;
    float* t = s->p[L]; s->p[L] = s->p_alt[L]; s->p_alt[L] = t;
    if (write_fine) { t = s->r[L]; s->r[L] = s->r_alt[L]; s->r_alt[L] = t; }
    return SS_OK;
}

}  // namespace ss
