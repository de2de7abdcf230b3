// k_mixed.cu - FP64 parts of the mixed-precision pressure projection.
//
// The mixed solve keeps the level-0 pressure in FP64 (p64) and refines it:
// each iteration evaluates the fine-level residual of the projection in FP64,
//     rho_i = div_i - k * (sum_{fluid nb j} p64_j - n_i * p64_i),   k = dt/(rho h),
// which is exactly the divergence the velocity update would leave, hands it
// to one FP32 V-cycle as the right-hand side of the correction equation
// (level 0 FP32, coarse levels FP16/BF16 storage), and adds the correction
// back in FP64.  The residual norm (and its maximum, which sets the power-of-
// two scale of the coarse storage) are FP64 reductions.  Extension of the
// reference, whose multigrid_pressure_solve (common/physics/grid.c:173-209)
// runs FP32 V-cycles on the pressure itself.
#include <utility>

#include "common.cuh"
#include "ss_internal.h"

namespace ss {

static inline dim3 grid3(int ax, int ay, int az, dim3 b) {
    return dim3((ax + b.x - 1) / b.x, (ay + b.y - 1) / b.y, (az + b.z - 1) / b.z);
}

SS_D int rb_pos(int x, int y, int z, int nx, int ny, int nz) {
    const int half = nx >> 1;
    return (((x + y + z) & 1) ? half * ny * nz : 0) + (z * ny + y) * half + (x >> 1);
}

SS_D void block_sum_max(double v, double m, double* sum_out, double* max_out) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_down_sync(0xffffffffu, v, o);
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    }
    __shared__ double ws[32], wm[32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    if ((tid & 31) == 0) { ws[tid >> 5] = v; wm[tid >> 5] = m; }
    __syncthreads();
    if (tid < 32) {
        double r = tid < (nthreads + 31) / 32 ? ws[tid] : 0.0;
        double q = tid < (nthreads + 31) / 32 ? wm[tid] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_down_sync(0xffffffffu, r, o);
            q = fmax(q, __shfl_down_sync(0xffffffffu, q, o));
        }
        if (tid == 0) { *sum_out = r; *max_out = q; }
    }
}

__global__ void k_p64_from_f32(const float* __restrict__ p, double* __restrict__ p64, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p64[i] = (double)p[i];
}

__global__ void k_f32_from_p64(const double* __restrict__ p64, float* __restrict__ p, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = (float)p64[i];
}

// FP64 residual of the projection at every fluid cell; writes the FP32
// right-hand sides of the correction equation colour-split (smoother form
// rho/k, residual form rho/(k h^2)) and per-block sum of squares / max |rho|.
// With ACC the pending correction e (colour-split FP32) is first added to the
// fluid cells' pressure: p_out = p_in + e, and the residual is that of p_out
// (p_in and p_out are different buffers - neighbours read p_in + e).  Each
// block takes kIrChunk z planes of a 32x8 column, so a block reduces up to
// 256 * kIrChunk cells.
// A block owns a 32x8 column of cells and marches up kIrChunk z planes.  The
// pressure after the pending correction, P = p_in + e, is evaluated once per
// cell: the column's own values roll through registers (the z neighbours),
// each plane's tile plus its one-cell x/y rim goes through shared memory (the
// x and y neighbours), double-buffered so a plane costs one barrier.
constexpr int kIrTX = 32, kIrTY = 8, kIrChunk = 16;   // largest z chunk
constexpr int kIrRim = 2 * kIrTX + 2 * kIrTY;   // rim cells of a tile (no corners: 5/7-point stencil)

// DEC: the launch carries the device-side convergence test (IrDecide) of the
// tolerance loop's graph.  Only those instantiations contain the call that
// sets a graph condition; the others stay plain kernels (profilers skip graph
// kernel nodes that can set conditions).
template <int DIM, bool ACC, bool DEC = false>
__global__ void __launch_bounds__(kIrTX * kIrTY) k_ir_residual(
    const double* __restrict__ p_in, const float* __restrict__ e, double* __restrict__ p_out,
    const float* __restrict__ div0, const uint8_t* __restrict__ fmask, int nx, int ny, int nz, double k,
    double inv_k, double inv_khh, float* __restrict__ rhs_s, float* __restrict__ rhs_r, double* __restrict__ psum,
    double* __restrict__ pmax, unsigned int* __restrict__ ticket, double* __restrict__ out, int slot,
    float* __restrict__ scale, int planes, IrDecide dec) {
    pdl_entry();
    __shared__ double sP[2][kIrTY + 2][kIrTX + 2];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kIrTX * ty;
    const int x0 = blockIdx.x * kIrTX, y0 = blockIdx.y * kIrTY;
    const int x = x0 + tx, y = y0 + ty;
    const int zb = blockIdx.z * planes, ze = min(zb + planes, nz);
    const bool in = x < nx && y < ny;
    // this thread's rim cell (tid < kIrRim), in tile coordinates
    int hx = 0, hy = 0;
    if (tid < kIrTX) { hx = tid + 1; hy = 0; }
    else if (tid < 2 * kIrTX) { hx = tid - kIrTX + 1; hy = kIrTY + 1; }
    else if (tid < 2 * kIrTX + kIrTY) { hx = 0; hy = tid - 2 * kIrTX + 1; }
    else if (tid < kIrRim) { hx = kIrTX + 1; hy = tid - 2 * kIrTX - kIrTY + 1; }
    const int gx = x0 - 1 + hx, gy = y0 - 1 + hy;
    const bool hin = tid < kIrRim && gx >= 0 && gx < nx && gy >= 0 && gy < ny;
    auto P = [&](int xx, int yy, int zz) -> double {
        double v = p_in[idx3(xx, yy, zz, nx, ny)];
        if (ACC) v = v + (double)e[rb_pos(xx, yy, zz, nx, ny, nz)];
        return v;
    };
    double pm = 0.0, p0 = 0.0, pp = 0.0, h0 = 0.0;
    if (in) {
        if (zb > 0) pm = P(x, y, zb - 1);
        p0 = P(x, y, zb);
        if (zb + 1 < nz) pp = P(x, y, zb + 1);
    }
    if (hin) h0 = P(gx, gy, zb);
    uint8_t m = in ? fmask[idx3(x, y, zb, nx, ny)] : 0;
    float dv = in ? div0[idx3(x, y, zb, nx, ny)] : 0.f;
    double acc = 0.0, amax = 0.0;
    // The values the next two planes rotate in are in flight across each
    // plane's barrier and work: queue A holds what plane z+1 needs (its mask,
    // divergence and rim, and the pressure of plane z+2), queue B the same one
    // plane further, issued at the top of plane z.  They stay as loaded
    // (pressure and correction apart) and are combined only when they rotate
    // in, so no instruction waits on them early.
    struct Ahead {
        double p = 0.0, h = 0.0;
        float e = 0.f, he = 0.f, dv = 0.f;
        uint8_t m = 0;
    };
    auto fetch = [&](int zn, Ahead& A) {   // zn: the plane whose mask and rim the entry holds
        if (in && zn < ze) {
            if (zn + 1 < nz) {
                A.p = p_in[idx3(x, y, zn + 1, nx, ny)];
                if (ACC) A.e = e[rb_pos(x, y, zn + 1, nx, ny, nz)];
            }
            A.m = fmask[idx3(x, y, zn, nx, ny)];
            A.dv = div0[idx3(x, y, zn, nx, ny)];
        }
        if (hin && zn < ze) {
            A.h = p_in[idx3(gx, gy, zn, nx, ny)];
            if (ACC) A.he = e[rb_pos(gx, gy, zn, nx, ny, nz)];
        }
    };
    Ahead qa;
    fetch(zb + 1, qa);
    for (int z = zb; z < ze; ++z) {
        const int sl = z & 1;
        sP[sl][ty + 1][tx + 1] = p0;
        if (tid < kIrRim) sP[sl][hy][hx] = h0;
        Ahead qb;
        fetch(z + 2, qb);
        const int c = idx3(x, y, z, nx, ny);
        __syncthreads();
        if (in) {
            const int q = rb_pos(x, y, z, nx, ny, nz);
            float s_out = 0.f, r_out = 0.f;
            if (m & M_FLUID) {
                // out-of-grid neighbours (a set bit on an open grid) hold +0 in the
                // tile, the rim and the z registers: no bounds tests needed
                const double t = (m & M_TOP) ? sP[sl][ty + 2][tx + 1] : 0.0;
                const double b = (m & M_BOTTOM) ? sP[sl][ty][tx + 1] : 0.0;
                const double r = (m & M_RIGHT) ? sP[sl][ty + 1][tx + 2] : 0.0;
                const double l = (m & M_LEFT) ? sP[sl][ty + 1][tx] : 0.0;
                double sum = t + b;
                sum = sum + r;
                sum = sum + l;
                if constexpr (DIM == 3) {
                    const double f = (m & M_FRONT) ? pp : 0.0;
                    const double k2 = (m & M_BACK) ? pm : 0.0;
                    sum = sum + f;
                    sum = sum + k2;
                }
                if (ACC) p_out[c] = p0;
                const double cnt = (double)__popc(m & 0x7Eu);
                const double rho = (double)dv - k * (sum - cnt * p0);
                acc += rho * rho;
                const double ar = fabs(rho);
                amax = ar > amax ? ar : amax;
                s_out = (float)(rho * inv_k);
                r_out = (float)(rho * inv_khh);
            } else if (ACC) {
                p_out[c] = p_in[c];
            }
            rhs_s[q] = s_out;
            if (rhs_r) rhs_r[q] = r_out;
        }
        pm = p0;
        p0 = pp;
        pp = ACC ? qa.p + (double)qa.e : qa.p;   // P(x, y, z + 2): the same value P() forms
        h0 = ACC ? qa.h + (double)qa.he : qa.h;
        m = qa.m;
        dv = qa.dv;
        qa = qb;
    }
    block_sum_max(acc, amax, psum + blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
                  pmax + blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z));
    // The last block to finish folds every block's partials: each thread sums
    // a fixed stride of them, then a fixed tree - the same order whichever
    // block is last.  It writes the residual norm (slot >= 0), max |rho| and
    // the power-of-two scale of the coarse storage derived from it - with
    // max|rho| / (k h^2) = m * 2^e (m in [0.5, 1)) the restricted residual is
    // multiplied by 2^-e on its way to the FP16 / BF16 level and the prolonged
    // correction by 2^e on its way back - and re-arms the ticket for the next
    // launch.
    const unsigned int nblocks = gridDim.x * gridDim.y * gridDim.z;
    __shared__ bool last;
    if (tid == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == nblocks - 1;
    }
    __syncthreads();
    if (!last) return;
    // (one load in flight per thread: the eight-accumulator fold costs this
    // kernel registers, and so occupancy, in its main loop)
    double s = 0.0, mx = 0.0;
    for (unsigned int i = tid; i < nblocks; i += kIrTX * kIrTY) {
        s += __ldcg(psum + i);
        mx = fmax(mx, __ldcg(pmax + i));
    }
    __shared__ double fs[kIrTX * kIrTY], fm[kIrTX * kIrTY];
    fs[tid] = s;
    fm[tid] = mx;
    __syncthreads();
    for (int o = kIrTX * kIrTY / 2; o > 0; o >>= 1) {
        if (tid < o) {
            fs[tid] += fs[tid + o];
            fm[tid] = fmax(fm[tid], fm[tid + o]);
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (slot >= 0) out[slot] = fs[0];
        out[SLOT_AMAX] = fm[0];
        int e = 0;
        frexp(fm[0] * inv_khh, &e);
        e = max(-100, min(100, e));
        scale[0] = (float)ldexp(1.0, -e);
        scale[1] = (float)ldexp(1.0, e);
        *ticket = 0u;
        if (DEC && dec.active) {
            // the host loop's test, on the same doubles: stop once
            // sqrt(residual) <= tol sqrt(divergence before the solve)
            out[SLOT_STEPS] = (double)dec.k;
            const double res = sqrt(fs[0]), db = sqrt(out[SLOT_DIV_BEFORE]);
            if (dec.more && !(res <= dec.tol * db)) cudaGraphSetConditional(dec.next, 1u);
        }
    }
}


// p64 += e at every fluid cell (e: the correction, colour-split FP32)
template <int DIM>
__global__ void __launch_bounds__(256) k_ir_accumulate(double* __restrict__ p64, const float* __restrict__ e,
                                                       const uint8_t* __restrict__ fmask, int nx, int ny, int nz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= nx || y >= ny || z >= nz) return;
    const int c = idx3(x, y, z, nx, ny);
    if (!(fmask[c] & M_FLUID)) return;
    p64[c] = p64[c] + (double)e[rb_pos(x, y, z, nx, ny, nz)];
}

int launch_p64_from_p0(ss_sim* s, cudaStream_t st) {
    k_p64_from_f32<<<4 * 148, 256, 0, st>>>(s->p[0], s->p64, s->ncell);
    s->nlaunch += 1;
    s->p64_valid = 1;
    return check_cuda(cudaGetLastError(), "k_p64_from_f32");
}


int launch_p0_from_p64(ss_sim* s, cudaStream_t st) {
    k_f32_from_p64<<<4 * 148, 256, 0, st>>>(s->p64, s->p[0], s->ncell);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_f32_from_p64");
}

int launch_ir_residual(ss_sim* s, const StepConsts& c, int slot, bool accumulate, cudaStream_t st,
                       const IrDecide* dec) {
    const IrDecide d = dec ? *dec : IrDecide{};
    if (d.active && slot != SLOT_RESIDUAL) return set_error(SS_E_INVALID, "the convergence test reads the residual slot");
    dim3 b(kIrTX, kIrTY, 1);
    const int tx = (s->nx + kIrTX - 1) / kIrTX, ty = (s->ny + kIrTY - 1) / kIrTY;
    const int planes = z_planes((long long)tx * ty, s->nz, kIrChunk);
    dim3 g(tx, ty, (s->nz + planes - 1) / planes);
    const int nblocks = (int)(g.x * g.y * g.z);
    if (nblocks > s->red.max_blocks) return set_error(SS_E_INVALID, "reduction scratch too small");
    const double k = (double)c.dt / ((double)c.rho * (double)s->h);
    const double inv_k = 1.0 / k;
    const double inv_khh = 1.0 / (k * (double)s->lv[0].hh);
    // with h^2 == 1 the residual form rho/(k h^2) is the smoother form rho/k
    // to the bit: only rhs_s is written, and the level-0 residual reads it
    s->rhs_r_is_s = s->lv[0].hh == 1.0f ? 1 : 0;
    float* rhs_r = s->rhs_r_is_s ? nullptr : s->rhs_r;
#define IR_ARGS(ACC) s->p64, s->p_alt[0], s->p64b, s->div0, s->fmask, s->nx, s->ny, s->nz, k, inv_k, inv_khh, \
                     s->rhs_s, rhs_r, s->red.partial, s->red.partial_max, s->red.ticket, s->red.out, slot, \
                     s->d_scale, planes, d
    if (s->dim == 3) {
        if (d.active) {
            if (accumulate) launch_k(s->pdl, g, b, 0, st, k_ir_residual<3, true, true>, IR_ARGS(true));
            else launch_k(s->pdl, g, b, 0, st, k_ir_residual<3, false, true>, IR_ARGS(false));
        } else {
            if (accumulate) launch_k(s->pdl, g, b, 0, st, k_ir_residual<3, true>, IR_ARGS(true));
            else launch_k(s->pdl, g, b, 0, st, k_ir_residual<3, false>, IR_ARGS(false));
        }
    } else {
        if (d.active) {
            if (accumulate) launch_k(s->pdl, g, b, 0, st, k_ir_residual<2, true, true>, IR_ARGS(true));
            else launch_k(s->pdl, g, b, 0, st, k_ir_residual<2, false, true>, IR_ARGS(false));
        } else {
            if (accumulate) launch_k(s->pdl, g, b, 0, st, k_ir_residual<2, true>, IR_ARGS(true));
            else launch_k(s->pdl, g, b, 0, st, k_ir_residual<2, false>, IR_ARGS(false));
        }
    }
#undef IR_ARGS
    s->nlaunch += 1;
    int rc = check_cuda(cudaGetLastError(), "k_ir_residual");
    if (rc) return rc;
    // with accumulate the caller swaps s->p64 / s->p64b afterwards (the launch
    // may be recorded into a graph and replayed, the swap is host state); the
    // norms and the coarse scale are folded by the kernel's last block
    return rc;
}

int launch_ir_accumulate(ss_sim* s, cudaStream_t st) {
    dim3 b(32, 8, 1);
    dim3 g = grid3(s->nx, s->ny, s->nz, b);
    if (s->dim == 3) k_ir_accumulate<3><<<g, b, 0, st>>>(s->p64, s->p_alt[0], s->fmask, s->nx, s->ny, s->nz);
    else k_ir_accumulate<2><<<g, b, 0, st>>>(s->p64, s->p_alt[0], s->fmask, s->nx, s->ny, s->nz);
    s->nlaunch += 1;
    return check_cuda(cudaGetLastError(), "k_ir_accumulate");
}

}  // namespace ss
