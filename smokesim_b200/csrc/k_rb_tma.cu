// k_rb_tma.cu - one colour of a level-0 red-black half-sweep (3D, colour-split
// arrays, four cells per thread) fed by a TMA pipeline.
//
// A block works on a segment of `boxx` half-cells of `ty` consecutive rows
// and marches up z.  Warp 8 is the producer: one elected lane issues, for
// every plane, three cp.async.bulk.tensor loads into a ring of kRbStages
// shared-memory stages - the other colour's pressure rows y0-1 .. y0+ty, with
// four extra columns on either side (the box starts on a 16-byte boundary and
// carries the row-end neighbours), and this colour's right-hand-side and
// fluid-mask rows.  Warps 0-7 are the consumers (one quad of four same-colour
// cells a thread): plane z is computed from the stages of planes z-1, z and
// z+1 as soon as their "full" barriers complete, after which the stage of
// plane z-1 is handed back through its "empty" barrier.  No block-wide
// barrier sits in the loop, so the producer runs up to kRbStages - 3 planes
// ahead and DRAM latency is hidden by the ring rather than by occupancy.
// Out-of-grid rows, columns and planes arrive as zeros - the pressure the
// operator assumes outside the grid.  The arithmetic per cell is
// k_rb_smooth4's in k_rb.cu (bit-identical results).  Every wait is bounded:
// a wait that gives up sets the error word and ends the warp's loop, and the
// producer lets the loads it issued land before it exits.
//
// The grid is persistent: the planes of all (segment, row block) columns are
// laid out column-major in z and split evenly among the blocks, so each
// block runs one or two uninterrupted pipelines of about the same length.
#include <algorithm>

#include "common.cuh"
#include "ss_internal.h"
#include "tma.cuh"

namespace ss {

constexpr int kRbStages = 6;
constexpr int kRbConsumers = 256;   // warps 0-7; warp 8 issues the loads

struct RbTmaArgs {
    float* pc;          // this colour's pressure (written)
    int* err;           // error word: bit 0 = a bounded wait gave up
    int half, ny, nz;   // colour-split level 0: half = nx / 2 cells per colour row
    int boxx, ty;       // segment width (half-cells) and rows per block
    int nseg, nrow;     // segments per row, row blocks per plane
    long long total;    // nseg * nrow * nz planes
    int colour;
};

struct RbStageLayout {
    size_t po, rhs, mask, stage;
    uint32_t po_tx, rm_tx;
};

__host__ __device__ inline RbStageLayout rb_stage_layout(int boxx, int ty) {
    RbStageLayout l;
    const int w = boxx + 8;
    l.po = ((size_t)w * (ty + 2) * 4 + 127) & ~(size_t)127;
    l.rhs = ((size_t)boxx * ty * 4 + 127) & ~(size_t)127;
    l.mask = ((size_t)boxx * ty + 127) & ~(size_t)127;
    l.stage = l.po + l.rhs + l.mask;
    l.po_tx = (uint32_t)(w * (ty + 2) * 4);
    l.rm_tx = (uint32_t)(boxx * ty * 5);
    return l;
}

// one plane's loads into a stage, completion counted on its barrier
SS_D void rb_issue_plane(uint64_t* bar, unsigned char* st, const RbStageLayout& lay, const CUtensorMap* tm_po,
                         const CUtensorMap* tm_rhs, const CUtensorMap* tm_mask, int xs, int y0, int z, bool rm) {
    mbar_expect_tx(bar, lay.po_tx + (rm ? lay.rm_tx : 0u));
    tma_load_3d(st, tm_po, xs - 4, y0 - 1, z, bar);
    if (rm) {
        tma_load_3d(st + lay.po, tm_rhs, xs, y0, z, bar);
        tma_load_3d(st + lay.po + lay.rhs, tm_mask, xs, y0, z, bar);
    }
}

// the planes of this block, split into pipelines of one column each
struct RbRange {
    long long L, L1;
};

__global__ void __launch_bounds__(kRbConsumers + 32, 3) k_rb_smooth_tma(const __grid_constant__ CUtensorMap tm_po,
                                                                     const __grid_constant__ CUtensorMap tm_rhs,
                                                                     const __grid_constant__ CUtensorMap tm_mask,
                                                                     RbTmaArgs a) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[kRbStages], empty[kRbStages];
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    const RbStageLayout lay = rb_stage_layout(a.boxx, a.ty);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < kRbStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kRbConsumers);
        }
        mbar_fence_init();
    }
    __syncthreads();
    const long long L0 = a.total * blockIdx.x / gridDim.x, L1 = a.total * (blockIdx.x + 1) / gridDim.x;
    // Planes are numbered j = 0, 1, ... in issue order over the block's
    // pipelines (zs-1 .. ze each): plane j uses stage j % S, and it is the
    // (j / S)-th use of that stage, waited for with parity (j / S) & 1.
    if (tid >= kRbConsumers) {
        // ---------------- producer warp
        if (tid != kRbConsumers) return;
        uint32_t j = 0;
        bool ok = true;
        for (long long L = L0; L < L1 && ok;) {
            const long long col = L / a.nz;
            const int zs = (int)(L - col * a.nz);
            const int ze = (int)min((long long)a.nz, (long long)zs + (L1 - L));
            L += ze - zs;
            const int xs = (int)(col % a.nseg) * a.boxx, y0 = (int)(col / a.nseg) * a.ty;
            for (int z = zs - 1; z <= ze; ++z, ++j) {
                const int s = j % kRbStages;
                const uint32_t use = j / kRbStages;
                if (use > 0 && !wait_bounded(&empty[s], (use - 1) & 1)) {
                    atomicOr(a.err, 1);
                    ok = false;
                    break;
                }
                rb_issue_plane(&full[s], base + s * lay.stage, lay, &tm_po, &tm_rhs, &tm_mask, xs, y0, z,
                               z >= zs && z < ze);
            }
        }
        // let every issued load land before the block's shared memory can go
        for (uint32_t k = j > kRbStages ? j - kRbStages : 0; k < j; ++k)
            wait_bounded(&full[k % kRbStages], (k / kRbStages) & 1);
        return;
    }
    // ---------------- consumer warps
    const int W = a.boxx + 8;
    const int qw = a.boxx >> 2;
    const int qx = tid % qw, ty = tid / qw;
    uint32_t J = 0;
    for (long long L = L0; L < L1;) {
        const long long col = L / a.nz;
        const int zs = (int)(L - col * a.nz);
        const int ze = (int)min((long long)a.nz, (long long)zs + (L1 - L));
        L += ze - zs;
        const int xs = (int)(col % a.nseg) * a.boxx, y0 = (int)(col / a.nseg) * a.ty;
        const uint32_t J0 = J;   // plane z of this pipeline <-> j = J0 + (z - zs + 1)
        auto jof = [&](int z) -> uint32_t { return J0 + (uint32_t)(z - zs + 1); };
        auto stage_of = [&](int z) -> unsigned char* { return base + (jof(z) % kRbStages) * lay.stage; };
        auto wait_full = [&](int z) -> bool {
            const uint32_t j = jof(z);
            if (wait_bounded(&full[j % kRbStages], (j / kRbStages) & 1)) return true;
            atomicOr(a.err, 1);
            return false;
        };
        auto release = [&](int z) { mbar_arrive(&empty[jof(z) % kRbStages]); };
        if (!wait_full(zs - 1) || !wait_full(zs)) return;
        const int y = y0 + ty, xh0 = xs + 4 * qx;
        for (int z = zs; z < ze; ++z) {
            if (!wait_full(z + 1)) return;
            if (y < a.ny) {
                const int row = (ty + 1) * W + 4 + 4 * qx;   // first cell of the quad in a pressure stage
                const float* Pk = reinterpret_cast<const float*>(stage_of(z - 1)) + row;
                const float* P0 = reinterpret_cast<const float*>(stage_of(z)) + row;
                const float* Pf = reinterpret_cast<const float*>(stage_of(z + 1)) + row;
                const unsigned char* S0 = stage_of(z);
                const float4 pm = *reinterpret_cast<const float4*>(P0);
                const float4 pt = *reinterpret_cast<const float4*>(P0 + W);
                const float4 pb = *reinterpret_cast<const float4*>(P0 - W);
                const float4 pf = *reinterpret_cast<const float4*>(Pf);
                const float4 pk = *reinterpret_cast<const float4*>(Pk);
                const int par = (y + z + a.colour) & 1;   // x = 2*xh + par
                // row-end neighbour: left of the first cell (par 0) or right of the last (par 1)
                const float extra = par == 0 ? P0[-1] : P0[4];
                const float4 rhs = *reinterpret_cast<const float4*>(
                    reinterpret_cast<const float*>(S0 + lay.po) + ty * a.boxx + 4 * qx);
                const uint32_t m4 = *reinterpret_cast<const uint32_t*>(S0 + lay.po + lay.rhs + ty * a.boxx + 4 * qx);
                release(z - 1);   // every read of the back plane is in registers
                const int i = (z * a.ny + y) * a.half + xh0;
                float out[4];
                bool wr[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint32_t m = (m4 >> (8 * k)) & 0xFFu;
                    const int fs = __popc(m & 0x7Eu);
                    wr[k] = (m & M_FLUID) && fs != 0;
                    const float left = par ? f4(pm, k) : (k ? f4(pm, k - 1) : extra);
                    const float right = par ? (k < 3 ? f4(pm, k + 1) : extra) : f4(pm, k);
                    float sum = ((m & M_TOP) ? f4(pt, k) : 0.f) + ((m & M_BOTTOM) ? f4(pb, k) : 0.f);
                    sum = sum + ((m & M_RIGHT) ? right : 0.f);
                    sum = sum + ((m & M_LEFT) ? left : 0.f);
                    sum = sum + ((m & M_FRONT) ? f4(pf, k) : 0.f);
                    sum = sum + ((m & M_BACK) ? f4(pk, k) : 0.f);
                    out[k] = wr[k] ? div_by_count(sum - f4(rhs, k), fs) : 0.f;
                }
                if (wr[0] && wr[1] && wr[2] && wr[3]) {
                    *reinterpret_cast<float4*>(a.pc + i) = make_float4(out[0], out[1], out[2], out[3]);
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (wr[k]) a.pc[i + k] = out[k];
                }
            } else {
                release(z - 1);
            }
        }
        release(ze - 1);
        release(ze);
        J = J0 + (uint32_t)(ze - zs + 2);
    }
}

// ------------------------------------------------------------------ host
// Segment width: the whole colour row when it is at most 128 half-cells,
// else 128-wide segments; 256 / (boxx / 4) rows per block.  The mask rows
// must be whole 16-byte units and the colour arrays 16-byte aligned.
static bool rb_tma_geometry(const ss_sim* s, int* boxx, int* ty) {
    const int half = s->nx / 2;
    if (s->dim != 3 || !s->rb_vec || s->use_tma < 2 || half % 16 != 0) return false;
    int b = half <= 128 ? half : (half % 128 == 0 ? 128 : 0);
    if (b != 16 && b != 32 && b != 64 && b != 128) return false;
    if (((size_t)half * s->ny * s->nz) % 16 != 0) return false;
    if (tma_encode_fn() == nullptr) return false;
    *boxx = b;
    *ty = 1024 / b;
    return true;
}

bool rb_tma_supported(const ss_sim* s) {
    int b, t;
    return rb_tma_geometry(s, &b, &t);
}

// One half-sweep of colour c: pc (this colour's pressure) from po (the other
// colour's), rhs and mask of colour c (the caller counts the launch).
int launch_rb_smooth_tma(ss_sim* s, float* pc, const float* po, const float* rhs, const uint8_t* mask, int colour,
                         cudaStream_t st) {
    int boxx, ty;
    if (!rb_tma_geometry(s, &boxx, &ty)) return set_error(SS_E_UNSUPPORTED, "TMA level-0 sweep: layout not supported");
    const int half = s->nx / 2;
    const int dims[3] = {half, s->ny, s->nz};
    const int pbox[3] = {boxx + 8, ty + 2, 1};
    const int rbox[3] = {boxx, ty, 1};
    CUtensorMap tp, tr, tm;
    int rc = tma_tensor_map(s, po, false, dims, pbox, &tp);
    if (!rc) rc = tma_tensor_map(s, rhs, false, dims, rbox, &tr);
    if (!rc) rc = tma_tensor_map(s, mask, true, dims, rbox, &tm);
    if (rc) return rc;
    const RbStageLayout lay = rb_stage_layout(boxx, ty);
    const size_t smem = kRbStages * lay.stage + 128;
    static int occ = 0, sms = 0;
    static size_t occ_smem = 0;
    if (occ == 0 || occ_smem != smem) {
        int dev = 0;
        rc = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        if (!rc) rc = check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
        if (!rc)
            rc = check_cuda(cudaFuncSetAttribute(k_rb_smooth_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(k_rb_smooth_tma)");
        if (!rc)
            rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rb_smooth_tma, kRbConsumers + 32, smem),
                            "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        if (rc) {
            occ = 0;
            return rc;
        }
        if (occ < 1) return set_error(SS_E_UNSUPPORTED, "TMA level-0 sweep does not fit an SM");
        occ_smem = smem;
    }
    RbTmaArgs a{};
    a.pc = pc;
    a.err = s->d_err;
    a.half = half; a.ny = s->ny; a.nz = s->nz;
    a.boxx = boxx; a.ty = ty;
    a.nseg = half / boxx;
    a.nrow = (s->ny + ty - 1) / ty;
    a.total = (long long)a.nseg * a.nrow * s->nz;
    a.colour = colour;
    // persistent grid: every resident block slot, but at least four planes a block
    long long blocks = (long long)sms * occ;
    blocks = std::max(1LL, std::min(blocks, a.total / 4));
    k_rb_smooth_tma<<<(unsigned)blocks, kRbConsumers + 32, smem, st>>>(tp, tr, tm, a);
    return check_cuda(cudaGetLastError(), "k_rb_smooth_tma");
}

}  // namespace ss
