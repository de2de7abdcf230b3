// k_render.cu - headless renderer: the reference's smoke fragment shaders as
// CUDA kernels writing an RGBA8 image.
//
//  3D: ray_march_smoke.frag:114-175 - a ray per pixel through the box
//      [0, n/min(n)]^3, front-to-back compositing of alpha =
//      1 - exp(-density * smoke_density_factor * step) with a shadow march
//      of shadow_steps samples towards the light, light = ambient +
//      light_color * exp(-shadow density) * phase (Henyey-Greenstein,
//      g = 0.5, the shader's PI = 3.14 and factor 3), first sample jittered
//      by the shader's per-pixel sine hash, early exit below 0.001
//      transmittance.  Output (colour, 1 - transmittance).
//  2D: draw_smoke.frag:43-58 - mix(ambient, smoke / max channel, alpha).
// Texture fetches are the GL_LINEAR + CLAMP_TO_BORDER(0) filtering the
// simulation kernels use (texel centres at integers); the camera is a pinhole
// (the shader's inverse projection / look-at), and without a scene depth
// buffer every ray runs to the box exit.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "common.cuh"
#include "ss_internal.h"

namespace ss {

struct RenderArgs {
    int W, H;
    int nx, ny, nz, nch;
    const float* dens;
    float cam[3], fwd[3], right[3], up[3];
    float tan_half, aspect;
    float light[3];          // normalised
    float light_color[3], ambient[3];
    float kd, ks, step, shadow_step;
    int shadow_steps;
    float g;
    float box[3];
};

SS_D float fract_(float x) { return x - floorf(x); }

// smoke rgb at a box-space point (single channel: grey)
SS_D void smoke_rgb(const RenderArgs& a, float px, float py, float pz, float rgb[3]) {
    const float tx = (px / a.box[0]) * (float)a.nx - 0.5f;
    const float ty = (py / a.box[1]) * (float)a.ny - 0.5f;
    const float tz = (pz / a.box[2]) * (float)a.nz - 0.5f;
    const Taps t = make_taps<3>(a.nx, a.ny, a.nz, tx, ty, tz);
    const size_t n = (size_t)a.nx * a.ny * a.nz;
    rgb[0] = sample_taps_fast<3>(a.dens, a.nx, a.ny, a.nz, t, 0.f);
    if (a.nch == 3) {
        rgb[1] = sample_taps_fast<3>(a.dens + n, a.nx, a.ny, a.nz, t, 0.f);
        rgb[2] = sample_taps_fast<3>(a.dens + 2 * n, a.nx, a.ny, a.nz, t, 0.f);
    } else {
        rgb[1] = rgb[0];
        rgb[2] = rgb[0];
    }
}

SS_D unsigned char to_unorm8(float v) {
    v = fminf(fmaxf(v, 0.f), 1.f);
    return (unsigned char)(v * 255.f + 0.5f);
}

__global__ void __launch_bounds__(256) k_raymarch(RenderArgs a, uchar4* __restrict__ out) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= a.W || row >= a.H) return;
    const int py = a.H - 1 - row;   // the shader's gl_FragCoord.y runs upwards
    const float u = ((float)px + 0.5f) / (float)a.W, v = ((float)py + 0.5f) / (float)a.H;
    const float ndx = 2.f * u - 1.f, ndy = 2.f * v - 1.f;
    const float sx = ndx * a.tan_half * a.aspect, sy = ndy * a.tan_half;
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = a.fwd[k] + a.right[k] * sx + a.up[k] * sy;
    const float dl = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    float dir[3] = {d[0] / dl, d[1] / dl, d[2] / dl};
    // intersect_aabb(camera, dir, 0, box)
    float enter = -INFINITY, exit_ = INFINITY;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float inv = 1.f / dir[k];
        const float t0 = (0.f - a.cam[k]) * inv, t1 = (a.box[k] - a.cam[k]) * inv;
        enter = fmaxf(enter, fminf(t0, t1));
        exit_ = fminf(exit_, fmaxf(t0, t1));
    }
    const int o = row * a.W + px;
    if (exit_ < fmaxf(enter, 0.f)) {   // the shader discards the fragment
        out[o] = make_uchar4(0, 0, 0, 0);
        return;
    }
    const int steps = (int)((exit_ - enter) / a.step) + 1;
    const float noise = fract_(sinf(u * 12.9898f + v * 78.233f) * 43758.5453f);
    float t = enter + noise * a.step;
    // phase_function(g, dot(-dir, light)) * 3, with the shader's PI = 3.14
    const float cos_t = (-dir[0]) * a.light[0] + (-dir[1]) * a.light[1] + (-dir[2]) * a.light[2];
    float phase;
    if (a.g == 0.f) {
        phase = 1.f / 3.14f;
    } else {
        const float den = 1.f + a.g * a.g - 2.f * a.g * cos_t;
        phase = 1.f / (4.f * 3.14f) * (1.f - a.g * a.g) / (den * sqrtf(den));
    }
    phase = phase * 3.f;
    float T = 1.f;
    float col[3] = {0.f, 0.f, 0.f};
    for (int i = 0; i < steps; ++i) {
        if (t > exit_) break;
        const float pos[3] = {a.cam[0] + dir[0] * t, a.cam[1] + dir[1] * t, a.cam[2] + dir[2] * t};
        float rgb[3];
        smoke_rgb(a, pos[0], pos[1], pos[2], rgb);
        const float total = rgb[0] + rgb[1] + rgb[2];
        if (total > 0.001f) {
            float ld = 0.f;
            float lp[3] = {pos[0], pos[1], pos[2]};
            for (int j = 0; j < a.shadow_steps; ++j) {
#pragma unroll
                for (int k = 0; k < 3; ++k) lp[k] = lp[k] + a.light[k] * a.shadow_step;
                float s[3];
                smoke_rgb(a, lp[0], lp[1], lp[2], s);
                ld = ld + (s[0] + s[1] + s[2]);
            }
            const float atten = expf(-ld * a.ks * a.shadow_step);
            const float alpha = 1.f - expf(-total * a.kd * a.step);
            const float ta = T * alpha;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float light = a.ambient[k] + (a.light_color[k] * atten) * phase;
                col[k] = col[k] + ta * ((rgb[k] / total) * light);
            }
            T = T * (1.f - alpha);
            if (T < 0.001f) break;
        }
        t = t + a.step;
    }
    out[o] = make_uchar4(to_unorm8(col[0]), to_unorm8(col[1]), to_unorm8(col[2]), to_unorm8(1.f - T));
}

__global__ void __launch_bounds__(256) k_draw2d(RenderArgs a, uchar4* __restrict__ out) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= a.W || row >= a.H) return;
    const int py = a.H - 1 - row;
    const float u = ((float)px + 0.5f) / (float)a.W, v = ((float)py + 0.5f) / (float)a.H;
    const Taps t = make_taps<2>(a.nx, a.ny, 1, u * (float)a.nx - 0.5f, v * (float)a.ny - 0.5f, 0.f);
    const size_t n = (size_t)a.nx * a.ny;
    float rgb[3];
    rgb[0] = sample_taps<2>(a.dens, a.nx, a.ny, 1, t, 0.f);
    if (a.nch == 3) {
        rgb[1] = sample_taps<2>(a.dens + n, a.nx, a.ny, 1, t, 0.f);
        rgb[2] = sample_taps<2>(a.dens + 2 * n, a.nx, a.ny, 1, t, 0.f);
    } else {
        rgb[1] = rgb[0];
        rgb[2] = rgb[0];
    }
    const float raw = fmaxf(rgb[0], fmaxf(rgb[1], rgb[2]));
    const float alpha = 1.f - expf(-raw * a.kd);
    float c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float sc = raw > 0.001f ? rgb[k] / raw : 0.f;
        c[k] = a.ambient[k] * (1.f - alpha) + sc * alpha;   // mix(ambient, smoke, alpha)
    }
    out[row * a.W + px] = make_uchar4(to_unorm8(c[0]), to_unorm8(c[1]), to_unorm8(c[2]), 255);
}

static void normalize3(float v[3]) {
    const float l = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int k = 0; k < 3; ++k) v[k] = v[k] / l;
}

static void cross3(const float a[3], const float b[3], float o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace ss

using namespace ss;

extern "C" {

int ss_render_default(const ss_sim* s, int width, int height, ss_render_desc* d) {
    if (!s || !d || width < 1 || height < 1) return set_error(SS_E_INVALID, "NULL argument or empty image");
    memset(d, 0, sizeof *d);
    d->width = width;
    d->height = height;
    const float m = (float)std::min(s->nx, std::min(s->ny, s->dim == 3 ? s->nz : s->ny));
    const float box[3] = {(float)s->nx / m, (float)s->ny / m, s->dim == 3 ? (float)s->nz / m : 1.f};
    d->camera_target[0] = 0.5f * box[0]; d->camera_target[1] = 0.5f * box[1]; d->camera_target[2] = 0.5f * box[2];
    d->camera_pos[0] = 0.5f * box[0]; d->camera_pos[1] = 0.5f * box[1]; d->camera_pos[2] = box[2] + 1.8f;
    d->camera_up[1] = 1.f;
    d->fov_y = 0.78539816f;   // 45 degrees
    d->light_direction[0] = 1.f; d->light_direction[1] = 1.f; d->light_direction[2] = 1.f;
    d->light_color[0] = 1.5f; d->light_color[1] = 0.9f * 1.5f; d->light_color[2] = 0.8f * 1.5f;
    d->ambient_color[0] = 0.678f; d->ambient_color[1] = 0.847f; d->ambient_color[2] = 0.902f;
    d->smoke_density_factor = 50.f;
    d->shadow_density_factor = 50.f;
    d->step_size = 0.01f;
    d->shadow_step_factor = 3.f;
    d->shadow_steps = 6;
    d->phase_g = 0.5f;
    return SS_OK;
}

int ss_render(ss_sim* s, const ss_render_desc* d, uint8_t* rgba, int on_device, void* stream) {
    if (!s || !d || !rgba) return set_error(SS_E_INVALID, "NULL argument");
    if (d->width < 1 || d->height < 1 || (long long)d->width * d->height > (1ll << 28))
        return set_error(SS_E_INVALID, "image size out of range");
    if (!(d->step_size > 0.f) || d->shadow_steps < 0 || d->shadow_steps > 1024)
        return set_error(SS_E_INVALID, "step size / shadow steps out of range");
    const float* fl = &d->camera_pos[0];
    const size_t nf = (offsetof(ss_render_desc, shadow_steps) - offsetof(ss_render_desc, camera_pos)) / sizeof(float);
    for (size_t k = 0; k < nf; ++k)
        if (!std::isfinite(fl[k])) return set_error(SS_E_NONFINITE, "render parameter");
    if (!std::isfinite(d->phase_g)) return set_error(SS_E_NONFINITE, "render parameter");
    cudaStream_t st = (cudaStream_t)stream;
    RenderArgs a{};
    a.W = d->width; a.H = d->height;
    a.nx = s->nx; a.ny = s->ny; a.nz = s->nz; a.nch = s->nch;
    a.dens = s->dens[s->si];
    const float m = (float)std::min(s->nx, std::min(s->ny, s->dim == 3 ? s->nz : s->ny));
    a.box[0] = (float)s->nx / m; a.box[1] = (float)s->ny / m; a.box[2] = s->dim == 3 ? (float)s->nz / m : 1.f;
    for (int k = 0; k < 3; ++k) {
        a.cam[k] = d->camera_pos[k];
        a.fwd[k] = d->camera_target[k] - d->camera_pos[k];
        a.light[k] = d->light_direction[k];
        a.light_color[k] = d->light_color[k];
        a.ambient[k] = d->ambient_color[k];
    }
    normalize3(a.fwd);
    cross3(a.fwd, d->camera_up, a.right);
    normalize3(a.right);
    cross3(a.right, a.fwd, a.up);
    normalize3(a.light);
    a.tan_half = tanf(0.5f * d->fov_y);
    a.aspect = (float)d->width / (float)d->height;
    a.kd = d->smoke_density_factor;
    a.ks = d->shadow_density_factor;
    a.step = d->step_size;
    a.shadow_step = d->step_size * d->shadow_step_factor;
    a.shadow_steps = d->shadow_steps;
    a.g = d->phase_g;
    const size_t bytes = (size_t)d->width * d->height * 4;
    uchar4* dst = (uchar4*)rgba;
    if (!on_device) {
        if (s->render_bytes < bytes) {
            cudaFree(s->render_buf);
            s->render_buf = nullptr;
            s->render_bytes = 0;
            cudaError_t e = cudaMalloc(&s->render_buf, bytes);
            if (e != cudaSuccess) return check_cuda(e, "cudaMalloc(render)");
            s->render_bytes = bytes;
        }
        dst = (uchar4*)s->render_buf;
    }
    dim3 b(32, 8, 1), g((d->width + 31) / 32, (d->height + 7) / 8, 1);
    if (s->dim == 3) k_raymarch<<<g, b, 0, st>>>(a, dst);
    else k_draw2d<<<g, b, 0, st>>>(a, dst);
    int rc = check_cuda(cudaGetLastError(), "render");
    if (rc) return rc;
    if (!on_device) {
        rc = check_cuda(cudaMemcpyAsync(rgba, dst, bytes, cudaMemcpyDeviceToHost, st), "render read-back");
        if (rc) return rc;
        rc = check_cuda(cudaStreamSynchronize(st), "render sync");
    }
    return rc;
}

}  // extern "C"
