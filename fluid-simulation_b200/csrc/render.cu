// render.cu — headless impostor-sphere rendering of the particles into a
// device image (the particle view of the reference's renderer without a
// graphics stack).
//
// The reference draws each particle as a camera-facing quad of half-width
// RADIUS (shaders/instanced_ball.vert:20-32) and shades it as a sphere in the
// fragment shader (shaders/instanced_ball.frag): billboard coordinates c in the
// unit disk give the normal n = (c, sqrt(1 - |c|^2)), the depth of the point
// center_view + n R, and the colour base * n.z, where base is the fluid or
// boundary colour or a visualised field.
//
// Here each particle is one thread: it projects its quad to a pixel box and,
// for every pixel centre in the box, intersects the pixel's view ray with the
// quad's plane. The hit point's coordinates in the quad's (right, up) frame
// divided by R are the billboard coordinates the rasteriser would interpolate
// (perspective-correct interpolation of an attribute that is linear on the
// plane). The depth test is an atomicMin on (depth bits << 32 | rgba8): the
// nearest fragment wins; equal depths keep the smaller colour word.
#include <cmath>

#include "render.cuh"

namespace wcsph {

namespace {

__device__ __forceinline__ float3 mat_vec3(const float* m, float3 v, float w, float& ow) {
    // column-major 4x4 times (v, w)
    const float x = m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12] * w;
    const float y = m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13] * w;
    const float z = m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14] * w;
    ow = m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15] * w;
    return make_float3(x, y, z);
}

__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 scale3(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3f(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 a) { return scale3(a, rsqrtf(dot3f(a, a))); }

__device__ __forceinline__ u32 to_u8(float c) {
    c = fminf(fmaxf(c, 0.f), 1.f);
    return static_cast<u32>(__float2int_rn(c * 255.f));
}

__global__ void splat_kernel(const RenderArgs r, const float4* __restrict__ fluid, u32 nf,
                             const float4* __restrict__ boundary, u32 nb, const float* __restrict__ scalar,
                             const float4* __restrict__ vec, unsigned long long* __restrict__ zbuf) {
    const u32 id = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 total = nf + (r.show_boundary ? nb : 0u);
    if (id >= total) return;
    const bool is_boundary = id >= nf;
    const float4 q = is_boundary ? boundary[id - nf] : fluid[id];
    const float3 p = make_float3(q.x, q.y, q.z);
    const float3 eye = make_float3(r.eye[0], r.eye[1], r.eye[2]);
    // billboard frame (instanced_ball.vert): to_camera, right = up0 x to_camera, up = to_camera x right
    const float3 to_cam3 = sub3(eye, p);
    if (dot3f(to_cam3, to_cam3) <= 0.f) return;
    const float3 to_cam = normalize3(to_cam3);
    const float3 rc = cross3(make_float3(0.f, 1.f, 0.f), to_cam);
    const float rl2 = dot3f(rc, rc);
    if (!(rl2 > 1e-20f)) return;   // camera straight above or below: no frame
    const float3 right = scale3(rc, rsqrtf(rl2));
    const float3 up = cross3(to_cam, right);
    const float R = r.radius;
    // pixel box of the quad's corners (skip quads that reach behind the camera)
    float xmin = 1e30f, xmax = -1e30f, ymin = 1e30f, ymax = -1e30f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float sx = (c & 1) ? R : -R, sy = (c & 2) ? R : -R;
        const float3 wp = add3(p, add3(scale3(right, sx), scale3(up, sy)));
        float w;
        const float3 cp = mat_vec3(r.vp, wp, 1.f, w);
        if (!(w > 1e-6f)) return;
        const float px = (cp.x / w * 0.5f + 0.5f) * static_cast<float>(r.width);
        const float py = (cp.y / w * 0.5f + 0.5f) * static_cast<float>(r.height);
        xmin = fminf(xmin, px); xmax = fmaxf(xmax, px);
        ymin = fminf(ymin, py); ymax = fmaxf(ymax, py);
    }
    if (!(isfinite(xmin) && isfinite(xmax) && isfinite(ymin) && isfinite(ymax))) return;
    // pixel centres (x + 0.5, y + 0.5) inside [min, max], clamped to the image before any cast
    const float fx0 = fmaxf(ceilf(xmin - 0.5f), 0.f);
    const float fx1 = fminf(floorf(xmax - 0.5f), static_cast<float>(r.width) - 1.f);
    const float fy0 = fmaxf(ceilf(ymin - 0.5f), 0.f);
    const float fy1 = fminf(floorf(ymax - 0.5f), static_cast<float>(r.height) - 1.f);
    if (fx0 > fx1 || fy0 > fy1) return;
    const int x0 = static_cast<int>(fx0), x1 = static_cast<int>(fx1);
    const int y0 = static_cast<int>(fy0), y1 = static_cast<int>(fy1);
    if ((x1 - x0 + 1) * (y1 - y0 + 1) > r.max_pixels) return;   // bounded work per particle

    // colour (instanced_ball.frag)
    float3 base = is_boundary ? make_float3(1.f, 0.5f, 0.f) : make_float3(0.f, 0.5f, 1.f);
    const bool vis = r.mode != RENDER_PLAIN && !is_boundary;
    float sval = 0.f;
    float3 vval = make_float3(0.f, 0.f, 0.f);
    if (vis && r.mode == RENDER_SCALAR) sval = scalar[id];
    if (vis && r.mode == RENDER_VECTOR) { const float4 t = vec[id]; vval = make_float3(t.x, t.y, t.z); }
    float wc;
    const float3 center_view = mat_vec3(r.view, p, 1.f, wc);
    const float pn = dot3f(p, to_cam);

    for (int y = y0; y <= y1; ++y) {
        for (int x = x0; x <= x1; ++x) {
            // view ray of the pixel centre: far-plane point of the inverse view-projection
            const float ndx = (static_cast<float>(x) + 0.5f) / static_cast<float>(r.width) * 2.f - 1.f;
            const float ndy = (static_cast<float>(y) + 0.5f) / static_cast<float>(r.height) * 2.f - 1.f;
            float fw;
            const float3 fp = mat_vec3(r.inv_vp, make_float3(ndx, ndy, 1.f), 1.f, fw);
            const float3 d = sub3(scale3(fp, 1.f / fw), eye);
            const float den = dot3f(d, to_cam);
            if (!(fabsf(den) > 1e-20f)) continue;
            const float t = (pn - dot3f(eye, to_cam)) / den;
            const float3 h = sub3(add3(eye, scale3(d, t)), p);
            const float cx = dot3f(h, right) / R, cy = dot3f(h, up) / R;
            float nz = 1.f - (cx * cx + cy * cy);
            if (nz < 0.f) continue;
            nz = sqrtf(nz);
            const float3 n = make_float3(cx, cy, nz);
            const float3 vpos = add3(center_view, scale3(n, R));
            float cw;
            const float3 cp = mat_vec3(r.proj, vpos, 1.f, cw);
            const float depth = cp.z / cw * 0.5f + 0.5f;
            if (!(depth >= 0.f && depth <= 1.f)) continue;
            float3 col = base;
            if (vis) {
                if (r.mode == RENDER_SCALAR) col = make_float3(sval, sval, sval);
                else col = scale3(base, dot3f(vval, n));
                if (r.normalize) {
                    const float inv = 1.f / (r.max_value - r.min_value);
                    col = make_float3((col.x - r.min_value) * inv, (col.y - r.min_value) * inv,
                                      (col.z - r.min_value) * inv);
                }
            }
            col = scale3(col, nz);   // dot(n, (0, 0, 1))
            const u32 rgba = to_u8(col.x) | (to_u8(col.y) << 8) | (to_u8(col.z) << 16) | (255u << 24);
            const unsigned long long key =
                (static_cast<unsigned long long>(__float_as_uint(depth)) << 32) | rgba;
            // image row 0 is the top row
            const size_t pix = static_cast<size_t>(r.height - 1 - y) * r.width + x;
            atomicMin(zbuf + pix, key);
        }
    }
}

__global__ void resolve_kernel(const unsigned long long* __restrict__ zbuf, u32 npix, u32 background,
                               u32* __restrict__ rgba, float* __restrict__ depth) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const unsigned long long k = zbuf[i];
    const bool empty = k == ~0ull;
    rgba[i] = empty ? background : static_cast<u32>(k & 0xffffffffull);
    if (depth) depth[i] = empty ? 1.f : __uint_as_float(static_cast<u32>(k >> 32));
}

}  // namespace

void enqueue_render(const RenderArgs& r, const float4* fluid, u32 nf, const float4* boundary, u32 nb,
                    const float* scalar, const float4* vec, unsigned long long* zbuf, u32* rgba, float* depth,
                    cudaStream_t stream) {
    const u32 npix = r.width * r.height;
    cudaMemsetAsync(zbuf, 0xff, sizeof(unsigned long long) * npix, stream);
    const u32 total = nf + (r.show_boundary ? nb : 0u);
    if (total) splat_kernel<<<(total + 127) / 128, 128, 0, stream>>>(r, fluid, nf, boundary, nb, scalar, vec, zbuf);
    const u32 bg = (static_cast<u32>(std::lround(std::fmin(std::fmax(r.background[0], 0.f), 1.f) * 255.f))) |
                   (static_cast<u32>(std::lround(std::fmin(std::fmax(r.background[1], 0.f), 1.f) * 255.f)) << 8) |
                   (static_cast<u32>(std::lround(std::fmin(std::fmax(r.background[2], 0.f), 1.f) * 255.f)) << 16) |
                   (255u << 24);
    resolve_kernel<<<(npix + 255) / 256, 256, 0, stream>>>(zbuf, npix, bg, rgba, depth);
}

// ---- camera (glm::perspective / glm::lookAt conventions, column-major) ------
void mat4_mul(const float* a, const float* b, float* out) {
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += static_cast<double>(a[k * 4 + r]) * b[c * 4 + k];
            out[c * 4 + r] = static_cast<float>(s);
        }
}

bool mat4_inverse(const float* m, float* out) {
    // Gauss-Jordan on a row-major copy in double
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            a[r][c] = m[c * 4 + r];
            a[r][c + 4] = r == c ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int r = c + 1; r < 4; ++r) if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
        if (std::fabs(a[piv][c]) < 1e-300) return false;
        if (piv != c) for (int k = 0; k < 8; ++k) std::swap(a[c][k], a[piv][k]);
        const double inv = 1.0 / a[c][c];
        for (int k = 0; k < 8; ++k) a[c][k] *= inv;
        for (int r = 0; r < 4; ++r) {
            if (r == c) continue;
            const double f = a[r][c];
            for (int k = 0; k < 8; ++k) a[r][k] -= f * a[c][k];
        }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) out[c * 4 + r] = static_cast<float>(a[r][c + 4]);
    return true;
}

}  // namespace wcsph

extern "C" void wcsph_camera_look(const float position[3], float yaw, float pitch, uint32_t width,
                                  uint32_t height, wcsph_camera* out) {
    if (!position || !out) return;
    // Camera::update_vectors / set_view / set_projection (src/render/camera.cpp:7-33):
    // FOV 45 deg, near 0.1, far 100, world up (0, 1, 0)
    const double fx = std::cos(yaw) * std::cos(pitch), fy = std::sin(pitch), fz = std::sin(yaw) * std::cos(pitch);
    const double fl = std::sqrt(fx * fx + fy * fy + fz * fz);
    const double f[3] = {fx / fl, fy / fl, fz / fl};
    // right = normalize(front x world_up), up = normalize(right x front)
    double r[3] = {f[1] * 0.0 - f[2] * 1.0, f[2] * 0.0 - f[0] * 0.0, f[0] * 1.0 - f[1] * 0.0};
    double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (double& v : r) v /= rl;
    double u[3] = {r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]};
    const double ul = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    for (double& v : u) v /= ul;
    // lookAt(eye, eye + front, up): s = normalize(front x up), u' = s x front
    double s[3] = {f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0]};
    const double sl = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (double& v : s) v /= sl;
    const double u2[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
    const double e[3] = {position[0], position[1], position[2]};
    float* V = out->view;
    for (int k = 0; k < 16; ++k) V[k] = 0.f;
    for (int k = 0; k < 3; ++k) {
        V[k * 4 + 0] = static_cast<float>(s[k]);
        V[k * 4 + 1] = static_cast<float>(u2[k]);
        V[k * 4 + 2] = static_cast<float>(-f[k]);
    }
    V[12] = static_cast<float>(-(s[0] * e[0] + s[1] * e[1] + s[2] * e[2]));
    V[13] = static_cast<float>(-(u2[0] * e[0] + u2[1] * e[1] + u2[2] * e[2]));
    V[14] = static_cast<float>(f[0] * e[0] + f[1] * e[1] + f[2] * e[2]);
    V[15] = 1.f;
    // perspective(fovy, aspect, near, far), clip z in [-w, w]
    const double fovy = 45.0 * 3.14159265358979323846 / 180.0, zn = 0.1, zf = 100.0;
    const double aspect = static_cast<double>(width) / static_cast<double>(height ? height : 1);
    const double th = std::tan(fovy / 2.0);
    float* P = out->projection;
    for (int k = 0; k < 16; ++k) P[k] = 0.f;
    P[0] = static_cast<float>(1.0 / (aspect * th));
    P[5] = static_cast<float>(1.0 / th);
    P[10] = static_cast<float>(-(zf + zn) / (zf - zn));
    P[11] = -1.f;
    P[14] = static_cast<float>(-(2.0 * zf * zn) / (zf - zn));
    out->eye[0] = position[0];
    out->eye[1] = position[1];
    out->eye[2] = position[2];
}

extern "C" void wcsph_default_render_opts(wcsph_render_opts* o) {
    if (!o) return;
    *o = wcsph_render_opts{};
    o->width = 640;
    o->height = 480;
    o->radius = 0.02f;   // instanced_ball.vert/.frag RADIUS
    o->show_boundary = 0;
    o->field = -1;
    o->normalize = 0;
    o->min_value = 0.f;
    o->max_value = 1.f;
    o->background[0] = o->background[1] = o->background[2] = 0.f;
    o->max_pixels = 1 << 16;
}
