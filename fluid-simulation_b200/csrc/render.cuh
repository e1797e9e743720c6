// render.cuh — headless impostor-sphere rendering (see render.cu).
#pragma once
#include "../../include/wcsph.h"
#include "sph_common.cuh"

namespace wcsph {

enum RenderMode : int { RENDER_PLAIN = 0, RENDER_SCALAR = 1, RENDER_VECTOR = 2 };

struct RenderArgs {
    float proj[16], view[16], vp[16], inv_vp[16];   // column-major; vp = proj * view
    float eye[3];
    u32 width, height;
    float radius;
    int show_boundary;
    int mode;               // RenderMode (fluid particles only)
    int normalize;
    float min_value, max_value;
    float background[3];
    int max_pixels;         // per-particle pixel box limit (quads larger than this are skipped)
};

// Clears the depth buffer, splats the particles and resolves RGBA8 (+ depth)
// on `stream`. zbuf, rgba and depth (optional) hold width * height entries.
void enqueue_render(const RenderArgs& r, const float4* fluid, u32 nf, const float4* boundary, u32 nb,
                    const float* scalar, const float4* vec, unsigned long long* zbuf, u32* rgba, float* depth,
                    cudaStream_t stream);

void mat4_mul(const float* a, const float* b, float* out);   // out = a * b (column-major)
bool mat4_inverse(const float* m, float* out);

}  // namespace wcsph
