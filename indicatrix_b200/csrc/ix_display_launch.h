// ix_display_launch.h -- launch records of the display kernels (ix_display.cu) shared with
// the host entry points (ix_display_host.cpp).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ix_display.h"
#include "../../include/ix_scene.h"

namespace ix {
namespace disp {

// Guide pass: one un-jittered camera ray per pixel.  Every output pointer may be null.
struct GuideLaunch {
    ix_camera camera;
    uint32_t width, height;
    const float4* planes;  // device, n_planes x {nx, ny, nz, d}
    uint32_t n_planes;
    float n_d;             // > 1: path signature at this index
    // The reference's GuideBuffers layout (row-major, normal as 3 floats).
    float* depth;
    float* normal;
    int32_t* facet;
    uint32_t* sig;
    // The A-Trous passes' packed guides: unit normal (w: sanitised depth), (facet, sig).
    float4* nrm;
    int2* fs;
};

// Guides given in the reference layout (depth non-null) -> the packed form, or already
// packed by the guide pass (depth null: nrm is read for the depth); colour (3 floats per
// pixel) times `scale` -> float4 {x, y, z, sanitised depth} when color_out is non-null.
struct PackLaunch {
    uint64_t pixels;
    const float* depth;
    const float* normal;
    const int32_t* facet;
    const uint32_t* sig;   // null: no signature (0 everywhere)
    float4* nrm;
    int2* fs;
    const float* color;    // 3 floats per pixel
    float scale;
    float4* color_out;
};

// One A-Trous pass at dilation `stride`.
struct PassLaunch {
    uint32_t width, height;
    int stride;
    const float4* src;     // {x, y, z, sanitised depth}
    const float4* nrm;     // unit normal
    const int2* fs;
    int facet_normals;     // the normal is a function of the facet id (guide-pass guides)
    float neg_inv_sigma_depth;
    float neg_inv_two_sigma_color_sq;
    float normal_power;    // max(power, 0)
    int squarings;         // >= 0: power = 2^squarings by repeated squaring; -1: pow
    float4* dst;           // colour out (or null)
    uchar4* rgba;          // sRGB RGBA8 out (or null): the tone-map fused into the pass
};

// Tone-map: XYZ (3 floats or float4 per pixel) times `scale` -> RGBA8 in `space`.
struct TonemapLaunch {
    uint64_t pixels;
    const float* xyz3;     // 3 floats per pixel, or null
    const float4* xyz4;    // float4 per pixel when xyz3 is null
    float scale;
    uint32_t space;
    uchar4* rgba;
};

// float4 -> 3 floats per pixel (the reference's Vec3 buffer layout).
struct UnpackLaunch {
    uint64_t pixels;
    const float4* src;
    float* dst;
};

// The guide pass and the packing are geometry and bookkeeping: exact build only.
cudaError_t launch_guides_exact(const GuideLaunch& L, cudaStream_t s);
cudaError_t launch_pack_exact(const PackLaunch& L, cudaStream_t s);
cudaError_t launch_atrous_pass_exact(const PassLaunch& L, cudaStream_t s);
cudaError_t launch_atrous_pass_fast(const PassLaunch& L, cudaStream_t s);
cudaError_t launch_tonemap_exact(const TonemapLaunch& L, cudaStream_t s);
cudaError_t launch_tonemap_fast(const TonemapLaunch& L, cudaStream_t s);
cudaError_t launch_unpack_exact(const UnpackLaunch& L, cudaStream_t s);
cudaError_t launch_unpack_fast(const UnpackLaunch& L, cudaStream_t s);

}  // namespace disp
}  // namespace ix
