// Headless disk splat: the reference's particle image (plotParticles,
// functions.cu:557-599 -> plotSpheresD, particles_kernel.cuh:629-718) drawn
// into a caller's device uchar4 buffer instead of a GL pixel buffer.
//
// Per particle the pixels, shading and colours are the reference's, with the
// same float and integer operations: the centre pixel
// (int)(DIMx / Lx * x), (int)(DIMy / Ly * y); the square of half-side
// ceil(pRadius) with pRadius = DIMy / Ly * r; a pixel inside x^2 + y^2 <
// pRadius^2; the shade fscale = sqrtf((pR^2 - x^2 - y^2) / pR^2); the colour
// of the particle's type (or of its pressure / maxPressure on the
// reference's colour bar) times fscale, alpha 255 * fscale; pixel indices in
// unsigned arithmetic with the reference's clamp to the last pixel; the
// orientation line of black pixels along (cos theta, sin theta).
//
// Where the reference's threads race -- two particles covering one pixel, a
// line crossing another particle -- the result is made deterministic: the
// particle with the highest index among those covering a pixel colours it
// (an atomicMax pass, then a colouring pass), and orientation lines are drawn
// after every disk.  cos and sin of theta are evaluated in double and
// rounded to float.
#include <algorithm>

#include "../../include/demso_b200.h"
#include "dem_kernels.cuh"

namespace dem {
namespace {

constexpr int kRenderThreads = 256;

inline unsigned blocks_for(size_t n, int t) { return (unsigned)((n + (size_t)t - 1) / (size_t)t); }

// particles_kernel.cuh:632-652
__device__ __forceinline__ float colorbar(float x) {
    const float top = 1.5f, bottom = -0.5f;
    float rv;
    if (x < 0.5f) rv = x / 0.5f * (top - bottom) + bottom;
    else rv = (x - 0.5f) / 0.5f * (bottom - top) + top;
    if (rv > 1.0f) return 255.0f;
    if (rv < 0.0f) return 0.0f;
    return rv * 255.0f;
}

struct Splat {
    int cx, cy;
    float pR;
    int h;  // -h .. h-1 covers the square
};

__device__ __forceinline__ Splat splat_of(const DemRenderParams& rp, float Lx, float Ly, float2 p,
                                          float r) {
    Splat s;
    s.pR = (float)rp.imageDIMy / Ly * r;
    s.cx = (int)((float)rp.imageDIMx / Lx * p.x);
    s.cy = (int)((float)rp.imageDIMy / Ly * p.y);
    s.h = (int)ceilf(s.pR);
    return s;
}

__device__ __forceinline__ uint32_t pixel_of(const DemRenderParams& rp, int gx, int gy) {
    const uint32_t size = rp.imageDIMx * rp.imageDIMy;
    uint32_t pixel = (uint32_t)gx + (uint32_t)gy * rp.imageDIMx;
    if (pixel >= size) pixel = size - 1u;
    return pixel;
}

__global__ void fill_kernel(uint32_t* __restrict__ p, uint32_t value, size_t count) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = value;
}

// pass 1: the highest particle index (+1) covering each pixel
__global__ void __launch_bounds__(kRenderThreads)
owner_kernel(DemRenderParams rp, float Lx, float Ly, const float2* __restrict__ pos,
             const float* __restrict__ radius, uint32_t n, uint32_t* __restrict__ owner) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Splat s = splat_of(rp, Lx, Ly, pos[i], radius[i]);
    for (int x = -s.h; x < s.h; ++x)
        for (int y = -s.h; y < s.h; ++y)
            if ((float)(x * x + y * y) < s.pR * s.pR)
                atomicMax(owner + pixel_of(rp, s.cx + x, s.cy + y), i + 1u);
}

// pass 2: each particle colours the pixels it owns
__global__ void __launch_bounds__(kRenderThreads)
color_kernel(DemRenderParams rp, float Lx, float Ly, const float2* __restrict__ pos,
             const float* __restrict__ radius, const uint32_t* __restrict__ type,
             const float* __restrict__ pressure, uint32_t n, const uint32_t* __restrict__ owner,
             uchar4* __restrict__ image) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Splat s = splat_of(rp, Lx, Ly, pos[i], radius[i]);
    const uint32_t t = type ? type[i] : 0u;
    float cr = rp.color[t][0], cg = rp.color[t][1], cb = rp.color[t][2];
    if (rp.colorByPressure) {
        const float pr = (pressure ? pressure[i] : 0.0f) / rp.maxPressure;
        cr = colorbar(pr - 0.25f);
        cg = colorbar(pr);
        cb = colorbar(pr + 0.25f);
    }
    const float r2 = s.pR * s.pR;
    for (int x = -s.h; x < s.h; ++x)
        for (int y = -s.h; y < s.h; ++y) {
            if (!((float)(x * x + y * y) < r2)) continue;
            const uint32_t pixel = pixel_of(rp, s.cx + x, s.cy + y);
            if (owner[pixel] != i + 1u) continue;
            const float f = sqrtf((r2 - (float)(x * x) - (float)(y * y)) / r2);
            uchar4 c;
            c.x = (unsigned char)(cr * f);
            c.y = (unsigned char)(cg * f);
            c.z = (unsigned char)(cb * f);
            c.w = (unsigned char)(255.0f * f);
            image[pixel] = c;
        }
}

// pass 3: orientation lines (particles_kernel.cuh:697-716)
__global__ void __launch_bounds__(kRenderThreads)
line_kernel(DemRenderParams rp, float Lx, float Ly, const float2* __restrict__ pos,
            const float* __restrict__ radius, const float* __restrict__ theta, uint32_t n,
            uchar4* __restrict__ image) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Splat s = splat_of(rp, Lx, Ly, pos[i], radius[i]);
    const double th = (double)theta[i];
    const float c = (float)cos(th), sn = (float)sin(th);
    for (int r = 0; (float)r < s.pR; ++r) {
        // float -> unsigned conversions saturate (negative -> 0)
        const uint32_t gx = (uint32_t)((float)s.cx + (float)r * c);
        const uint32_t gy = (uint32_t)((float)s.cy + (float)r * sn);
        const uint32_t size = rp.imageDIMx * rp.imageDIMy;
        uint32_t pixel = gx + gy * rp.imageDIMx;
        if (pixel >= size) pixel = size - 1u;
        image[pixel] = make_uchar4(0, 0, 0, 0);
    }
}

}  // namespace

cudaError_t launch_render(const DemRenderParams& rp, float Lx, float Ly, const float2* pos,
                          const float* theta, const uint32_t* type, const float* radius,
                          const float* pressure, uint32_t n, uint32_t* owner, uchar4* image,
                          cudaStream_t st) {
    const size_t pixels = (size_t)rp.imageDIMx * rp.imageDIMy;
    const uint32_t bg = rp.bgColor & 0xffu;
    const unsigned fb = std::min<unsigned>(blocks_for(pixels, kRenderThreads), 148u * 16u);
    fill_kernel<<<fb, kRenderThreads, 0, st>>>(reinterpret_cast<uint32_t*>(image),
                                               bg | bg << 8 | bg << 16 | bg << 24, pixels);
    fill_kernel<<<fb, kRenderThreads, 0, st>>>(owner, 0u, pixels);
    if (n) {
        const unsigned b = blocks_for(n, kRenderThreads);
        owner_kernel<<<b, kRenderThreads, 0, st>>>(rp, Lx, Ly, pos, radius, n, owner);
        color_kernel<<<b, kRenderThreads, 0, st>>>(rp, Lx, Ly, pos, radius, type, pressure, n,
                                                   owner, image);
        if (rp.viewRotations)
            line_kernel<<<b, kRenderThreads, 0, st>>>(rp, Lx, Ly, pos, radius, theta, n, image);
    }
    return cudaGetLastError();
}

}  // namespace dem
