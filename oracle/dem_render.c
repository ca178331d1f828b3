/* Test infrastructure (oracle only) -- never linked into the product.
 *
 * CPU restatement of the headless disk splat: the reference's plotSpheresD
 * (particles_kernel.cuh:629-718, launched by plotParticles, functions.cu:
 * 557-599) with the deterministic rule the library uses where the
 * reference's threads race: the highest particle index covering a pixel
 * colours it, and orientation lines are drawn after all disks.  Float
 * operations are the reference's (compile with -ffp-contract=off); float to
 * integer conversions saturate as CUDA's do (NaN -> 0); cos and sin of theta
 * are taken in double and rounded to float.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int32_t sat_i32(float v) {
    if (!(v == v)) return 0;
    if (v >= 2147483647.0f) return INT32_MAX;
    if (v <= -2147483648.0f) return INT32_MIN;
    return (int32_t)v;
}
static uint32_t sat_u32(float v) {
    if (!(v == v) || v <= 0.0f) return 0u;
    if (v >= 4294967295.0f) return UINT32_MAX;
    return (uint32_t)v;
}

/* particles_kernel.cuh:632-652 */
static float colorbar(float x) {
    const float top = 1.5f, bottom = -0.5f;
    float rv;
    if (x < 0.5f) rv = x / 0.5f * (top - bottom) + bottom;
    else rv = (x - 0.5f) / 0.5f * (bottom - top) + top;
    if (rv > 1.0f) return 255.0f;
    if (rv < 0.0f) return 0.0f;
    return rv * 255.0f;
}

static uint32_t pixel_of(uint32_t DIMx, uint32_t DIMy, int gx, int gy) {
    const uint32_t size = DIMx * DIMy;
    uint32_t pixel = (uint32_t)gx + (uint32_t)gy * DIMx;
    if (pixel >= size) pixel = size - 1u;
    return pixel;
}

/* image: 4 bytes per pixel (RGBA), DIMx * DIMy pixels; color: 3 floats per
 * material; type and pressure may be NULL. */
void orc_render(uint32_t DIMx, uint32_t DIMy, uint32_t bg, int viewRotations, int byPressure,
                float maxPressure, const float* color, float Lx, float Ly, const float* pos,
                const float* theta, const uint32_t* type, const float* radius,
                const float* pressure, uint32_t n, uint8_t* image) {
    const size_t pixels = (size_t)DIMx * DIMy;
    uint32_t* owner = (uint32_t*)calloc(pixels ? pixels : 1, sizeof(uint32_t));
    memset(image, (int)(bg & 0xffu), 4 * pixels);
    for (int pass = 0; pass < 2; ++pass) {
        for (uint32_t i = 0; i < n; ++i) {
            const float pR = (float)DIMy / Ly * radius[i];
            const int cx = sat_i32((float)DIMx / Lx * pos[2 * i]);
            const int cy = sat_i32((float)DIMy / Ly * pos[2 * i + 1]);
            const int h = sat_i32(ceilf(pR));
            const uint32_t t = type ? type[i] : 0u;
            float cr = color[3 * t], cg = color[3 * t + 1], cb = color[3 * t + 2];
            if (byPressure) {
                const float pr = (pressure ? pressure[i] : 0.0f) / maxPressure;
                cr = colorbar(pr - 0.25f);
                cg = colorbar(pr);
                cb = colorbar(pr + 0.25f);
            }
            const float r2 = pR * pR;
            for (int x = -h; x < h; ++x)
                for (int y = -h; y < h; ++y) {
                    if (!((float)(x * x + y * y) < r2)) continue;
                    const uint32_t p = pixel_of(DIMx, DIMy, cx + x, cy + y);
                    if (pass == 0) {
                        if (owner[p] < i + 1u) owner[p] = i + 1u;
                    } else if (owner[p] == i + 1u) {
                        const float f = sqrtf((r2 - (float)(x * x) - (float)(y * y)) / r2);
                        image[4 * p] = (uint8_t)(cr * f);
                        image[4 * p + 1] = (uint8_t)(cg * f);
                        image[4 * p + 2] = (uint8_t)(cb * f);
                        image[4 * p + 3] = (uint8_t)(255.0f * f);
                    }
                }
        }
    }
    if (viewRotations) {
        for (uint32_t i = 0; i < n; ++i) {
            const float pR = (float)DIMy / Ly * radius[i];
            const int cx = sat_i32((float)DIMx / Lx * pos[2 * i]);
            const int cy = sat_i32((float)DIMy / Ly * pos[2 * i + 1]);
            const float c = (float)cos((double)theta[i]), s = (float)sin((double)theta[i]);
            for (int r = 0; (float)r < pR; ++r) {
                const uint32_t gx = sat_u32((float)cx + (float)r * c);
                const uint32_t gy = sat_u32((float)cy + (float)r * s);
                uint32_t p = gx + gy * DIMx;
                if (p >= DIMx * DIMy) p = DIMx * DIMy - 1u;
                memset(image + 4 * (size_t)p, 0, 4);
            }
        }
    }
    free(owner);
}

/* One line of the reference's output.csv (writeOutputFile, functions.cu:
 * 608-661): "%f," with the elapsed time, then per followed particle
 * "%u,%u,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f" (id, type, x, y, vx, vy, ax, ay,
 * theta, omega, alpha, pressure) separated by commas, then a newline.  rows:
 * 12 words per particle as dem_get_followed returns them. */
#include <stdio.h>
size_t orc_followed_line(float elapsed, const float* rows, uint32_t count, char* buf,
                         size_t cap) {
    size_t k = (size_t)snprintf(buf, cap, "%f,", elapsed);
    for (uint32_t i = 0; i < count && k < cap; ++i) {
        const float* r = rows + 12 * (size_t)i;
        uint32_t id, type;
        memcpy(&id, r, 4);
        memcpy(&type, r + 1, 4);
        k += (size_t)snprintf(buf + k, cap - k, "%u,%u,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f", id, type,
                              r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10], r[11]);
        if (i != count - 1 && k < cap) k += (size_t)snprintf(buf + k, cap - k, ",");
    }
    if (k < cap) k += (size_t)snprintf(buf + k, cap - k, "\n");
    return k;
}
