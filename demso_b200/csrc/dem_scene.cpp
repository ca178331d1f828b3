// Host-side scene generation: seeded random sequential placement of disks.
//
// The reference creates its blocks with device kernels seeded from the wall
// clock (createRectanglesD with time(NULL), main.cu:291), which cannot be
// reproduced; scenes here are generated from explicit seeds on the host.
//
// Placement: disks are taken in order of decreasing radius and dealt round-
// robin to `strips` horizontal strips of equal height, which are filled
// independently (one OpenMP task each, with their own random stream, so the
// result does not depend on the thread count).  A disk stays inside its
// strip, so strips never overlap each other.  For each disk, uniform random
// trials come first; if all fail, random cells of the strip's bucket grid are
// probed on a jittered 5x5 lattice of candidate centres.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/demso_b200.h"

namespace {

struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Strip {
    double y0, y1, W, h;
    int gx, gy;
    std::vector<int> head, next;
    std::vector<double> px, py, pr;

    bool fits(double x, double y, double r) const {
        const int cx = (int)(x / h), cy = (int)((y - y0) / h);
        for (int yy = cy - 1; yy <= cy + 1; ++yy) {
            if (yy < 0 || yy >= gy) continue;
            for (int xx = cx - 1; xx <= cx + 1; ++xx) {
                if (xx < 0 || xx >= gx) continue;
                for (int j = head[(size_t)yy * gx + xx]; j >= 0; j = next[j]) {
                    const double dx = px[j] - x, dy = py[j] - y, d = r + pr[j];
                    if (dx * dx + dy * dy < d * d) return false;
                }
            }
        }
        return true;
    }
    void add(double x, double y, double r) {
        const int k = (int)px.size();
        px.push_back(x);
        py.push_back(y);
        pr.push_back(r);
        const int c = std::min((int)((y - y0) / h), gy - 1) * gx + std::min((int)(x / h), gx - 1);
        next.push_back(head[c]);
        head[c] = k;
    }
};

}  // namespace

extern "C" int dem_scene_rsa(uint32_t n, const float* radius, float Lx, float Ly, uint64_t seed,
                             uint32_t strips, uint32_t trials, float* pos, uint32_t* placed) {
    if (placed) *placed = 0;
    if (n == 0) return DEM_OK;
    if (!radius || !pos || !(Lx > 0.0f) || !(Ly > 0.0f) || strips == 0) return DEM_ERR_INVALID_ARG;
    double rmax = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!(radius[i] > 0.0f)) return DEM_ERR_INVALID_ARG;
        rmax = std::max(rmax, (double)radius[i]);
    }
    const double stripH = (double)Ly / strips;
    if (stripH < 2.0 * rmax || (double)Lx < 2.0 * rmax) return DEM_ERR_INVALID_ARG;
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [radius](uint32_t a, uint32_t b) { return radius[a] > radius[b]; });
    std::vector<uint32_t> placedPer(strips, 0);
    const double h = 2.0 * rmax;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long s = 0; s < (long long)strips; ++s) {
        Strip st;
        st.y0 = stripH * (double)s;
        st.y1 = st.y0 + stripH;
        st.W = Lx;
        st.h = h;
        st.gx = std::max(1, (int)std::ceil(Lx / h));
        st.gy = std::max(1, (int)std::ceil(stripH / h));
        st.head.assign((size_t)st.gx * st.gy, -1);
        SplitMix rng{seed * 0x100000001B3ull + (uint64_t)s * 0x9E3779B97F4A7C15ull + 1};
        uint32_t ok = 0;
        for (uint32_t k = (uint32_t)s; k < n; k += strips) {
            const uint32_t i = order[k];
            const double r = radius[i];
            bool done = false;
            double x = 0, y = 0;
            for (uint32_t a = 0; a < trials && !done; ++a) {
                x = r + rng.uniform() * (st.W - 2 * r);
                y = st.y0 + r + rng.uniform() * (stripH - 2 * r);
                done = st.fits(x, y, r);
            }
            for (int t = 0; t < 20000 && !done; ++t) {
                const uint64_t c = rng.next() % ((uint64_t)st.gx * st.gy);
                const int cx = (int)(c % st.gx), cy = (int)(c / st.gx);
                const double ox = rng.uniform(), oy = rng.uniform();
                for (int q = 0; q < 25 && !done; ++q) {
                    x = (cx + ((q % 5) + ox) / 5.0) * h;
                    y = st.y0 + (cy + ((q / 5) + oy) / 5.0) * h;
                    if (x < r || x > st.W - r || y < st.y0 + r || y > st.y1 - r) continue;
                    done = st.fits(x, y, r);
                }
            }
            if (!done) {
                pos[2 * i] = pos[2 * i + 1] = NAN;
                continue;
            }
            st.add(x, y, r);
            pos[2 * i] = (float)x;
            pos[2 * i + 1] = (float)y;
            ++ok;
        }
        placedPer[s] = ok;
    }
    uint32_t total = 0;
    for (uint32_t v : placedPer) total += v;
    if (placed) *placed = total;
    return total == n ? DEM_OK : DEM_ERR_CAPACITY;
}
