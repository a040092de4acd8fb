// gradients.cpp - dense gradient mip pyramid of a small terrain.
#include "gradients.h"

#include <cmath>
#include <stdexcept>

#include "terrain.h"

namespace vv {

void qt_normalize(float v[3]) {
    double len = (double)v[0] * (double)v[0] + (double)v[1] * (double)v[1] + (double)v[2] * (double)v[2];
    if (std::fabs(len - 1.0) <= 1e-12 || std::fabs(len) <= 1e-12) return;
    len = std::sqrt(len);
    v[0] = (float)((double)v[0] / len);
    v[1] = (float)((double)v[1] / len);
    v[2] = (float)((double)v[2] / len);
}

GradientPyramid::GradientPyramid(const TerrainVolume& v) {
    const int L = v.depth();
    if (L > 6) throw std::length_error("dense gradient pyramid: depth > 6");
    const int n0 = v.dim();
    lv_.resize(L + 1);
    dim_.resize(L + 1);
    // leaf level
    {
        dim_[0] = n0;
        std::vector<float>& g = lv_[0];
        g.assign((size_t)n0 * n0 * n0 * 3, 0.0f);
        auto alpha = [&](int x, int y, int z) -> float {
            return (float)(v.voxel(0, x, y, z) >> 24) / 255.0f;
        };
#pragma omp parallel for schedule(static)
        for (int z = 0; z < n0; ++z)
            for (int y = 0; y < n0; ++y)
                for (int x = 0; x < n0; ++x) {
                    const float s1x = x == 0 ? 0.0f : alpha(x - 1, y, z);
                    const float s2x = x == n0 - 1 ? 0.0f : alpha(x + 1, y, z);
                    const float s1y = y == 0 ? 0.0f : alpha(x, y - 1, z);
                    const float s2y = y == n0 - 1 ? 0.0f : alpha(x, y + 1, z);
                    const float s1z = z == 0 ? 0.0f : alpha(x, y, z - 1);
                    const float s2z = z == n0 - 1 ? 0.0f : alpha(x, y, z + 1);
                    double nx = (double)(s1x - s2x), ny = (double)(s1y - s2y), nz = (double)(s1z - s2z);
                    const double len = std::sqrt(nx * nx + ny * ny + nz * nz);
                    if (len > 0) {
                        nx /= len;
                        ny /= len;
                        nz /= len;
                    } else {
                        nx = ny = nz = 0.0;
                    }
                    float* o = &g[(((size_t)z * n0 + y) * n0 + x) * 3];
                    o[0] = (float)nx;
                    o[1] = (float)ny;
                    o[2] = (float)nz;
                }
    }
    // coarser levels
    for (int m = 1; m <= L; ++m) {
        const int nc = dim_[m - 1], n = nc / 2;
        dim_[m] = n;
        const std::vector<float>& f = lv_[m - 1];
        std::vector<float>& g = lv_[m];
        g.assign((size_t)n * n * n * 3, 0.0f);
        const float k = 1.0f / 8.0f;
#pragma omp parallel for schedule(static)
        for (int z = 0; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    float a[3] = {0.0f, 0.0f, 0.0f};
                    for (int zz = 2 * z; zz < 2 * z + 2; ++zz)
                        for (int yy = 2 * y; yy < 2 * y + 2; ++yy)
                            for (int xx = 2 * x; xx < 2 * x + 2; ++xx) {
                                const float* c = &f[(((size_t)zz * nc + yy) * nc + xx) * 3];
                                a[0] += c[0];
                                a[1] += c[1];
                                a[2] += c[2];
                            }
                    a[0] *= k;
                    a[1] *= k;
                    a[2] *= k;
                    qt_normalize(a);
                    float* o = &g[(((size_t)z * n + y) * n + x) * 3];
                    o[0] = a[0];
                    o[1] = a[1];
                    o[2] = a[2];
                }
    }
}

void GradientPyramid::at(int m, int x, int y, int z, float g[3]) const {
    const int n = dim_[m];
    if (x < 0 || y < 0 || z < 0 || x >= n || y >= n || z >= n) {
        g[0] = g[1] = g[2] = 0.0f;
        return;
    }
    const float* p = &lv_[m][(((size_t)z * n + y) * n + x) * 3];
    g[0] = p[0];
    g[1] = p[1];
    g[2] = p[2];
}

}  // namespace vv
