// CPU check of the uv transport's closest-point projection: the library's
// barycentric (csrc/placement.cuh, the code the kernels run) against the
// oracle's restatement (bo_barycentric, bit for bit) and against the
// definition (no sample of the triangle is closer to p than the returned
// point, up to FP32 rounding of the inputs).
// Prints "barycentric <cases> <mismatches> <not-closest>"; exit 0 only
// without either.
#include "../blitzremesher_b200/csrc/placement.cuh"
#include "../oracle/blitz_oracle.h"

#include <cstdio>
#include <cstring>
#include <random>

using namespace b200;

static double dist2(float3 p, double x, double y, double z) {
    const double dx = double(p.x) - x, dy = double(p.y) - y, dz = double(p.z) - z;
    return dx * dx + dy * dy + dz * dz;
}

int main() {
    std::mt19937_64 rng(777);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    uint64_t cases = 0, mismatch = 0, not_closest = 0;
    for (int t = 0; t < 20000; ++t) {
        float3 a = make_float3(U(rng), U(rng), U(rng)), b = make_float3(U(rng), U(rng), U(rng)),
               c = make_float3(U(rng), U(rng), U(rng));
        if (t % 11 == 0) c = make_float3(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z)); // collinear
        if (t % 13 == 0) b = a;                                                                       // repeated corner
        const float s = t % 3 == 0 ? 3.f : 1.f;
        float3 p = make_float3(s * U(rng), s * U(rng), s * U(rng));
        if (t % 5 == 0) { // near the triangle's plane, inside or just outside
            const float u = 1.2f * (U(rng) + 1) / 2, v = (1 - u) * (U(rng) + 1) / 2;
            p = make_float3(a.x + u * (b.x - a.x) + v * (c.x - a.x), a.y + u * (b.y - a.y) + v * (c.y - a.y),
                            a.z + u * (b.z - a.z) + v * (c.z - a.z) + 1e-3f * U(rng));
        }
        const float3 w = barycentric(p, a, b, c);
        float pa[3] = {p.x, p.y, p.z}, aa[3] = {a.x, a.y, a.z}, ba[3] = {b.x, b.y, b.z}, ca[3] = {c.x, c.y, c.z}, wo[3];
        if (bo_barycentric(pa, aa, ba, ca, wo) != 0) return 2;
        ++cases;
        if (std::memcmp(&w.x, &wo[0], 4) || std::memcmp(&w.y, &wo[1], 4) || std::memcmp(&w.z, &wo[2], 4)) ++mismatch;
        // optimality on triangles that are not degenerate
        const double ex = double(b.x) - a.x, ey = double(b.y) - a.y, ez = double(b.z) - a.z;
        const double fx = double(c.x) - a.x, fy = double(c.y) - a.y, fz = double(c.z) - a.z;
        const double nx = ey * fz - ez * fy, ny = ez * fx - ex * fz, nz = ex * fy - ey * fx;
        const double area2 = nx * nx + ny * ny + nz * nz, scale = ex * ex + ey * ey + ez * ez + fx * fx + fy * fy + fz * fz;
        if (area2 < 1e-6 * scale * scale) continue;
        const double got = dist2(p, double(w.x) * a.x + double(w.y) * b.x + double(w.z) * c.x,
                                 double(w.x) * a.y + double(w.y) * b.y + double(w.z) * c.y,
                                 double(w.x) * a.z + double(w.y) * b.z + double(w.z) * c.z);
        double best = 1e300;
        const int n = 200;
        for (int i = 0; i <= n; ++i)
            for (int j = 0; i + j <= n; ++j) {
                const double u = double(i) / n, v = double(j) / n;
                best = std::min(best, dist2(p, a.x + u * ex + v * fx, a.y + u * ey + v * fy, a.z + u * ez + v * fz));
            }
        if (got > best + 1e-5 * (1 + best)) ++not_closest;
    }
    printf("barycentric %llu %llu %llu\n", (unsigned long long)cases, (unsigned long long)mismatch,
           (unsigned long long)not_closest);
    return mismatch || not_closest ? 1 : 0;
}
