// Closest-point placement math of the uv transport (place_vertices,
// action_gpu.cu:919-1067): host and device, so the CPU tests check the same
// code the kernels run against the oracle and against brute force.
#pragma once
#include <vector_functions.h>
#include <vector_types.h>

#include "common.cuh"

namespace b200 {

BH float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
BH double dotd(float3 a, float3 b) {
    return double(a.x) * double(b.x) + double(a.y) * double(b.y) + double(a.z) * double(b.z);
}
// Closest point of triangle (a, b, c) to p as barycentric weights
// (action_gpu.cu:919-952): Voronoi regions of the vertices and edges, then
// the interior.
BH float3 barycentric(float3 p, float3 a, float3 b, float3 c) {
    const float3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
    const double d1 = dotd(ab, ap), d2 = dotd(ac, ap);
    if (d1 <= 0 && d2 <= 0) return make_float3(1, 0, 0);
    const float3 bp = sub3(p, b);
    const double d3 = dotd(ab, bp), d4 = dotd(ac, bp);
    if (d3 >= 0 && d4 <= d3) return make_float3(0, 1, 0);
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const double v = d1 / (d1 - d3);
        return make_float3(float(1 - v), float(v), 0);
    }
    const float3 cp = sub3(p, c);
    const double d5 = dotd(ab, cp), d6 = dotd(ac, cp);
    if (d6 >= 0 && d5 <= d6) return make_float3(0, 0, 1);
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const double w = d2 / (d2 - d6);
        return make_float3(float(1 - w), 0, float(w));
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        return make_float3(0, float(1 - w), float(w));
    }
    const double sum = va + vb + vc;
    if (std::fabs(sum) < 1e-30) return make_float3(1, 0, 0);
    const double v = vb / sum, w = vc / sum;
    return make_float3(float(1 - v - w), float(v), float(w));
}
BH float3 scale3(float3 a, double s) {
    return make_float3(float(a.x * s), float(a.y * s), float(a.z * s));
}
// blend3 (action_gpu.cu:953-955)
BH float3 blend3(float3 a, float3 b, float3 c, float3 w) {
    const float3 x = scale3(a, w.x), y = scale3(b, w.y), z = scale3(c, w.z);
    return make_float3(x.x + y.x + z.x, x.y + y.y + z.y, x.z + y.z + z.z);
}

} // namespace b200
