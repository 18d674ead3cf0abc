// Learned audit surrogate: per-candidate 1-ring features, a 48 -> 128 -> 128
// -> 2 MLP with BF16 weights and FP32 accumulation on the tcgen05 tensor
// cores (forward, and a fused forward + backward train step), Adam, and the
// top-k pruning of the executor's ranked edits.
//
// The network predicts, per candidate collapse, the logit of "accepted by the
// exact four-gate audit" and the ratio error / limit of the worst gate. It
// only orders and prunes: every collapse the executor commits is still judged
// by the exact audit.
#include "kernels.cuh"
#include "surrogate.cuh"
#include "tcgen05.cuh"

#include <cuda_bf16.h>

namespace b200 {

namespace {
constexpr int kThreads = 256;
inline uint32_t blocks_for(uint64_t n, int threads = kThreads) { return uint32_t((n + threads - 1) / threads); }

__device__ __forceinline__ float3 ld3(const float* p, uint32_t i) {
    return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 crs(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dt(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float nrm(float3 a) { return sqrtf(dt(a, a)); }

// Features of one legal edit, in pixels of the gate's screen (scale = screen /
// diameter): the collapse's `from` end and its ten nearest ring vertices
// relative to the midpoint placement, the ring size, the placement's quadric
// error over the faces around the edge, normal deviation and area change of
// the surviving faces, the edge length (linear, log, at the second screen),
// boundary and seam flags, removed faces, both valences and the ShortestEdge
// score.
__global__ void k_features(DevMesh m, DevTopology t, const Edit* edits, const uint32_t* count, float px,
                           float px2, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count) return;
    const Edit e = edits[i];
    float f[kSurrogateIn];
    for (int k = 0; k < kSurrogateIn; ++k) f[k] = 0;
    const float3 a = ld3(m.pos, e.from), b = ld3(m.pos, e.to);
    const float3 s = make_float3(a.x + b.x, a.y + b.y, a.z + b.z);
    const float3 mid = make_float3(float(double(s.x) * .5), float(double(s.y) * .5), float(double(s.z) * .5));
    const float3 ha = sub(a, mid);
    f[0] = ha.x * px, f[1] = ha.y * px, f[2] = ha.z * px;
    // ten nearest ring vertices (classes adjacent to from or to)
    float best_d[10];
    uint32_t best_v[10];
    int nb = 0;
    uint32_t ring = 0;
    for (int side = 0; side < 2; ++side) {
        const uint32_t u = side ? e.to : e.from;
        for (uint32_t k = t.nbr_offsets[u]; k < t.nbr_offsets[u + 1]; ++k) {
            const uint32_t v = t.neighbors[k];
            if (v == e.from || v == e.to) continue;
            if (side) { // skip neighbours of `to` already counted through `from`
                bool dup = false;
                for (uint32_t q = t.nbr_offsets[e.from]; q < t.nbr_offsets[e.from + 1]; ++q)
                    dup |= t.neighbors[q] == v;
                if (dup) continue;
            }
            ++ring;
            const float d = nrm(sub(ld3(m.pos, v), mid));
            int at = nb < 10 ? nb++ : 10;
            if (at == 10) {
                if (d >= best_d[9]) continue;
                at = 9;
            }
            while (at > 0 && best_d[at - 1] > d) {
                best_d[at] = best_d[at - 1], best_v[at] = best_v[at - 1];
                --at;
            }
            best_d[at] = d, best_v[at] = v;
        }
    }
    for (int k = 0; k < nb; ++k) {
        const float3 r = sub(ld3(m.pos, best_v[k]), mid);
        f[3 + 3 * k] = r.x * px, f[4 + 3 * k] = r.y * px, f[5 + 3 * k] = r.z * px;
    }
    f[33] = float(ring);
    // faces around the edge: quadric error, normal deviation, area change
    float quadric = 0, max_dev = 0, sum_dev = 0, area_before = 0, area_after = 0, min_ratio = 1;
    uint32_t faces = 0;
    for (int side = 0; side < 2; ++side) {
        const uint32_t u = side ? e.to : e.from;
        for (uint32_t k = t.face_offsets[u]; k < t.face_offsets[u + 1]; ++k) {
            const uint32_t face = t.faces[k];
            uint32_t c[3], g[3];
            bool has_from = false, has_to = false;
            for (int j = 0; j < 3; ++j) {
                c[j] = m.idx[3 * face + j];
                g[j] = t.geometry[c[j]];
                has_from |= g[j] == e.from;
                has_to |= g[j] == e.to;
            }
            if (side && has_from) continue; // counted through `from`
            const float3 p0 = ld3(m.pos, c[0]), p1 = ld3(m.pos, c[1]), p2 = ld3(m.pos, c[2]);
            const float3 n0 = crs(sub(p1, p0), sub(p2, p0));
            const float len0 = nrm(n0);
            area_before += 0.5f * len0 * px * px;
            if (len0 > 0) {
                const float h = dt(n0, sub(mid, p0)) / len0 * px;
                quadric += h * h;
            }
            ++faces;
            if (has_from && has_to) continue; // removed by the collapse
            float3 q[3] = {p0, p1, p2};
            for (int j = 0; j < 3; ++j)
                if (g[j] == e.from || g[j] == e.to) q[j] = mid;
            const float3 n1 = crs(sub(q[1], q[0]), sub(q[2], q[0]));
            const float len1 = nrm(n1);
            area_after += 0.5f * len1 * px * px;
            const float cosv = len0 > 0 && len1 > 0 ? dt(n0, n1) / (len0 * len1) : -1.f;
            const float dev = 1.f - cosv;
            max_dev = fmaxf(max_dev, dev);
            sum_dev += dev;
            if (len0 > 0) min_ratio = fminf(min_ratio, len1 / len0);
        }
    }
    const float len = nrm(sub(b, a));
    f[34] = quadric;
    f[35] = max_dev;
    f[36] = min_ratio;
    f[37] = len * px;
    f[38] = log2f(1.f + len * px);
    f[39] = len * px2;
    f[40] = float(t.boundary[e.from] | t.boundary[e.to]);
    f[41] = float(e.wedges > 1);
    f[42] = float(e.removed);
    f[43] = float(t.nbr_offsets[e.from + 1] - t.nbr_offsets[e.from]);
    f[44] = float(t.nbr_offsets[e.to + 1] - t.nbr_offsets[e.to]);
    f[45] = area_before;
    f[46] = area_after;
    f[47] = faces ? sum_dev / float(faces) : 0.f;
    float* o = out + size_t(i) * kSurrogateIn;
    for (int k = 0; k < kSurrogateIn; ++k) o[k] = f[k];
}

// ---------------------------------------------------------------------------
// MLP on the tensor cores. One CTA of 128 threads owns 128 candidate rows at a
// time (thread t = row t = TMEM lane t) and loops over row tiles. All operand
// tiles live in shared memory in the K-major no-swizzle layout; the backward
// GEMMs read the same tiles through MN-major descriptors (transposes for free).
constexpr uint32_t kRows = 128;
constexpr uint32_t kSX = 0;                    // X   128 x 64
constexpr uint32_t kSW1 = kSX + 16384;         // W1  128 x 64
constexpr uint32_t kSW2 = kSW1 + 16384;        // W2  128 x 128
constexpr uint32_t kSW3 = kSW2 + 32768;        // W3   16 x 128
constexpr uint32_t kSH1 = kSW3 + 4096;         // H1  128 x 128
constexpr uint32_t kSH2 = kSH1 + 32768;        // H2  128 x 128
constexpr uint32_t kSG = kSH2 + 32768;         // G2 / G1 128 x 128 (train)
constexpr uint32_t kSG3 = kSG + 32768;         // G3  128 x 16 (train)
constexpr uint32_t kSVec = kSG3 + 4096;        // b1, b2, b3, mean, inv_std, g0, g1 (floats)
constexpr uint32_t kVecFloats = 128 + 128 + 16 + 48 + 48 + 128 + 128;
constexpr uint32_t kSmemTrain = kSVec + kVecFloats * 4;
// TMEM columns
constexpr uint32_t kColD1 = 0, kColD2 = 128, kColDW2 = 256, kColDW1 = 384, kColD3 = 448, kTmemCols = 512;
constexpr uint32_t kWaitLimit = 1u << 24;

struct MlpArgs {
    const float* features; // n x 48
    uint32_t n;
    const __nv_bfloat16 *w1, *w2, *w3; // 128x64, 128x128, 16x128 row-major
    const float *b1, *b2, *b3, *mean, *inv_std;
    float* out;          // n x 2
    const float* labels; // n x 2 (train)
    float grad_scale;
    float *gw1, *gw2, *gw3, *gb1, *gb2, *gb3, *loss;
    uint32_t* error;
};

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }
__device__ __forceinline__ float round_bf16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Row-major BF16 [rows x kext] weights -> K-major shared tile.
__device__ void load_weights(uint8_t* smem, uint32_t base, const __nv_bfloat16* w, uint32_t rows, uint32_t kext) {
    const uint32_t chunks = rows * (kext / 8);
    for (uint32_t c = threadIdx.x; c < chunks; c += blockDim.x) {
        const uint32_t r = c / (kext / 8), k = (c % (kext / 8)) * 8;
        const uint4 v = *reinterpret_cast<const uint4*>(w + size_t(r) * kext + k);
        *reinterpret_cast<uint4*>(smem + base + tc::kmajor_offset(r, k, kext)) = v;
    }
}

// Reads 128 TMEM columns of this thread's lane from `col`, applies
// f(column, value) and stores the BF16 results as row `row` of a K-major
// 128-wide tile.
template <class F>
__device__ __forceinline__ void epilogue_row(uint32_t tmem, uint32_t col, uint8_t* tile, uint32_t row, F f) {
    for (uint32_t c = 0; c < 128; c += 8) {
        float v[8];
        tc::tmem_ld8(tmem + col + c, v);
        uint4 packed;
        packed.x = pack_bf16(f(c + 0, v[0]), f(c + 1, v[1]));
        packed.y = pack_bf16(f(c + 2, v[2]), f(c + 3, v[3]));
        packed.z = pack_bf16(f(c + 4, v[4]), f(c + 5, v[5]));
        packed.w = pack_bf16(f(c + 6, v[6]), f(c + 7, v[7]));
        *reinterpret_cast<uint4*>(tile + tc::kmajor_offset(row, c, 128)) = packed;
    }
}
__device__ __forceinline__ bool relu_on(const uint8_t* tile, uint32_t row, uint32_t c) {
    const uint16_t h = *reinterpret_cast<const uint16_t*>(tile + tc::kmajor_offset(row, c, 128));
    return (h & 0x8000u) == 0 && (h & 0x7fffu) != 0;
}
__device__ __forceinline__ float tile_value(const uint8_t* tile, uint32_t row, uint32_t c, uint32_t kext) {
    const uint16_t h = *reinterpret_cast<const uint16_t*>(tile + tc::kmajor_offset(row, c, kext));
    return __uint_as_float(uint32_t(h) << 16);
}

// Shared-memory operands written by threads become visible to the tensor
// core, and TMEM reads of the previous stage are ordered before the next MMA.
__device__ __forceinline__ void handoff_to_mma() {
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
}

template <bool kTrain>
__global__ void __launch_bounds__(128, 1) k_mlp(MlpArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base_s;
    float* vec = reinterpret_cast<float*>(smem + kSVec);
    float *sb1 = vec, *sb2 = vec + 128, *sb3 = vec + 256, *smean = vec + 272, *sinv = vec + 320;
    float *sg0 = vec + 368, *sg1 = vec + 496;
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const uint32_t tiles = (a.n + kRows - 1) / kRows;
    if (blockIdx.x >= tiles) return;
    if (warp == 0) tc::tmem_alloc(&tmem_base_s, kTmemCols);
    if (t == 0) tc::mbar_init(&mbar, 1);
    load_weights(smem, kSW1, a.w1, 128, 64);
    load_weights(smem, kSW2, a.w2, 128, 128);
    load_weights(smem, kSW3, a.w3, 16, 128);
    for (uint32_t i = t; i < 128; i += blockDim.x) sb1[i] = a.b1[i], sb2[i] = a.b2[i];
    if (t < 16) sb3[t] = a.b3[t];
    if (t < kSurrogateIn) smean[t] = a.mean[t], sinv[t] = a.inv_std[t];
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tmem_base_s + ((warp * 32u) << 16);
    const uint32_t tmem0 = tmem_base_s;
    const uint32_t sbase = tc::smem_addr(smem);
    uint32_t phase = 0;
    bool failed = false;
    // accumulators of the train step
    float acc_w3_0 = 0, acc_w3_1 = 0, acc_b1 = 0, acc_b2 = 0, acc_b3_0 = 0, acc_b3_1 = 0, acc_loss = 0;
    bool first_tile = true;
    auto wait_mma = [&]() -> bool {
        const bool ok = tc::mbar_wait(&mbar, phase, kWaitLimit);
        phase ^= 1;
        tc::fence_after();
        return !__syncthreads_or(!ok);
    };
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t row = tile * kRows + t;
        const bool live = row < a.n;
        // X: normalised features, BF16, K padded to 64.
        {
            float x[64];
            for (int k = 0; k < 64; ++k) x[k] = 0;
            if (live) {
                const float4* src = reinterpret_cast<const float4*>(a.features + size_t(row) * kSurrogateIn);
                for (int q = 0; q < kSurrogateIn / 4; ++q) {
                    const float4 v = src[q];
                    x[4 * q] = (v.x - smean[4 * q]) * sinv[4 * q];
                    x[4 * q + 1] = (v.y - smean[4 * q + 1]) * sinv[4 * q + 1];
                    x[4 * q + 2] = (v.z - smean[4 * q + 2]) * sinv[4 * q + 2];
                    x[4 * q + 3] = (v.w - smean[4 * q + 3]) * sinv[4 * q + 3];
                }
            }
            for (int c = 0; c < 64; c += 8) {
                uint4 p;
                p.x = pack_bf16(x[c], x[c + 1]), p.y = pack_bf16(x[c + 2], x[c + 3]);
                p.z = pack_bf16(x[c + 4], x[c + 5]), p.w = pack_bf16(x[c + 6], x[c + 7]);
                *reinterpret_cast<uint4*>(smem + kSX + tc::kmajor_offset(t, c, 64)) = p;
            }
        }
        // Layer 1: D1 = X W1^T (M 128, N 128, K 64)
        handoff_to_mma();
        if (t == 0) {
            tc::fence_after();
            constexpr uint32_t id = tc::idesc_bf16(128, 128, false, false);
            for (uint32_t k = 0; k < 4; ++k)
                tc::mma_bf16(tmem0 + kColD1, tc::desc(sbase + kSX + k * 256, 128, 1024),
                             tc::desc(sbase + kSW1 + k * 256, 128, 1024), id, k > 0);
            tc::commit(&mbar);
        }
        if (!wait_mma()) { failed = true; break; }
        epilogue_row(tmem, kColD1, smem + kSH1, t, [&](uint32_t c, float v) { return fmaxf(v + sb1[c], 0.f); });
        // Layer 2: D2 = H1 W2^T (K 128)
        handoff_to_mma();
        if (t == 0) {
            tc::fence_after();
            constexpr uint32_t id = tc::idesc_bf16(128, 128, false, false);
            for (uint32_t k = 0; k < 8; ++k)
                tc::mma_bf16(tmem0 + kColD2, tc::desc(sbase + kSH1 + k * 256, 128, 2048),
                             tc::desc(sbase + kSW2 + k * 256, 128, 2048), id, k > 0);
            tc::commit(&mbar);
        }
        if (!wait_mma()) { failed = true; break; }
        epilogue_row(tmem, kColD2, smem + kSH2, t, [&](uint32_t c, float v) { return fmaxf(v + sb2[c], 0.f); });
        // Layer 3: D3 = H2 W3^T (N 16)
        handoff_to_mma();
        if (t == 0) {
            tc::fence_after();
            constexpr uint32_t id = tc::idesc_bf16(128, 16, false, false);
            for (uint32_t k = 0; k < 8; ++k)
                tc::mma_bf16(tmem0 + kColD3, tc::desc(sbase + kSH2 + k * 256, 128, 2048),
                             tc::desc(sbase + kSW3 + k * 256, 128, 2048), id, k > 0);
            tc::commit(&mbar);
        }
        if (!wait_mma()) { failed = true; break; }
        float o[8];
        tc::tmem_ld8(tmem + kColD3, o);
        const float o0 = o[0] + sb3[0], o1 = o[1] + sb3[1];
        if (!kTrain) {
            if (live) a.out[2 * size_t(row)] = o0, a.out[2 * size_t(row) + 1] = o1;
            continue;
        }
        // ---- backward ----
        float g0 = 0, g1 = 0;
        if (live) {
            const float y = a.labels[2 * size_t(row)], target = a.labels[2 * size_t(row) + 1];
            const float sig = 1.f / (1.f + expf(-o0));
            const float d = o1 - target;
            const float ad = fabsf(d);
            acc_loss += (fmaxf(o0, 0.f) + log1pf(expf(-fabsf(o0))) - y * o0) + (ad <= 1.f ? 0.5f * d * d : ad - 0.5f);
            g0 = (sig - y) * a.grad_scale;
            g1 = fminf(fmaxf(d, -1.f), 1.f) * a.grad_scale;
            if (a.out) a.out[2 * size_t(row)] = o0, a.out[2 * size_t(row) + 1] = o1;
        }
        g0 = round_bf16(g0), g1 = round_bf16(g1);
        sg0[t] = g0, sg1[t] = g1;
        acc_b3_0 += g0, acc_b3_1 += g1;
        {
            uint4 p0, p1;
            p0.x = pack_bf16(g0, g1), p0.y = p0.z = p0.w = 0;
            p1.x = p1.y = p1.z = p1.w = 0;
            *reinterpret_cast<uint4*>(smem + kSG3 + tc::kmajor_offset(t, 0, 16)) = p0;
            *reinterpret_cast<uint4*>(smem + kSG3 + tc::kmajor_offset(t, 8, 16)) = p1;
        }
        // dH2 = G3 W3 (A K-major 128x16; B = W3 read MN-major: N 128, K 16)
        handoff_to_mma();
        if (t == 0) {
            tc::fence_after();
            constexpr uint32_t id = tc::idesc_bf16(128, 128, false, true);
            tc::mma_bf16(tmem0 + kColD1, tc::desc(sbase + kSG3, 128, 256), tc::desc(sbase + kSW3, 2048, 128), id, 0);
            tc::commit(&mbar);
        }
        // dW3 on the CUDA cores while the tensor core runs: thread t owns column t.
        for (uint32_t r = 0; r < kRows; ++r) {
            const float h = tile_value(smem + kSH2, r, t, 128);
            acc_w3_0 += sg0[r] * h;
            acc_w3_1 += sg1[r] * h;
        }
        if (!wait_mma()) { failed = true; break; }
        epilogue_row(tmem, kColD1, smem + kSG, t,
                     [&](uint32_t c, float v) { return relu_on(smem + kSH2, t, c) ? v : 0.f; });
        // dH1 = G2 W2 (B = W2 MN-major) and dW2 += G2^T H1 (both MN-major)
        handoff_to_mma();
        if (t == 0) {
            tc::fence_after();
            constexpr uint32_t id_h = tc::idesc_bf16(128, 128, false, true);
            constexpr uint32_t id_w = tc::idesc_bf16(128, 128, true, true);
            for (uint32_t k = 0; k < 8; ++k)
                tc::mma_bf16(tmem0 + kColD2, tc::desc(sbase + kSG + k * 256, 128, 2048),
                             tc::desc(sbase + kSW2 + k * 4096, 2048, 128), id_h, k > 0);
            for (uint32_t k = 0; k < 8; ++k)
                tc::mma_bf16(tmem0 + kColDW2, tc::desc(sbase + kSG + k * 4096, 2048, 128),
                             tc::desc(sbase + kSH1 + k * 4096, 2048, 128), id_w, !(first_tile && k == 0));
            tc::commit(&mbar);
        }
        for (uint32_t r = 0; r < kRows; ++r) acc_b2 += tile_value(smem + kSG, r, t, 128);
        if (!wait_mma()) { failed = true; break; }
        epilogue_row(tmem, kColD2, smem + kSG, t,
                     [&](uint32_t c, float v) { return relu_on(smem + kSH1, t, c) ? v : 0.f; });
        // dW1 += G1^T X (A MN-major 128 x K rows, B = X MN-major N 64)
        handoff_to_mma();
        if (t == 0) {
            tc::fence_after();
            constexpr uint32_t id = tc::idesc_bf16(128, 64, true, true);
            for (uint32_t k = 0; k < 8; ++k)
                tc::mma_bf16(tmem0 + kColDW1, tc::desc(sbase + kSG + k * 4096, 2048, 128),
                             tc::desc(sbase + kSX + k * 2048, 1024, 128), id, !(first_tile && k == 0));
            tc::commit(&mbar);
        }
        for (uint32_t r = 0; r < kRows; ++r) acc_b1 += tile_value(smem + kSG, r, t, 128);
        if (!wait_mma()) { failed = true; break; }
        first_tile = false;
    }
    if (kTrain && !failed && !first_tile) {
        // Weight gradients accumulated in TMEM over this CTA's tiles: lane t = output t.
        for (uint32_t c = 0; c < 128; c += 8) {
            float v[8];
            tc::tmem_ld8(tmem + kColDW2 + c, v);
            for (int j = 0; j < 8; ++j) atomicAdd(a.gw2 + size_t(t) * 128 + c + j, v[j]);
        }
        for (uint32_t c = 0; c < 64; c += 8) {
            float v[8];
            tc::tmem_ld8(tmem + kColDW1 + c, v);
            for (int j = 0; j < 8; ++j) atomicAdd(a.gw1 + size_t(t) * 64 + c + j, v[j]);
        }
        atomicAdd(a.gw3 + t, acc_w3_0);
        atomicAdd(a.gw3 + 128 + t, acc_w3_1);
        atomicAdd(a.gb1 + t, acc_b1);
        atomicAdd(a.gb2 + t, acc_b2);
        for (int s = 16; s; s >>= 1) {
            acc_b3_0 += __shfl_xor_sync(0xffffffffu, acc_b3_0, s);
            acc_b3_1 += __shfl_xor_sync(0xffffffffu, acc_b3_1, s);
            acc_loss += __shfl_xor_sync(0xffffffffu, acc_loss, s);
        }
        if ((t & 31) == 0) {
            atomicAdd(a.gb3, acc_b3_0);
            atomicAdd(a.gb3 + 1, acc_b3_1);
            atomicAdd(a.loss, acc_loss);
        }
    }
    if (failed && t == 0) atomicExch(a.error, 1u);
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem_base_s, kTmemCols);
}

// Adam on the FP32 master weights; refreshes the BF16 copies and clears the
// gradient accumulators. `mask` zeroes the padded parameters.
__global__ void k_adam(float* w, float* g, float* m, float* v, __nv_bfloat16* wb, uint32_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2, const uint8_t* mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float grad = g[i];
    g[i] = 0;
    if (mask && !mask[i]) {
        w[i] = 0;
        if (wb) wb[i] = __float2bfloat16_rn(0.f);
        return;
    }
    const float mi = b1 * m[i] + (1 - b1) * grad;
    const float vi = b2 * v[i] + (1 - b2) * grad * grad;
    m[i] = mi, v[i] = vi;
    const float step = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    const float wi = w[i] - step;
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
}

// keep[i] = 1 for the `keep` highest-scored edits (by the sorted order).
__global__ void k_mark_top(const uint32_t* sorted_idx, uint32_t n, uint32_t keep, uint32_t* flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[sorted_idx[i]] = i < keep;
}
// ranked position p -> flag of the edit ranked there
__global__ void k_rank_flags(const uint32_t* order, uint32_t n, const uint32_t* flags, uint32_t* rank_flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rank_flags[i] = flags[order[i]];
    if (i == n) rank_flags[i] = 0;
}
__global__ void k_compact_order(const uint32_t* order, const uint32_t* rank_flags, const uint32_t* offsets,
                                uint32_t n, uint32_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && rank_flags[i]) out[offsets[i]] = order[i];
}
// pass probability as the pruning key
__global__ void k_pass_logits(const float* out, uint32_t n, float* keys, uint32_t* idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = out[2 * size_t(i)];
    idx[i] = i;
}
} // namespace

size_t mlp_smem_bytes() { return kSmemTrain; }

cudaError_t launch_mlp(const SurrogateDev& w, const float* features, uint32_t n, float* out, const float* labels,
                       float grad_scale, float* loss, uint32_t* error, uint32_t max_ctas, cudaStream_t s) {
    if (!n) return cudaSuccess;
    MlpArgs a{};
    a.features = features, a.n = n;
    a.w1 = w.w1b, a.w2 = w.w2b, a.w3 = w.w3b;
    a.b1 = w.b1, a.b2 = w.b2, a.b3 = w.b3, a.mean = w.mean, a.inv_std = w.inv_std;
    a.out = out, a.labels = labels, a.grad_scale = grad_scale;
    a.gw1 = w.gw1, a.gw2 = w.gw2, a.gw3 = w.gw3, a.gb1 = w.gb1, a.gb2 = w.gb2, a.gb3 = w.gb3, a.loss = loss;
    a.error = error;
    const uint32_t tiles = (n + kRows - 1) / kRows;
    const uint32_t grid = tiles < max_ctas ? tiles : max_ctas;
    const size_t smem = mlp_smem_bytes();
    cudaError_t err;
    if (labels) {
        err = cudaFuncSetAttribute(k_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (err != cudaSuccess) return err;
        k_mlp<true><<<grid, 128, smem, s>>>(a);
    } else {
        err = cudaFuncSetAttribute(k_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (err != cudaSuccess) return err;
        k_mlp<false><<<grid, 128, smem, s>>>(a);
    }
    return cudaGetLastError();
}

void launch_adam(float* w, float* g, float* m, float* v, __nv_bfloat16* wb, uint32_t n, float lr, float b1, float b2,
                 float eps, uint32_t step, const uint8_t* mask, cudaStream_t s) {
    const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
    k_adam<<<blocks_for(n), kThreads, 0, s>>>(w, g, m, v, wb, n, lr, b1, b2, eps, c1, c2, mask);
}

void launch_features(const DevMesh& m, const DevTopology& t, const Edit* edits, const uint32_t* count,
                     uint32_t capacity, float px, float px2, float* out, cudaStream_t s) {
    if (!capacity) return;
    k_features<<<blocks_for(capacity, 128), 128, 0, s>>>(m, t, edits, count, px, px2, out);
}

void launch_prune_prepare(const float* out, uint32_t n, float* keys, uint32_t* idx, cudaStream_t s) {
    if (n) k_pass_logits<<<blocks_for(n), kThreads, 0, s>>>(out, n, keys, idx);
}
void launch_prune_order(const uint32_t* sorted_idx, uint32_t n, uint32_t keep, uint32_t* flags,
                        const uint32_t* order, uint32_t* rank_flags, uint32_t* offsets, uint32_t* scan_scratch,
                        uint32_t* out, cudaStream_t s) {
    if (!n) return;
    k_mark_top<<<blocks_for(n), kThreads, 0, s>>>(sorted_idx, n, keep, flags);
    k_rank_flags<<<blocks_for(n + 1), kThreads, 0, s>>>(order, n, flags, rank_flags);
    launch_exclusive_scan(rank_flags, offsets, n + 1, scan_scratch, s);
    k_compact_order<<<blocks_for(n), kThreads, 0, s>>>(order, rank_flags, offsets, n, out);
}

} // namespace b200
