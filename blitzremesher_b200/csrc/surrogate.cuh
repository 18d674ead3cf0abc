// Learned audit surrogate: device parameter set and launchers.
#pragma once
#include "kernels.cuh"
#include <cuda_bf16.h>

namespace b200 {

constexpr int kSurrogateIn = 48;     // features per candidate
constexpr int kSurrogateInPad = 64;  // K of the first layer
constexpr int kSurrogateHidden = 128;
constexpr int kSurrogateOutPad = 16; // N of the last layer (2 used)

// Device parameters: FP32 masters, BF16 copies read by the kernels, FP32
// gradient accumulators, feature normalisation.
struct SurrogateDev {
    const __nv_bfloat16 *w1b, *w2b, *w3b; // 128x64, 128x128, 16x128 row-major
    const float *b1, *b2, *b3;            // 128, 128, 16
    const float *mean, *inv_std;          // 48
    float *gw1, *gw2, *gw3, *gb1, *gb2, *gb3;
};

size_t mlp_smem_bytes();
// Forward (labels == null) or fused forward + backward over n rows of
// features. out: n x 2 (logit of acceptance, predicted error / limit) or null
// in training. Training adds the gradients of mean(BCE + Huber) x grad_scale
// x n to the accumulators and the summed loss to *loss. error: set to 1 when
// a tensor-core wait gave up.
cudaError_t launch_mlp(const SurrogateDev& w, const float* features, uint32_t n, float* out, const float* labels,
                       float grad_scale, float* loss, uint32_t* error, uint32_t max_ctas, cudaStream_t s);
void launch_adam(float* w, float* g, float* m, float* v, __nv_bfloat16* wb, uint32_t n, float lr, float b1, float b2,
                 float eps, uint32_t step, const uint8_t* mask, cudaStream_t s);
// Features of the legal edits (count on the device, capacity rows).
void launch_features(const DevMesh& m, const DevTopology& t, const Edit* edits, const uint32_t* count,
                     uint32_t capacity, float px, float px2, float* out, cudaStream_t s);
// Pruning: keys = acceptance logits; then keep the `keep` best and compact the
// ShortestEdge order to those edits (out, count = keep).
void launch_prune_prepare(const float* out, uint32_t n, float* keys, uint32_t* idx, cudaStream_t s);
void launch_prune_order(const uint32_t* sorted_idx, uint32_t n, uint32_t keep, uint32_t* flags,
                        const uint32_t* order, uint32_t* rank_flags, uint32_t* offsets, uint32_t* scan_scratch,
                        uint32_t* out, cudaStream_t s);

} // namespace b200
