// Coverage distance without any device allocation.
//
// Some callers cannot call cudaMalloc: a plugin hosted by an engine whose
// device memory is owned by another allocator (a framework's caching
// allocator, or a host that hands each plugin a fixed budget up front), or a
// hot loop that must not take the device-wide synchronisation that
// cudaMalloc/cudaFree can imply. For them this file keeps the scratch of the
// exact distance transform in one file-scope __device__ array of a fixed,
// modest size, loaded with the library and held by every GPU that loads it
// until the process exits. The caller passes device inputs and a device
// output; nothing is allocated, freed or synchronised here.
#include "../../include/blitz_audit.h"
#include "kernels.cuh"

#include <cstring>
#include <mutex>

namespace b200 {
namespace {

// Largest mask handled: 512 x 512 samples.
constexpr size_t kStaticSamples = 512 * 512;
constexpr size_t align256(size_t n) { return (n + 255) & ~size_t(255); }
// Scratch layout: row distances g, squared distances d2, envelope stack
// (vertex, numerator, denominator), popcounts, directed maxima.
constexpr size_t kOffG = 0;
constexpr size_t kOffD2 = kOffG + align256(kStaticSamples * 4);
constexpr size_t kOffV = kOffD2 + align256(kStaticSamples * 4);
constexpr size_t kOffNum = kOffV + align256(kStaticSamples * 4);
constexpr size_t kOffDen = kOffNum + align256(kStaticSamples * 8);
constexpr size_t kOffPop = kOffDen + align256(kStaticSamples * 8);
constexpr size_t kOffMax = kOffPop + align256(4 * 8);
constexpr size_t kStaticBytes = kOffMax + align256(2 * 4);

static __device__ __align__(256) unsigned char g_distance_scratch[kStaticBytes];

// Device address of g_distance_scratch per device ordinal, looked up with
// that device current. Outside stream capture every call looks it up again
// (a context torn down and created anew, e.g. after cudaDeviceReset, loads
// the module at a new address); during capture the address of the last call
// outside capture is used, so the first call on a device must come before
// any capture.
std::mutex g_setup_mutex;
void* g_scratch_address[64] = {};

__global__ void k_static_clear(unsigned long long* pop, uint32_t* maxes) {
    if (threadIdx.x < 4) pop[threadIdx.x] = 0;
    if (threadIdx.x < 2) maxes[threadIdx.x] = 0;
}

// Same value as the session entry point (evaluate.cpp:202-208): equal masks 0,
// exactly one empty infinity, else sqrt(max squared distance)/supersample.
__global__ void k_static_finish(const unsigned long long* pop, const uint32_t* maxes, uint32_t ss, double* out) {
    if (threadIdx.x || blockIdx.x) return;
    ViewRecord r{};
    r.changed = pop[0] ? 1u : 0u;
    r.ca = pop[2] > 0;
    r.cb = pop[3] > 0;
    const double a = double(__uint_as_float(maxes[0])), c = double(__uint_as_float(maxes[1]));
    *out = coverage_value(r, ss, a > c ? a : c);
}

void message(char* out, size_t n, const char* text) {
    if (out && n) {
        size_t k = strlen(text) < n - 1 ? strlen(text) : n - 1;
        memcpy(out, text, k);
        out[k] = 0;
    }
}
} // namespace
} // namespace b200

using namespace b200;

extern "C" blitz_status blitz_audit_coverage_distance_static(const uint64_t* a_device, const uint64_t* b_device,
                                                             uint32_t width, uint32_t height, uint8_t supersample,
                                                             double* out_device, void* stream, char* error,
                                                             size_t error_capacity) {
    message(error, error_capacity, "");
    if (!a_device || !b_device || !out_device || !width || !height || !supersample) {
        message(error, error_capacity, "null pointer or zero extent");
        return BLITZ_INVALID_ARGUMENT;
    }
    if (uint64_t(width) * height > kStaticSamples) {
        message(error, error_capacity, "mask exceeds the static scratch maximum of 262144 samples (512 x 512)");
        return BLITZ_INVALID_ARGUMENT;
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) {
        cudaGetLastError();
        message(error, error_capacity, "no current CUDA device");
        return BLITZ_UNAVAILABLE;
    }
    // An error left by the caller's earlier work stays theirs: report it
    // without consuming it, and enqueue nothing.
    if (cudaPeekAtLastError() != cudaSuccess) {
        message(error, error_capacity, "a CUDA error from earlier work is pending on this thread; nothing enqueued");
        return BLITZ_INTERNAL_ERROR;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &capture) != cudaSuccess) {
        cudaGetLastError();
        message(error, error_capacity, "cudaStreamIsCapturing failed on the given stream");
        return BLITZ_INVALID_ARGUMENT;
    }
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (capture == cudaStreamCaptureStatusNone) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_distance_scratch);
            if (e != cudaSuccess || !ptr) {
                cudaGetLastError();
                message(error, error_capacity, "cudaGetSymbolAddress of the static scratch failed");
                return BLITZ_UNAVAILABLE;
            }
            g_scratch_address[device] = ptr;
        } else if (!g_scratch_address[device]) {
            message(error, error_capacity,
                    "first call on this device during stream capture: call once outside capture first");
            return BLITZ_INVALID_ARGUMENT;
        }
        base = static_cast<unsigned char*>(g_scratch_address[device]);
    }
    auto* g = reinterpret_cast<uint32_t*>(base + kOffG);
    auto* d2 = reinterpret_cast<uint32_t*>(base + kOffD2);
    auto* sv = reinterpret_cast<int32_t*>(base + kOffV);
    auto* sn = reinterpret_cast<long long*>(base + kOffNum);
    auto* sd = reinterpret_cast<long long*>(base + kOffDen);
    auto* pop = reinterpret_cast<unsigned long long*>(base + kOffPop);
    auto* maxes = reinterpret_cast<uint32_t*>(base + kOffMax);
    const auto* a = reinterpret_cast<const uint32_t*>(a_device);
    const auto* b = reinterpret_cast<const uint32_t*>(b_device);
    const uint32_t words = uint32_t(((uint64_t(width) * height + 63) / 64) * 2);
    // The counters keep the previous call's contents: clear them first.
    k_static_clear<<<1, 32, 0, st>>>(pop, maxes);
    // Bits at or past width x height are not samples: they do not count.
    launch_popcounts(a, b, words, pop, st, uint64_t(width) * height);
    launch_distance(a, b, width, height, g, d2, sv, sn, sd, maxes, st);
    launch_distance(b, a, width, height, g, d2, sv, sn, sd, maxes + 1, st);
    k_static_finish<<<1, 32, 0, st>>>(pop, maxes, supersample, out_device);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        message(error, error_capacity, cudaGetErrorString(e));
        return BLITZ_INTERNAL_ERROR;
    }
    return BLITZ_OK;
}
