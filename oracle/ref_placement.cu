// Runs the reference's own GPU placement path — TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile links this driver with the reference's unmodified
// src/neural/action_gpu.cu and src/mesh.cpp into oracle/_ref/placement_ref.
// For a mesh and a list of legal directed collapses it builds
// GpuActionState::trial(action, midpoint placement) on the GPU — the
// reference's place_vertices (action_gpu.cu:962-1067: positions, uv
// transport) and validate_placement (1103-1156: orientation, uv flip,
// position coincidence) — and writes each trial's validity, face count,
// indices, positions and uv. It needs a CUDA device; it is run once to make
// tests/golden/placement_ref.npz (tests/golden/make_placement_golden.py).
//
//   placement_ref INPUT OUTPUT
// INPUT: u32 vertices, faces, has_uv, preserve_uv, stride; f32 positions
// [3 V]; f32 uv [2 V] when has_uv; u32 indices [3 F]. The collapses are
// every `stride`-th legal action of the reference's enumeration.
// OUTPUT per collapse: u32 from, to, valid, faces; then, when valid, u32
// indices [3 faces], f32 positions [3 V], f32 uv [2 V] when has_uv.
#include "neural/action_gpu.hpp"

#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include <cuda_runtime.h>

namespace blitz::neural {
// The executor's learned ranking references the policy network; this driver
// never ranks, so these are never called.
void ActionCuda::predict_device(const float*, float*, uint32_t) { throw std::logic_error("no policy network here"); }
uint32_t ActionCuda::architecture() const { throw std::logic_error("no policy network here"); }
ModelUse ActionCuda::model_use() const { throw std::logic_error("no policy network here"); }
} // namespace blitz::neural

using namespace blitz;

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: placement_ref INPUT OUTPUT\n");
        return 2;
    }
    try {
        FILE* in = std::fopen(argv[1], "rb");
        if (!in) throw std::runtime_error("cannot open input");
        uint32_t head[5];
        if (std::fread(head, 4, 5, in) != 5) throw std::runtime_error("short input");
        const uint32_t nv = head[0], nf = head[1], has_uv = head[2], preserve_uv = head[3], stride = head[4];
        std::vector<float> pos(size_t(nv) * 3), uv(has_uv ? size_t(nv) * 2 : 0);
        std::vector<uint32_t> idx(size_t(nf) * 3);
        if (std::fread(pos.data(), 4, pos.size(), in) != pos.size() ||
            (has_uv && std::fread(uv.data(), 4, uv.size(), in) != uv.size()) ||
            std::fread(idx.data(), 4, idx.size(), in) != idx.size())
            throw std::runtime_error("short input");
        std::fclose(in);
        MeshView m;
        m.positions = Stream<Vec3>(reinterpret_cast<const Vec3*>(pos.data()), nv);
        if (has_uv) m.uv = Stream<Vec2>(reinterpret_cast<const Vec2*>(uv.data()), nv);
        m.indices = {idx.data(), idx.size()};
        NeuralOptions options;
        options.preserve_uv = preserve_uv != 0;
        neural::GpuActionState state(m, options, true);
        std::array<float, neural::conditions> c{};
        const auto actions = state.actions(c);
        FILE* out = std::fopen(argv[2], "wb");
        if (!out) throw std::runtime_error("cannot open output");
        std::vector<uint32_t> tidx;
        std::vector<float> tpos(size_t(nv) * 3), tuv(has_uv ? size_t(nv) * 2 : 0);
        for (size_t k = 0; k < actions.size(); k += std::max<uint32_t>(1, stride)) {
            const neural::Action a = actions[k].action;
            const Vec3 p = (m.positions[a.from] + m.positions[a.to]) * 0.5; // mesh.hpp:22-23 arithmetic
            neural::Placement placement{p, {Vec3{}, Vec3{}}};
            neural::DeviceMeshView view;
            const bool valid = state.trial(a, placement, view);
            uint32_t rec[4] = {a.from, a.to, uint32_t(valid), valid ? view.faces : 0u};
            std::fwrite(rec, 4, 4, out);
            if (!valid) continue;
            tidx.resize(size_t(view.faces) * 3);
            if (cudaMemcpy(tidx.data(), view.indices, tidx.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(tpos.data(), view.positions, tpos.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
                (has_uv && cudaMemcpy(tuv.data(), view.uv, tuv.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess))
                throw std::runtime_error("device copy failed");
            std::fwrite(tidx.data(), 4, tidx.size(), out);
            std::fwrite(tpos.data(), 4, tpos.size(), out);
            if (has_uv) std::fwrite(tuv.data(), 4, tuv.size(), out);
        }
        std::fclose(out);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
