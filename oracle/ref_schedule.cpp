// Runs the reference's own blitz::schedule (src/chain.cpp:101-118, with
// Curve::at 25-36) — TEST INFRASTRUCTURE ONLY. oracle/Makefile links this
// file with the reference's unmodified src/chain.cpp, keeping only what
// schedule() reaches (--gc-sections), into oracle/_ref/schedule_ref.
//
//   schedule_ref LEVELS BASE_PX LAST_PX LOD0_PX [X Y]...
// LOD0_PX 0 leaves the LOD0 bound uncapped. Prints one line per level:
// pixels, transition and source bound as C99 hex floats.
#include "blitz/remesher.hpp"

#include <cstdio>
#include <cstdlib>
#include <exception>

int main(int argc, char** argv) {
    if (argc < 7 || (argc - 5) % 2) {
        std::fprintf(stderr, "usage: schedule_ref LEVELS BASE LAST LOD0 X Y [X Y]...\n");
        return 2;
    }
    blitz::Settings s;
    s.levels = uint8_t(std::atoi(argv[1]));
    s.base_pixels = std::strtod(argv[2], nullptr);
    s.last_pixels = std::strtod(argv[3], nullptr);
    const double lod0 = std::strtod(argv[4], nullptr);
    if (lod0 > 0) s.max_lod0_delta_px = lod0;
    s.transition.points.clear();
    for (int i = 5; i + 1 < argc; i += 2)
        s.transition.points.push_back({std::strtof(argv[i], nullptr), std::strtof(argv[i + 1], nullptr)});
    try {
        for (const auto& e : blitz::schedule(blitz::Bounds{}, s))
            std::printf("%a %a %a\n", e.pixels, e.transition, e.source);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
