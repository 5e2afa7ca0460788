#pragma once
// raymotion/metal.hpp - the backend entry point (reference
// include/raymotion/metal.hpp:6-7).  librmcuda.so defines it over the C ABI of
// rmcuda.h; the name is kept so that the engine's Renderer and its tests link
// unchanged.
#include <string>

#include "raymotion/pathtrace.hpp"

namespace raymotion {
// Returns false with a diagnostic when the frame cannot be completed.
bool render_image_metal(const Scene&, const Camera&, const RenderConfig&, uint64_t, std::vector<uint8_t>&,
                        std::string&);
}
