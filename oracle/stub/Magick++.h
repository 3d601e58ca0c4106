// Minimal stand-in for the Magick++ header so that the reference 2D solver
// (LMB2d/main.cpp + LMB2d/lbm.cpp) compiles without ImageMagick.  Only the
// names those two files use exist here.  The .dat and .ppm readers are plain
// C++ and work unchanged; a .gif input raises at run time instead of decoding.
// Used only by oracle/build_ref.sh for the CPU reference binary.
#pragma once
#include <stdexcept>
#include <string>

namespace Magick {
inline void InitializeMagick(const char *) {}
struct PixelPacket { unsigned short red, green, blue, opacity; };
class Image {
public:
    explicit Image(const std::string &name)
    { throw std::runtime_error("GIF decoding is not available in this build: " + name); }
    PixelPacket *getPixels(int, int, int, int) { return nullptr; }
};
}  // namespace Magick
