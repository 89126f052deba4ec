// TEST INFRASTRUCTURE: stands in for the header cuPoly's CMake configures from
// cuPolyConfig.h.in (version 0.3.5, tweak 12, CMakeLists.txt:4-8).
#pragma once
#define cuPoly_VERSION_MAJOR 0
#define cuPoly_VERSION_MINOR 3
#define cuPoly_VERSION_PATCH 5
#define cuPoly_VERSION_TWEAK 12
