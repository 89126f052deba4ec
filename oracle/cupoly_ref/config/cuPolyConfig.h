// TEST INFRASTRUCTURE: the same version header under the name cuPoly's
// settings.h includes ("cuPolyConfig.h").
#pragma once
#include <cuPoly/cuPolyConfig.h>
