// Stand-in for <NTL/ZZ.h> when NTL is not installed: exposes cupoly::ZZ
// (include/cuPoly/zz.h) under NTL's names, so code written against cuPoly's
// NTL-typed API (poly_set_coeff(ctx, p, i, to_ZZ(42)), CUDAEngine::RNSProduct,
// conv<ZZ>("...")) compiles unchanged with -I include -I include/ntl_shim.
// With NTL installed, leave this directory off the include path and build the
// layer with -DCUPOLY_WITH_NTL.
#pragma once
#include <cuPoly/zz.h>

namespace NTL {
using cupoly::abs;
using cupoly::conv;
using cupoly::IsZero;
using cupoly::NumBits;
using cupoly::power;
using cupoly::power2_ZZ;
using cupoly::sign;
using cupoly::to_long;
using cupoly::to_ZZ;
using cupoly::ZZ;
}  // namespace NTL

#ifndef NTL_CLIENT
#define NTL_CLIENT \
  using namespace std; \
  using namespace NTL;
#endif
