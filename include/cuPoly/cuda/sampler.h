// cuPoly's Sampler (include/cuPoly/cuda/sampler.h:38-101) over cp_sample.
// Counter-based (Philox4x32-10): each sample() call draws stream id = a
// per-process counter under the seed, so a sequence of calls is reproducible
// after Sampler::init / reset.  Distributions keep cuPoly's enum values and
// meanings: on a BFV engine UNIFORM is one value uniform below 2^32 written to
// every residue (sampler.cu:295-341) and ZO has exactly nphi/2 nonzero
// coefficients, each +-1 (sampler.cu:236-283).  UNIFORM_MOD_Q and ZO_IID give
// the library's independent forms; TERNARY and GAUSSIAN (signed) are
// additions.  Samples are returned in the DGT domain (RNSSTATE), as cuPoly's are.
#ifndef SAMPLER_H
#define SAMPLER_H
#include <cuPoly/arithmetic/polynomial.h>
#include <cuPoly/settings.h>

enum pdistributions {
  DISCRETE_GAUSSIAN = CP_DISCRETE_GAUSSIAN,
  HAMMINGWEIGHT = CP_HAMMINGWEIGHT,
  NARROW = CP_NARROW,
  ZO = CP_ZO,
  BINARY = CP_BINARY,
  UNIFORM = CP_UNIFORM,
  TERNARY = CP_TERNARY,
  GAUSSIAN = CP_GAUSSIAN,
  KINDS_COUNT,
  // The library's independent forms of UNIFORM and ZO (values of this layer only):
  UNIFORM_MOD_Q = 105,  // uniform mod each q_i, independently per residue
  ZO_IID = 103          // i.i.d. -1 : 1/4, 0 : 1/2, +1 : 1/4
};

#define SEED (unsigned long long)(42)

class Sampler {
 public:
  static uint64_t seed;       // Philox key (cuPoly: SEED)
  static uint32_t counter;    // next stream id
  static void init(Context* ctx);
  static void reset(Context* ctx);
  static void sample(Context* ctx, poly_t* p, int kind);
  static poly_t* sample(Context* ctx, int kind);  // new poly_t; the caller deletes it
  static void destroy() {}
};
#endif
