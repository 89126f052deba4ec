// cuPoly compatibility layer: enums, element type and macros of cuPoly's
// include/cuPoly/settings.h:33-80, 144-155, over the cupoly_b200 C ABI.
//
// Same names and values (bases, dgt_direction, add_mode_t, GaussianInteger's
// 16-byte layout), so poly_t device buffers are byte-compatible with cuPoly's.
// cudaCheckError() throws std::runtime_error where cuPoly calls exit(1).
#ifndef SETTINGS_H
#define SETTINGS_H
#include <cuda_runtime_api.h>
#include <cupoly_b200.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include <cuPoly/tool/version.h>

enum add_mode_t { ADD, SUB, MUL, MULMUL, ADDADD };
enum bases { QBase, BBase, QBBase, TBase, QTBBase };
enum dgt_direction { FORWARD, INVERSE };

static_assert((int)QBase == (int)CP_QBASE && (int)BBase == (int)CP_BBASE && (int)QBBase == (int)CP_QBBASE &&
                  (int)TBase == (int)CP_TBASE,
              "base numbering must match the C ABI");
static_assert((int)FORWARD == (int)CP_FORWARD && (int)INVERSE == (int)CP_INVERSE,
              "direction numbering must match the C ABI");
static_assert((int)ADD == (int)CP_ADD && (int)SUB == (int)CP_SUB && (int)MUL == (int)CP_MUL &&
                  (int)MULMUL == (int)CP_MULMUL && (int)ADDADD == (int)CP_ADDADD,
              "operation numbering must match the C ABI");

#define HAMMINGWEIGHT_H 64

typedef struct {
  uint64_t lo = 0;
  uint64_t hi = 0;
} uint128_t;

// One element of Z_p[i]: coefficient j (re) and j + N (imag) of a residue.
typedef struct GaussianInteger {
  uint64_t re;
  uint64_t imag;
  inline bool operator==(const GaussianInteger& b) const { return re == b.re && imag == b.imag; }
} GaussianInteger;
static_assert(sizeof(GaussianInteger) == 16, "GaussianInteger is two uint64 words");

#define FPERROR 1e-9
#ifdef CKKS_ENGINE_MODE
#define MAX_COPRIMES 200
#else
#define MAX_COPRIMES 30
#endif
#define MAX_COPRIMES_IN_A_BASE MAX_COPRIMES / 2
#define GAUSSIAN_STD_DEVIATION (float)3.2
#define GAUSSIAN_BOUND (float)0

#define cudaCheckError()                                                                                      \
  {                                                                                                           \
    cudaError_t cp_e_ = cudaGetLastError();                                                                  \
    if (cp_e_ != cudaSuccess)                                                                                 \
      throw std::runtime_error(std::string("Cuda failure ") + __FILE__ + ":" + std::to_string(__LINE__) + \
                               ": " + cudaGetErrorString(cp_e_));                                            \
  }

#endif
