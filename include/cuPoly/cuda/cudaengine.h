// cuPoly's CUDAEngine (include/cuPoly/cuda/cudaengine.h:59-406): the process-wide
// parameter set (k, kl, nphi, t) and its RNS bases, here backed by one cupoly_b200
// engine (cp_engine) reached through the C ABI.  init() selects cuPoly's primes
// (BFV: 63-bit bucket; with CKKS_ENGINE_MODE defined before inclusion, init()
// takes the CKKS precision instead of t, as in cuPoly's CKKS build).  Errors
// throw std::runtime_error (cuPoly: assert / exit(1)).
#ifndef CUDA_FUNCTIONS_H
#define CUDA_FUNCTIONS_H
#include <NTL/ZZ.h>
#include <cuPoly/settings.h>

#include <vector>

class Context;

typedef struct {
  int k;            // size of the main base Q
  int kl = -1;      // size of the auxiliary base B (k + 1 when negative)
  int nphi;         // ring degree
  uint64_t pt;      // plaintext modulus t (BFV) or precision in bits (CKKS)
} CUDAParams;

size_t poly_get_residues_size(int base);

class CUDAEngine {
 public:
  static int is_init;
  static int N;                  // nphi / 2: Gaussian elements per residue
  static uint64_t t;             // plaintext modulus (BFV) / precision (CKKS)
  static int scalingfactor;      // CKKS precision, 0 for BFV
  static int dnum;               // kept for source compatibility (CKKS bootstrap), unused
  static std::vector<uint64_t> RNSPrimes;   // Q
  static std::vector<uint64_t> RNSBPrimes;  // B
  static NTL::ZZ RNSProduct;                // prod Q
  static NTL::ZZ RNSBProduct;               // prod B
  static std::vector<NTL::ZZ> RNSMpi;       // Q / q_i
  static std::vector<uint64_t> RNSInvMpi;   // (Q / q_i)^-1 mod q_i
  static cp_engine* engine;                 // the C-ABI engine behind the statics

  static void init(const int k, const int kl, const int M, const uint64_t t) {
#ifdef CKKS_ENGINE_MODE
    init_ckks(k, kl, M, (int)t);
#else
    init_bfv(k, kl, M, t);
#endif
  }
  static void init(CUDAParams p) { init(p.k, p.kl, p.nphi, p.pt); }
  static void init_bfv(int k, int kl, int M, uint64_t t);
  static void init_ckks(int k, int kl, int M, int prec);
  static void destroy();
  static int get_n_residues(int base);
  static cp_engine* handle();  // the engine; throws when not initialised
  // DGT-domain roots: engines use the library's canonical root of i unless the
  // environment variable CUPOLY_COPRIMES_DIR names cuPoly's
  // src/arithmetic/coprimes directory at init, in which case they take
  // cuPoly's NTHROOT (coprimes.cu:868) from its qis_<bits>.json files and
  // poly_t::d_coefs holds cuPoly's own DGT-domain bytes.  This loads the same
  // table into the current engine explicitly (throws when a root is missing).
  static void load_nthroot_table(const std::string& coprimes_dir);

  // cudaengine.h:140-185 (elementwise, any domain)
  static void execute_polynomial_negate(GaussianInteger* b, const GaussianInteger* a, const int base, Context* ctx);
  static void execute_polynomial_op_by_int(GaussianInteger* b, GaussianInteger* a, const int base, uint64_t x,
                                           int OP, Context* ctx);
  static void execute_polynomial_double_op_by_int(GaussianInteger* b1, GaussianInteger* a1, GaussianInteger* b2,
                                                  GaussianInteger* a2, const int base, uint64_t x1, uint64_t x2,
                                                  int OP, Context* ctx);
};
#endif
