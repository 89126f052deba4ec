/*
 * cupoly_b200 -- C ABI of the B200-native cyclotomic-polynomial engine.
 *
 * This is the drop-in boundary for cuPoly's hot path (pdroalves/cupoly 0.3.5):
 * the hierarchical DGT, RNS pointwise arithmetic, HPS basis extension and
 * t/Q scaling, and the sampler.  Every entry point takes plain pointers,
 * sizes and a CUDA stream (as void*); none allocates device memory except
 * cp_engine_create.  Status codes are returned; the message of the last
 * failure on the calling thread is available from cp_last_error().
 *
 * Data layout (cuPoly include/cuPoly/settings.h:70-80,
 * src/arithmetic/polynomial.cu:206-217): a polynomial over a base with nres
 * primes is `uint64_t[nres][N][2]` (N = nphi / 2 Gaussian elements per
 * residue; element j of residue r holds (a_j mod p_r, a_{j+N} mod p_r)).
 * Values are canonical in [0, p_r).  "DGT domain" buffers hold the forward
 * transform in cuPoly's order (bit-reversed twisted DFT).
 *
 * Bases (cuPoly `enum bases`, settings.h:37): CP_QBASE = the first k primes,
 * CP_BBASE = the next kl primes, CP_QBBASE = Q followed by B, CP_TBASE = the
 * plaintext modulus t (one residue).
 */
#ifndef CUPOLY_B200_H
#define CUPOLY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define CP_OK 0
#define CP_ERR_INVALID 1     /* bad argument (cuPoly: assert / runtime_error) */
#define CP_ERR_CUDA 2        /* CUDA runtime error (cuPoly: cudaCheckError -> exit) */
#define CP_ERR_UNSUPPORTED 3 /* size/parameter outside the compiled range */
#define CP_ERR_OOM 4         /* device allocation failed */
#define CP_ERR_DEVICE 5      /* a kernel reported an error through the engine's flag */

/* ---- enums (values equal cuPoly's) ---- */
enum cp_base { CP_QBASE = 0, CP_BBASE = 1, CP_QBBASE = 2, CP_TBASE = 3 };
enum cp_direction { CP_FORWARD = 0, CP_INVERSE = 1 };                 /* dgt_direction, settings.h:41 */
enum cp_op { CP_ADD = 0, CP_SUB = 1, CP_MUL = 2, CP_MULMUL = 3, CP_ADDADD = 4 }; /* add_mode_t, settings.h:33 */
enum cp_distribution {                                                  /* pdistributions, sampler.h:38-47 */
  CP_DISCRETE_GAUSSIAN = 0, /* |nearbyint(3.2 Z)|, |x| <= 19 (cuPoly BFV semantics) */
  CP_HAMMINGWEIGHT = 1,     /* exactly min(64, nphi) coefficients in {-1, +1} */
  CP_NARROW = 2,            /* uniform {0, 1, 2} */
  CP_ZO = 3,                /* i.i.d. -1 : 1/4, 0 : 1/2, +1 : 1/4 */
  CP_BINARY = 4,            /* uniform {0, 1} */
  CP_UNIFORM = 5,           /* uniform mod q_i, independent per residue */
  CP_TERNARY = 6,           /* uniform {-1, 0, +1} (secrets) */
  CP_GAUSSIAN = 7,          /* discrete Gaussian, sigma = 3.19, |x| <= 19, signed (errors) */
  /* cuPoly's BFV meanings of UNIFORM and ZO, under their own values:           */
  CP_UNIFORM_U32 = 9,       /* one value uniform in [0, 2^32) per coefficient, the same on every
                               residue (sampler.cu:295-341: floor(u (2^32 - 1)) for all residues) */
  CP_ZO_HALF = 10           /* exactly nphi/2 coefficients nonzero, each +-1 with probability 1/2
                               (sampler.cu:236-283: N values in {1, 2} shuffled among 2N) */
};
/* flags of the composite scaling calls */
#define CP_DESTROY_INPUTS 1u /* inverse-transform the inputs in place, as cuPoly does (polynomial.h:346-347) */

typedef struct cp_engine cp_engine;

/* ---- library ---- */
const char* cp_version(void);
const char* cp_last_error(void);

/* ---- engine: replaces CUDAEngine::init(k, kl, M, t) / destroy() / get_n_residues(base)
 *      (cuPoly include/cuPoly/cuda/cudaengine.h:65-123, src/cuda/cudaengine.cu:1691-1779)
 *      and DGTEngine::init (src/cuda/dgt.cu:1694-1982).  nphi is the ring degree
 *      (cuPoly's M), 4 <= nphi <= 65536 a power of two; kl <= 0 selects k + 1;
 *      any t >= 2 coprime to Q (cuPoly requires a power of two).  The engine is
 *      created on the current CUDA device.  log_radix in {3, 4} picks the DGT
 *      register radix (0 = default).  The default plan keeps the whole transform in
 *      one CTA up to nphi 8192 and puts the top 2 bits in the split stage from nphi
 *      16384 on (log_cta = log2(nphi / 2) - 2), the fastest measured on B200. */
int cp_engine_create(cp_engine** out, int k, int kl, int nphi, uint64_t t, int log_radix);
/* CKKS-mode engine: replaces CUDAEngine::init(k, kl, M, prec) of cuPoly's CKKS build
 * (src/cuda/cudaengine.cu:1192-1290).  Q = the first 63-bit prime followed by k - 1
 * primes of the prec-bit bucket (prec in {45, 48, 52, 55}); B = kl primes of the
 * 45-bit (prec 45) or 55-bit bucket starting at index k - 1.  Every prime must have
 * 2 nphi | p - 1 (CP_ERR_UNSUPPORTED otherwise).  The BFV base conversions and
 * scalings (cp_basis_ext_*, cp_*_scaling, cp_xi/cp_rho, cp_bfv_mul*) refuse a CKKS
 * engine with CP_ERR_UNSUPPORTED; the DGT, pointwise, sampler, CRT and wire calls
 * work on both. */
int cp_ckks_engine_create(cp_engine** out, int k, int kl, int nphi, int prec, int log_radix);
/* precision bucket of a CKKS engine, 0 for a BFV engine */
int cp_engine_ckks_prec(const cp_engine* e);
/* DGT plan (no counterpart in cuPoly, whose split is fixed per size, include/cuPoly/cuda/dgt.h:41-50):
 * register radix 2^log_radix and the largest size kept whole in one CTA, 2^log_cta
 * (0 = 2^13); the remaining log2(N) - log_cta <= 2 bits run in an element-wise split
 * stage.  Rebuilds the engine's tables (synchronises the device).  The autotuner
 * (cupoly_b200/autotune.py) measures the candidates and caches the fastest. */
int cp_engine_set_plan(cp_engine* e, int log_radix, int log_cta);
int cp_engine_get_plan(const cp_engine* e, int* log_radix, int* log_cta, int* split_bits);
/* Second DGT plan for small launches (no counterpart in cuPoly): a transform launch of at
 * most max_units residue transforms (polynomials x residues) uses (log_radix, log_cta)
 * instead of the main plan; max_units = 0 removes it.  With few residues per launch, one
 * CTA per residue leaves most SMs idle, and a plan whose split stage spreads each residue
 * over 2-4 CTAs finishes sooner.  Results are identical.  Same limits as cp_engine_set_plan;
 * the split stage of this plan is always the separate kernel.  Rebuilds the engine's
 * tables (synchronises the device).  The autotuner picks the plan and the crossover.
 * Default: radix 4 (log_radix 2), log_cta = log2(nphi / 2) - 2, up to 96 units at nphi
 * 4096 and 8192, up to 16 at nphi 16384, none otherwise.  get: zeros when there is no
 * such plan. */
int cp_engine_set_narrow_plan(cp_engine* e, int log_radix, int log_cta, long long max_units);
int cp_engine_get_narrow_plan(const cp_engine* e, int* log_radix, int* log_cta, long long* max_units);
/* Form of the split stage of transforms larger than one CTA (plans with split bits > 0; no
 * counterpart in cuPoly, whose two-pass split always goes through HBM):
 * 0 = a separate element-wise kernel with its own HBM pass (default);
 * 1 = inside a thread-block cluster of 2^split_bits CTAs, the chunks exchanged through
 *     distributed shared memory.  Results are identical; where the cluster form has no kernel
 *     for the plan or the device cannot co-schedule the cluster, mode 1 falls back to 0. */
int cp_engine_set_split_mode(cp_engine* e, int mode);
int cp_engine_get_split_mode(const cp_engine* e);
/* Diagnostic switch (no counterpart in cuPoly): 1 makes every base conversion and scaling
 * take its exact mixed-radix path instead of the FP64 fast path, 0 (default) restores it.
 * Results are identical either way; the tests use it to drive the exact paths on ordinary
 * inputs.  Synchronises the device. */
int cp_engine_set_hps_force_exact(cp_engine* e, int on);
int cp_engine_destroy(cp_engine* e);
int cp_engine_n_residues(const cp_engine* e, int base);
int cp_engine_nphi(const cp_engine* e);
/* primes of the engine, Q then B (cuPoly CUDAEngine::RNSPrimes / RNSBPrimes) */
int cp_engine_primes(const cp_engine* e, uint64_t* out, int capacity);
/* Replace the Gaussian root xi (xi^N = i) of every residue, e.g. with cuPoly's
 * NTHROOT[p][N] table (src/arithmetic/coprimes.cu:868), so that DGT-domain
 * bytes match cuPoly's; xi is uint64_t[nres_QB][2].  Default: the canonical
 * root ((u + u^-1)/2, (u - u^-1)/(2 s)), u = g^((p-1)/(4N)), s = g^((p-1)/4). */
int cp_engine_set_nthroot(cp_engine* e, const uint64_t* xi);
int cp_engine_get_nthroot(const cp_engine* e, uint64_t* xi_out);
/* bytes of scratch the composite calls below need */
size_t cp_workspace_bytes(const cp_engine* e);
/* read and clear the engine's device error flag (synchronises `stream`) */
int cp_engine_check(const cp_engine* e, void* stream);
/* the engine's error flag, copied into flag_host (page-locked host memory) on `stream` behind
 * the work already queued there, without waiting: nonzero once the copy has completed means
 * that cp_engine_check will report the error (and reset the flag). */
int cp_engine_check_async(const cp_engine* e, int* flag_host, void* stream);

/* ---- DGT: replaces DGTEngine::execute_dgt(data, base, direction, ctx)
 *      (src/cuda/dgt.cu:1069-1094).  In place on npolys consecutive polynomials
 *      of the base (poly_stride = 0 means densely packed). */
int cp_dgt(const cp_engine* e, void* data, int base, int direction, int npolys, int64_t poly_stride, void* stream);

/* ---- work-list forms (no counterpart in cuPoly): `nlist` residues of N Gaussian
 *      elements back to back; residue i uses the engine's prime rid_list[i]
 *      (device int array, values < cp_engine_n_residues(e, CP_QBBASE)).  Lets
 *      polynomials of different RNS widths share one launch. ---- */
int cp_dgt_list(const cp_engine* e, void* data, const int* rid_list, int nlist, int direction, void* stream);
int cp_mul_list(const cp_engine* e, void* c, const void* a, const void* b, const int* rid_list, int nlist,
                void* stream);

/* ---- fused negacyclic polymul, coefficient domain in and out (no counterpart in cuPoly,
 *      whose poly_mul composes upload DGTs, mul_dgt and a download IDGT,
 *      src/arithmetic/polynomial.cu:892-914 with :105-188): c = a b mod (x^nphi + 1, q_r)
 *      per residue, as forward DGT of a and b out of place into the workspace, then an
 *      inverse DGT that forms the Gaussian products while loading (3 launches).  c may
 *      alias a or b.  cp_polymul: npolys polynomials over `base`, workspace of
 *      cp_polymul_workspace_bytes bytes.  cp_polymul_list: work-list form (see
 *      cp_dgt_list), wa and wb each nlist x N x 16 bytes. ---- */
size_t cp_polymul_workspace_bytes(const cp_engine* e, int base, int npolys);
int cp_polymul(const cp_engine* e, void* c, const void* a, const void* b, int base, int npolys, void* workspace,
               void* stream);
int cp_polymul_list(const cp_engine* e, void* c, const void* a, const void* b, void* wa, void* wb,
                    const int* rid_list, int nlist, void* stream);
/* ---- the mixed-size batch of negacyclic products in ONE persistent launch (no
 *      counterpart in cuPoly: one parameter set per process there).  Size group
 *      lg = 0..3 holds rows[lg] residues of ring size N = 2^(10 + lg) (nphi 2048 ..
 *      16384): coefficient-domain rows a[lg], b[lg] -> c[lg] (each rows[lg] x N x 16
 *      bytes; c may alias a or b), residue i using prime rid[lg][i] (device int array)
 *      of engines[lg].  engines[lg] must have N = 2^(10 + lg) and the whole-CTA
 *      radix-8 plan (cp_engine_set_plan(e, 3, 10 + lg)); groups with rows[lg] = 0 may
 *      pass NULL.  `tiles` (device) lists ntiles tiles {lg, first row, count} as three
 *      ints each, count <= 8192 / N: one CTA per SM walks the list, each tile's
 *      residues transformed side by side in shared memory (forward a, forward b,
 *      product, inverse, in one pass over HBM).  A tile outside its group is skipped
 *      and sets the device error flag of the first engine given (cp_engine_check).
 *      Workspace: at least cp_polymul_tiles_workspace_bytes() bytes of device
 *      memory (the current device's SM count x 128 KB). ---- */
size_t cp_polymul_tiles_workspace_bytes(void);
int cp_polymul_tiles(const cp_engine* const* engines, void* const* c, const void* const* a, const void* const* b,
                     const int* const* rid, const int* rows, const void* tiles, int ntiles, void* workspace,
                     size_t workspace_bytes, void* stream);

/* ---- pointwise, DGT domain: replace DGTEngine::execute_{add,sub,double_add,
 *      mul_dgt_gi,mul_dgt_u64,muladd,dr2}_dgt (src/cuda/dgt.cu:1096-1499) ---- */
int cp_add(const cp_engine* e, void* c, const void* a, const void* b, int base, void* stream);
int cp_sub(const cp_engine* e, void* c, const void* a, const void* b, int base, void* stream);
int cp_double_add(const cp_engine* e, void* c1, const void* a1, const void* b1, void* c2, const void* a2,
                  const void* b2, int base, void* stream);
int cp_mul(const cp_engine* e, void* c, const void* a, const void* b, int base, void* stream);
int cp_mul_u64(const cp_engine* e, void* c, const void* a, const uint64_t* b, int base, void* stream);
/* cp_mul over npolys densely packed polynomials (no counterpart in cuPoly) */
int cp_mul_batch(const cp_engine* e, void* c, const void* a, const void* b, int base, int npolys, void* stream);
int cp_muladd(const cp_engine* e, void* d, const void* a, const void* b, const void* c, int base, void* stream);
/* replaces poly_dot (src/arithmetic/polynomial.cu:1439-1451), which composes one
 * poly_mul and n-1 poly_mul_add calls: c = sum_i a[i] b[i] over `base` in the DGT domain
 * in one pass, each operand read once and each sum reduced once per element.  a and b are
 * HOST arrays of n >= 1 device pointers.  c may be the same buffer as any operand among the
 * first 64 pairs (the result is the sum over the inputs as they were before the call); c equal
 * to a later operand returns CP_ERR_INVALID; any other overlap of c with an operand is not
 * allowed. */
int cp_dot(const cp_engine* e, void* c, const void* const* a, const void* const* b, int n, int base,
           void* stream);
/* batched cp_dot (no counterpart in cuPoly): for q < npolys, polynomial q of c = sum_{t<n}
 * a[q n + t] b[q n + t], or b[t] when b_shared (one key set for every q, as in
 * relinearization); a, b, c are densely packed polynomials over `base`, 1 <= n <= 64.  The
 * layout of a is cp_xi_batch's output (n = k).  c must not overlap a or b. */
int cp_dot_batch(const cp_engine* e, void* c, const void* a, const void* b, int n, int npolys, int b_shared,
                 int base, void* stream);
int cp_dr2(const cp_engine* e, void* c21, void* c22, void* c23, const void* c01, const void* c02, const void* c11,
           const void* c12, int base, void* stream);
/* replace CUDAEngine::execute_polynomial_negate / _op_by_int / _double_op_by_int
 * (src/cuda/cudaengine.cu:115-302); op is a cp_op */
int cp_negate(const cp_engine* e, void* b, const void* a, int base, void* stream);
int cp_op_by_int(const cp_engine* e, void* b, const void* a, int base, uint64_t x, int op, void* stream);
int cp_double_op_by_int(const cp_engine* e, void* b1, const void* a1, void* b2, const void* a2, int base,
                        uint64_t x1, uint64_t x2, int op, void* stream);

/* ---- HPS, coefficient domain: replace CUDAEngine::execute_polynomial_basis_ext_Q_to_B /
 *      _B_to_Q / _complex_scaling / _simple_scaling (src/cuda/cudaengine.cu:304-798).
 *      X mod m for the X in [0, S) with the given residues (S = Q, resp. B), lifted as
 *      cuPoly lifts it: X - S when S - X <= S FPERROR (FPERROR = 1e-9, cuPoly's
 *      tolerance, settings.h:105; cuPoly's double overflow count rounds up there),
 *      decided exactly; complex scaling: exact round(t X / Q) mod b_j. */
int cp_basis_ext_q_to_b(const cp_engine* e, void* out_b, const void* in_q, int npolys, void* stream);
int cp_basis_ext_b_to_q(const cp_engine* e, void* out_q, const void* in_b, int npolys, void* stream);
int cp_complex_scaling(const cp_engine* e, void* out_b, const void* in_q, const void* in_b, int npolys,
                       void* stream);
int cp_simple_scaling(const cp_engine* e, void* out_t, const void* in_q, void* stream);
/* replace CUDAEngine::execute_xi_rns / execute_rho_bfv_rns (src/cuda/cudaengine.cu:992-1062):
 * out is k polynomials over Q; polynomial i has residue i set, the rest zero */
int cp_xi(const cp_engine* e, void* out, const void* in, void* stream);
int cp_rho(const cp_engine* e, void* out, const void* in, void* stream);
/* batched forms (no counterpart in cuPoly): npolys input polynomials over Q back to back, out =
 * npolys x k polynomials (input p's decomposition at polynomials p k .. p k + k - 1);
 * npolys k <= 65535 */
int cp_xi_batch(const cp_engine* e, void* out, const void* in, int npolys, void* stream);
int cp_rho_batch(const cp_engine* e, void* out, const void* in, int npolys, void* stream);

/* ---- composite polynomial calls, DGT domain in and out: replace
 *      poly_basis_extension_Q_to_B / _Q_to_QB / _B_to_Q, poly_complex_scaling_tDivQ,
 *      poly_simple_scaling_tDivQ (src/arithmetic/polynomial.cu:310-527).
 *      `workspace` holds cp_workspace_bytes(e) bytes of device memory. */
int cp_poly_basis_extension_q_to_b(const cp_engine* e, void* out_b, const void* in_q, void* workspace,
                                   void* stream);
int cp_poly_basis_extension_q_to_qb(const cp_engine* e, void* out_qb, const void* in_q, void* workspace,
                                    void* stream);
int cp_poly_basis_extension_b_to_q(const cp_engine* e, void* out_q, const void* in_b, void* workspace,
                                   void* stream);
int cp_poly_complex_scaling_tdivq(const cp_engine* e, void* out_q, void* in_q, void* in_b, unsigned flags,
                                  void* workspace, void* stream);
int cp_poly_simple_scaling_tdivq(const cp_engine* e, void* out_t, const void* in_q, void* workspace, void* stream);

/* ---- BFV homomorphic multiplication kernel chain (basis extension Q -> Q u B, DGT
 *      tensor product, HPS t/Q scaling back to Q):
 *      (c0, c1, c2) = round(t/Q * (a0 + a1 s)(b0 + b1 s)) in Q, all DGT domain.
 *      cp_bfv_mul is the plain per-call composition of the calls above, in cuPoly's
 *      order (src/arithmetic/polynomial.cu:350-527, 951-999). ---- */
int cp_bfv_mul(const cp_engine* e, void* c0, void* c1, void* c2, const void* a0, const void* a1, const void* b0,
               const void* b1, void* workspace, void* stream);
/* cp_bfv_mul without a caller workspace, for callers that cannot allocate
 * device memory on this path (a runtime that reserves all HBM up front and
 * forbids later allocation, code that must not take cudaMalloc's implicit
 * synchronisation, a plugin host with no allocator).  No counterpart in
 * cuPoly.  Scratch is a static device array of CP_NOALLOC_SCRATCH_BYTES inside
 * the library, present on a GPU from the first use of the library's device
 * code there until exit; parameter sets needing more (cp_workspace_bytes(e) >
 * CP_NOALLOC_SCRATCH_BYTES, e.g. nphi 16384 with k = 10) return
 * CP_ERR_UNSUPPORTED.  The current device must be the engine's
 * (CP_ERR_INVALID otherwise).  The first call on a device is a warm-up: it may
 * load the library's device code (and with it the array) and looks up the
 * array's device address, so make it before any stream capture and before the
 * part of the program that must not allocate.  All calls share the array:
 * calls that overlap on the GPU race; serialise them.  Calls after the first
 * allocate nothing (no cudaMalloc/cudaFree). */
#define CP_NOALLOC_SCRATCH_BYTES ((size_t)8 << 20)
int cp_bfv_mul_noalloc(const cp_engine* e, void* c0, void* c1, void* c2, const void* a0, const void* a1,
                       const void* b0, const void* b1, void* stream);
/* Batched form of the same chain: npairs ciphertext pairs per call, each input
 * uint64_t[npairs][k][N][2] (DGT domain), output c = uint64_t[3][npairs][k][N][2]
 * (c0 of every pair, then c1, then c2).  No counterpart in cuPoly (one
 * parameter set and one polynomial per call there). */
size_t cp_bfv_mul_batch_workspace_bytes(const cp_engine* e, int npairs);
int cp_bfv_mul_batch(const cp_engine* e, void* c, const void* a0, const void* a1, const void* b0, const void* b1,
                     int npairs, void* workspace, void* stream);

/* ---- integer-throughput calibration (no counterpart in cuPoly): times `iters`
 *      x 8 independent applications per thread of one primitive over nthreads
 *      threads (a multiple of 256) and returns the kernel time in *ms.  kind:
 *      0 Shoup constant multiply, 1 data x data modular multiply, 2 modular add,
 *      3 32-bit multiply-add.  sink: nthreads uint64 of device memory. ---- */
int cp_calibrate_int(int kind, int iters, void* sink, long long nthreads, float* ms, void* stream);

/* ---- the modular primitives, elementwise (no counterpart in cuPoly's API; its tests call the
 *      device functions directly: TestDGT.{mod, addmod, submod, mulmod, powmod, GIAdd, GISub,
 *      GIMul}, tests/unit_tests/test_bfv_mode.cu:243-438).  Device arrays of n words (GI ops:
 *      n elements of two words); p odd, 3 <= p < 2^63.  Operand ranges as the kernels use them:
 *      ADD / SUB a, b < p; NEG a < p; MULMOD a < p, any b; SHOUP any a, b < p,
 *      c = floor(b 2^64 / p); RED128 (a = high word, b = low word) < min(2^127, p 2^64);
 *      POW a < p, exponent b; GIMUL a, b < p; GIMUL_CONST3 a < p, b < p the constant, c three Shoup
 *      companions per element of (w_re, w_im - w_re, w_re + w_im). ---- */
enum cp_modop {
  CP_MODOP_ADD = 0, CP_MODOP_SUB = 1, CP_MODOP_NEG = 2, CP_MODOP_MULMOD = 3, CP_MODOP_SHOUP = 4,
  CP_MODOP_RED128 = 5, CP_MODOP_POW = 6, CP_MODOP_GIMUL = 7, CP_MODOP_GIMUL_CONST3 = 8
};
int cp_modarith_eval(int op, const uint64_t* a, const uint64_t* b, const uint64_t* c, uint64_t* out, long long n,
                     uint64_t p, void* stream);

/* ---- CKKS operations (CKKS engines only), DGT domain in and out, level l in [0, k)
 *      (rescale: [1, k)); Q_l = q_0 ... q_l.  They replace fast_conv_Q_to_B /
 *      fast_conv_B_to_Q / ckks_rescale / xi_ckks_rns_rid / rho_ckks_rns_rid
 *      (src/cuda/cudaengine.cu:800-981, 1086-1184) and poly_approx_basis_raising_Q_to_QB /
 *      poly_approx_basis_reduction_QB_to_Q / poly_ckks_rescale / poly_xi_ckks /
 *      poly_rho_ckks (src/arithmetic/polynomial.cu:530-608, 696-800).
 *  raising:   out_qb Q part = in_q; B part y_j = sum_{i<=l} [x_i (Q_l/q_i)^-1]_{q_i} (Q_l/q_i) mod b_j.
 *  reduction: out_q residues i <= l: (x_i - sum_j [y_j (B/b_j)^-1]_{b_j} (B/b_j)) B^-1 mod q_i;
 *             residues above l are not written.
 *  rescale:   in place on a and b (b may be NULL): x_i <- (x_i - x_l) q_l^-1 mod q_i for i < l;
 *             residues l and above are left as they were.
 *  xi / rho:  out_i = x_i B^-1 mod q_i / x_i B mod q_i over the Q residues.
 *  `workspace` holds cp_workspace_bytes(e) bytes of device memory. ---- */
int cp_ckks_modulus_raising(const cp_engine* e, void* out_qb, const void* in_q, int level, void* workspace,
                            void* stream);
int cp_ckks_modulus_reduction(const cp_engine* e, void* out_q, const void* in_qb, int level, void* workspace,
                              void* stream);
int cp_ckks_rescale(const cp_engine* e, void* a, void* b, int level, void* stream);
/* Batched forms of the three calls above (no counterpart in cuPoly, one polynomial per call
 * there): npolys polynomials back to back (in_q / out_q over Q, in_qb / out_qb over QB, x over Q,
 * rescaled in place), same definitions per polynomial; the workspace holds
 * cp_ckks_batch_workspace_bytes(e, npolys) bytes; at most 65535 polynomials per call. */
size_t cp_ckks_batch_workspace_bytes(const cp_engine* e, int npolys);
int cp_ckks_modulus_raising_batch(const cp_engine* e, void* out_qb, const void* in_q, int level, int npolys,
                                  void* workspace, void* stream);
int cp_ckks_modulus_reduction_batch(const cp_engine* e, void* out_q, const void* in_qb, int level, int npolys,
                                    void* workspace, void* stream);
int cp_ckks_rescale_batch(const cp_engine* e, void* x, int npolys, int level, void* stream);
int cp_ckks_xi(const cp_engine* e, void* out, const void* in, void* stream);
int cp_ckks_rho(const cp_engine* e, void* out, const void* in, void* stream);

/* ---- coefficient I/O on the device: replaces the host NTL conversions poly_crt /
 *      poly_icrt (src/arithmetic/polynomial.cu:190-296).  Coefficients are unsigned
 *      integers of nlimbs 64-bit limbs, least significant first, coefficient-major:
 *      uint64_t[npolys][nphi][nlimbs] in device memory.  Residues are in the
 *      coefficient domain, uint64_t[npolys][nres][N][2].
 *      cp_crt: base Q, B or QB, 1 <= nlimbs <= 64, residue = coefficient mod q_r.
 *      cp_icrt: base Q or B (the unique X in [0, prod) with those residues, nlimbs >=
 *      residues of the base) or T (the residue itself). ---- */
int cp_crt(const cp_engine* e, void* out, const uint64_t* coefs, int nlimbs, int base, int npolys, void* stream);
int cp_icrt(const cp_engine* e, uint64_t* coefs, int nlimbs, const void* in, int base, int npolys, void* stream);

/* ---- binary residue wire format: replaces the string forms poly_export_residues /
 *      poly_import_residues (src/arithmetic/polynomial.cu:1291-1383) for the serving
 *      front-end.  Layout: a 64-byte header of sixteen little-endian uint32 words
 *      {magic, version, nphi, nres, base, npolys, domain (0 coefficient, 1 DGT), flags
 *      (0), 8 reserved zero words}, then the nres primes (uint64), then the residues in
 *      the device layout uint64_t[npolys][nres][N][2].  Import checks the header, the
 *      primes, the size and that every residue is reduced, before any copy. ---- */
#define CP_WIRE_MAGIC 0x53525043u /* "CPRS" */
#define CP_WIRE_VERSION 1u
size_t cp_wire_bytes(const cp_engine* e, int base, int npolys);
int cp_export_residues(const cp_engine* e, void* host_out, size_t cap, const void* poly, int base, int npolys,
                       int domain, void* stream);
int cp_import_residues(const cp_engine* e, void* poly, const void* host_in, size_t size, int base, int npolys,
                       int* domain_out, void* stream);

/* ---- sampler: replaces Sampler::sample(ctx, p, kind) (src/cuda/sampler.cu:576-645).
 *      On a CKKS engine CP_NARROW is uniform {-1, 0, +1} and CP_DISCRETE_GAUSSIAN is
 *      nearbyint(3.2 Z) signed, as in cuPoly's CKKS build (sampler.cu:73-106, 459-493).
 *      npolys consecutive polynomials over `base` with stream ids stream_id ..
 *      stream_id + npolys - 1; to_dgt != 0 applies the forward DGT (cuPoly does). */
int cp_sample(const cp_engine* e, void* out, int base, int kind, uint64_t seed, uint32_t stream_id, int npolys,
              int to_dgt, void* stream);
/* Same, polynomial i drawn with stream id stream_ids[i] (a device array), so a
 * batch can hold requests whose operands have unrelated identities. */
int cp_sample_ids(const cp_engine* e, void* out, int base, int kind, uint64_t seed, const uint32_t* stream_ids,
                  int npolys, int to_dgt, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CUPOLY_B200_H */
