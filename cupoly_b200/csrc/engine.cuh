// Internal engine state: parameters and device-resident tables of one
// (nphi, k, kl, t) instance.
//
// Replaces cuPoly's process-wide singletons CUDAEngine / DGTEngine and their
// __constant__ tables (cuPoly src/cuda/cudaengine.cu:22-101,
// src/cuda/dgt.cu:20-33, precompute :1337-1673 and dgt.cu:1694-1982).  Each
// engine owns its own tables, so any number of parameter sets coexist.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "modarith.cuh"

namespace cpoly {

constexpr int kMaxLogNc = 13;   // largest transform kept whole in one CTA (8192 GIs, 136 KB smem)
constexpr int kMaxPasses = 8;
constexpr int kMaxResidues = 96; // |Q| + |B| limit of one engine
constexpr int kMaxLimbs = 64;    // 64-bit limbs of a big-integer coefficient in cp_crt (4096 bits)

// Radix plan of the in-CTA transform of size 2^logNc.  Passes run from the
// top index bits down; pass i covers bits [p[i], p[i] + w[i]).
struct DgtPlan {
  int logN = 0;     // full transform size (N = nphi / 2)
  int logNc = 0;    // size handled inside one CTA
  int S = 0;        // split bits handled by the element-wise split stage
  int cluster = 0;  // 1: run the split stage inside a 2^S-CTA thread-block cluster through
                    // distributed shared memory (no separate HBM pass) when compiled for the plan
  int logR = 0;     // register radix
  int npass = 0;
  int w[kMaxPasses] = {0};
  int p[kMaxPasses] = {0};
};

// logCta caps the size kept whole in one CTA (0: kMaxLogNc); the rest of the
// transform (at most 2 bits) runs in the element-wise split stage.
DgtPlan make_plan(int logN, int logR, int logCta = 0);

// Offsets (in 16-byte entries) inside one residue's table block.
struct DgtTableLayout {
  int off_rad = 0;                      // R entries: w_R^j (w, w')
  int off_fwd[kMaxPasses] = {0};        // per pass: 2^(p+w) entries
  int off_inv[kMaxPasses] = {0};
  int off_split_fwd = 0;                // N entries (only if S > 0)
  int off_split_inv = 0;
  int off_twist = 0;                    // 3N entries: xi^n as (re, im - re, re + im), Shoup pairs
  int off_untwist = 0;                  // 3N entries: xi^-n N^-1, same form
  // 3N entries each: xi^-n N^-1 times a per-residue factor, so that an inverse transform
  // also applies the first constant product of the base conversion that reads its output
  // (BFV engines; used by the batched multiplication chain):
  //   [0]: Q residue i: (Q/q_i)^-1 mod q_i;  B residue j: t Q^-1 (B/b_j)^-1 mod b_j;
  //   [1]: Q residue i: t (Q/q_i)^-1 mod q_i;  B residue j: 1.
  int off_untwist_pre[2] = {0, 0};
  int stride = 0;                       // entries per residue block
};

// Arguments of the DGT kernels (passed by value).
struct DgtArgs {
  const ulonglong2* tab;   // table block of residue 0 of the engine
  int stride;              // entries per residue block
  DgtTableLayout L;
  const ModConst* mc;      // per engine residue
  const int* rid_list;     // work list: residue i of the data uses engine prime rid_list[i] (nullptr: base order)
};

// Where the inverse DGT reads its input.
//  mode 0: p[0] (same layout as the output; p[0] == output for in place);
//  mode 1: the BFV tensor product of two ciphertexts (a0, a1) x (b0, b1) =
//          p[0..3], computed while loading; output polynomial j * npairs + q
//          is c_j of pair q: c0 = a0 b0, c1 = a0 b1 + a1 b0, c2 = a1 b1;
//  mode 2: gather: output polynomial j * npairs + q reads polynomial q of p[j];
//  mode 3: product: the Gaussian product p[0] * p[1] (both in the output's
//          layout), formed while loading -- pointwise multiply fused into the
//          inverse transform.
// `untwist` picks the untwist table of the inverse: 0 the plain xi^-n N^-1, 1 or 2
// off_untwist_pre[untwist - 1].
struct InvSrc {
  const ulonglong2* p[4];
  int mode;
  int npairs;
  int untwist;
};

// Mixed-radix conversion constants of one (source base -> targets) pair.
// Source base: n primes s_0..s_{n-1}; targets: K moduli m_0..m_{K-1}.
struct MrcTables {
  int n = 0, K = 0;
  // inv[i*(i-1)/2 + l] = s_l^-1 mod s_i (and companion), l < i
  std::vector<uint64_t> inv, inv_s;
  // horner[j*n + i] = s_i mod m_j (and companion), i < n - 1
  std::vector<uint64_t> hor, hor_s;
  // digits of (prod(s) - 1) / 2, for the centred lift
  std::vector<uint64_t> half_digits;
  // prod(s) mod m_j (and companion)
  std::vector<uint64_t> P_mod, P_mod_s;
};

struct Engine {
  int device = 0;
  int nphi = 0, N = 0, logN = 0;
  int k = 0, kl = 0;
  uint64_t t = 0;
  std::vector<uint64_t> primes;   // Q then B
  std::vector<uint64_t> roots;    // a primitive root of each prime
  int ckks_prec = 0;              // 0: BFV engine (63-bit primes); 45/48/52/55: CKKS precision bucket
  std::vector<ModConst> mconst;
  std::vector<std::pair<uint64_t, uint64_t>> xi;  // Gaussian root of i used for the twist, per residue
  DgtPlan plan;
  DgtTableLayout layout;
  // Small-launch plan: a launch of at most narrow_units residue transforms (polynomials x
  // residues) uses plan_narrow / layout_narrow instead (0: no such plan).  With few residues
  // per launch, one CTA per residue leaves most SMs idle; a plan whose split stage spreads
  // each residue over 2-4 CTAs finishes sooner.  Its radix, pass and split tables follow the
  // main plan's in each residue block; the twist tables are shared.
  DgtPlan plan_narrow;
  DgtTableLayout layout_narrow;
  long long narrow_units = 0;

  // device allocations
  ModConst* d_mc = nullptr;
  ulonglong2* d_tab = nullptr;     // (k + kl) residue blocks
  uint64_t* d_hps = nullptr;       // packed HPS/MRC constants
  size_t hps_words = 0;
  // word offsets inside d_hps
  struct HpsOffsets {
    int qb_inv, qb_inv_s, qb_hor, qb_hor_s, qb_half;           // Q -> B
    int q_lift, b_lift;  // MRC digits of T - 1, T = S - floor(S FPERROR): the lift threshold of Q, of B
    int bq_inv, bq_inv_s, bq_hor, bq_hor_s;                    // B -> Q
    int qt_hor, qt_hor_s;                                      // Q -> t
    int q_mod_b, q_mod_b_s;        // Q mod b_j
    int qinv_b, qinv_b_s;          // Q^-1 mod b_j
    int t_q, t_q_s;                // t mod q_i
    int t_b, t_b_s;                // t mod b_j
    int q_mod_t, q_mod_t_s;        // Q mod t
    int qinv_t, qinv_t_s;          // Q^-1 mod t
    int xi_q, xi_q_s;              // (Q/q_i)^-1 mod q_i
    int rho_q, rho_q_s;            // (Q/q_i) mod q_i
    int qb_pm, bq_pm;              // mixed-radix weights prod_{l<i} s_l mod m_j, [target][i]
    int qq_w, bb_w;                // Garner weights of Q and of B, [i][l]
    int q_pinv, q_pinv_s, b_pinv, b_pinv_s;  // (prod_{j<i} s_j)^-1 mod s_i
    // fast base conversion (FP64 overflow count, exact fallback): S = prod of the source base
    int fq_hinv, fq_hinv_s;        // (Q/q_i)^-1 mod q_i, [i]
    int fq_thinv, fq_thinv_s;      // t (Q/q_i)^-1 mod q_i, [i] (complex scaling)
    int fq_hmod;                   // (Q/q_i) mod b_j, [j][i]
    int fq_negv;                   // (-v Q) mod b_j, [j][v], v in [0, k]
    int fq_invd;                   // 1/q_i as IEEE-754 double bits, [i]
    int fb_hinv, fb_hinv_s;        // (B/b_j)^-1 mod b_j, [j]
    int fb_hmod;                   // (B/b_j) mod q_i, [i][j]
    int fb_negv;                   // (-v B) mod q_i, [i][v], v in [0, kl]
    int fb_invd;                   // 1/b_j as double bits, [j]
    // conversions of prescaled inputs (the untwist tables off_untwist_pre); the recovery
    // factors undo the prescaling for coefficients that take the exact path
    int fq_trec, fq_trec_s;        // (t (Q/q_i)^-1)^-1 mod q_i, [i]
    int fb_rec, fb_rec_s;          // (B/b_j) mod b_j, [j]
    int cs_brec, cs_brec_s;        // (t Q^-1 (B/b_j)^-1)^-1 mod b_j, [j]
    int cs_hm2;                    // q_i^-1 (B/b_j)^-1 mod b_j, [j][i]
    int cs_negw2;                  // (-w (B/b_j)^-1) mod b_j, [j][w], w in [0, k]
    int pow64;                     // 2^(64 l) mod p_r, [residue][kMaxLimbs]
    int pow64m;                    // 2^(64 (l + 1)) mod p_r (Montgomery form of pow64), same shape
    // CKKS (only when ckks_prec != 0); every constant with its Shoup companion
    int ck_inv_ql, ck_inv_ql_s;    // q_l^-1 mod q_i, [l][i]
    int ck_qlqi_inv, ck_qlqi_inv_s;  // (Q_l / q_i)^-1 mod q_i, [l][i]; Q_l = q_0 ... q_l
    int ck_qlqi_b, ck_qlqi_b_s;    // (Q_l / q_i) mod b_j, [l][i][j]
    int ck_bbj_inv, ck_bbj_inv_s;  // (B / b_j)^-1 mod b_j, [j]
    int ck_bbj_q, ck_bbj_q_s;      // (B / b_j) mod q_i, [j][i]
    int ck_binv_q, ck_binv_q_s;    // B^-1 mod q_i, [i]
    int ck_b_q, ck_b_q_s;          // B mod q_i, [i]
  } ho{};
  uint64_t t_shoup_one = 0;        // floor(2^64 / t)
  uint64_t h_q_mod_t = 0, h_qinv_t = 0, h_qinv_t_s = 0;  // Q mod t, Q^-1 mod t
  int* d_err = nullptr;            // device-side error flag (sampler rejection exhaustion)
  int hps_force_exact = 0;         // 1: every base conversion and scaling takes its exact path (tests)

  int n_residues(int base) const;
  int rid_offset(int base) const;
};

// thread-local error reporting
void set_error(const std::string& msg);
const char* last_error();

// table construction (tables.cu)
int build_tables(Engine& e);
void free_tables(Engine& e);

}  // namespace cpoly

// The C ABI's opaque handle (include/cupoly_b200.h): one engine.
struct cp_engine {
  cpoly::Engine e;
};
