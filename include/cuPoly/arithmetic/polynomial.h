// cuPoly's polynomial API (include/cuPoly/arithmetic/polynomial.h:39-626) in C++
// over the cupoly_b200 C ABI (include/cupoly_b200.h).
//
// poly_t keeps cuPoly's fields and lazy host/device state machine: `coefs`
// (host, NTL-style ZZ) is current in HOSTSTATE / BOTHSTATE, `d_coefs` (device,
// DGT domain, GaussianInteger[nres][N]) in RNSSTATE / BOTHSTATE.  Operations
// run on the device in the DGT domain and leave their outputs in RNSSTATE;
// coefficient reads recombine on the device (cp_icrt) and synchronise the
// context's stream.  Differences from cuPoly:
//  * errors throw std::runtime_error (cuPoly: assert / exit(1));
//  * every d_coefs buffer is allocated for a QB polynomial, so a poly_t can
//    change base (e.g. as the output of a basis extension) without reallocation;
//  * HPS scaling is exact round(t X / Q) for every input (cuPoly's float path is
//    within 1); base conversions lift X within FPERROR of the modulus to X - S as
//    cuPoly does, decided exactly (cuPoly decides it in double precision);
//  * poly_complex_scaling_tDivQ leaves its inputs unchanged (cuPoly
//    inverse-transforms them in place);
//  * poly_are_equal compares every coefficient up to the degree (cuPoly skips
//    the top one), and poly_get_residues writes residue i at offset i * nphi;
//  * poly_norm_2 (an NTL RR) is not provided; poly_set_nth_cyclotomic and
//    poly_change_repr, declared by cuPoly but defined nowhere, are left out.
#ifndef POLYNOMIAL_H
#define POLYNOMIAL_H
#include <NTL/ZZ.h>
#include <cuPoly/settings.h>
#include <cuPoly/tool/log.h>

#include <string>
#include <vector>

NTL_CLIENT

class Context;

enum poly_states {
  HOSTSTATE,  // host coefficients current, device data may be stale
  RNSSTATE,   // device data current, host coefficients may be stale
  BOTHSTATE   // both current
};

struct polynomial {
  bool init = false;
  std::vector<NTL::ZZ> coefs;
  GaussianInteger* d_coefs = NULL;
  int status = BOTHSTATE;
  int base = QBase;
};
typedef struct polynomial poly_t;

size_t poly_get_residues_size(int base);
void poly_init(Context* ctx, poly_t* a, int base = QBase);
void poly_free(Context* ctx, poly_t* a);
void poly_clear(Context* ctx, poly_t* a);
void poly_copy_to_device(Context* ctx, poly_t* a);
void poly_copy_to_host(Context* ctx, poly_t* a);
void poly_copy(Context* ctx, poly_t* b, poly_t* a);
// Coefficient-domain residues of a's host coefficients, computed on the device
// into the context's aux buffer (device pointer; cuPoly returns a host array).
GaussianInteger* poly_crt(Context* ctx, poly_t* a);
// a->coefs <- the unique X in [0, prod) with a's residues (Q, B or T base).
void poly_icrt(Context* ctx, poly_t* a);
int poly_get_deg(Context* ctx, poly_t* a);

void poly_add(Context* ctx, poly_t* c, poly_t* a, poly_t* b);
void poly_double_add(Context* ctx, poly_t* c1, poly_t* a1, poly_t* b1, poly_t* c2, poly_t* a2, poly_t* b2);
void poly_sub(Context* ctx, poly_t* c, poly_t* a, poly_t* b);
void poly_mul(Context* ctx, poly_t* c, poly_t* a, poly_t* b);
void poly_mul_add(Context* ctx, poly_t* d, poly_t* a, poly_t* b, poly_t* c);
void poly_dr2(Context* ctx, poly_t* ct21, poly_t* ct22, poly_t* ct23, poly_t* ct01, poly_t* ct02, poly_t* ct11,
              poly_t* ct12);
void poly_mul_int(Context* ctx, poly_t* c, poly_t* a, uint64_t x);
void poly_double_mul_int(Context* ctx, poly_t* b1, poly_t* a1, poly_t* b2, poly_t* a2, uint64_t x1, uint64_t x2);
void poly_double_add_int(Context* ctx, poly_t* b1, poly_t* a1, poly_t* b2, poly_t* a2, uint64_t x1, uint64_t x2);
void poly_add_int(Context* ctx, poly_t* c, poly_t* a, uint64_t x);
void poly_sub_int(Context* ctx, poly_t* c, poly_t* a, uint64_t x);
void poly_div_by_ZZ(Context* ctx, poly_t* c, poly_t* a, NTL::ZZ x);
void poly_mod_by_ZZ(Context* ctx, poly_t* c, poly_t* a, NTL::ZZ x);
void poly_negate(Context* ctx, poly_t* a);
void poly_right_shift(Context* ctx, poly_t* b, poly_t* a, int bits);
void poly_dot(Context* ctx, poly_t* c, poly_t* a, poly_t* b, const int k);

// HPS (BFV): b (T) = round(t a / Q) mod t; b (Q) = round(t X / Q) for X given by a_Q, a_B.
void poly_simple_scaling_tDivQ(Context* ctx, poly_t* b, poly_t* a);
void poly_complex_scaling_tDivQ(Context* ctx, poly_t* b, poly_t* a_Q, poly_t* a_B);
void poly_basis_extension_Q_to_B(Context* ctx, poly_t* a_B, poly_t* a_Q);
void poly_basis_extension_Q_to_QB(Context* ctx, poly_t* b, poly_t* a);
void poly_basis_extension_B_to_Q(Context* ctx, poly_t* a_Q, poly_t* a_B);
// Key-switching decomposition (BFV): c is an array of k poly_t; c[i] holds
// residue i of a times (Q / q_i)^-1 (xi) or Q / q_i (rho), the other residues zero.
void poly_xi_bfv(Context* ctx, poly_t* c, poly_t* a);
void poly_rho_bfv(Context* ctx, poly_t* c, poly_t* a);

// CKKS (engines made with init_ckks / CKKS_ENGINE_MODE).
void poly_approx_basis_raising_Q_to_QB(Context* ctx, poly_t* a, poly_t* b, int level);
void poly_approx_basis_reduction_QB_to_Q(Context* ctx, poly_t* a, poly_t* b, int level);
void poly_ckks_rescale(Context* ctx, poly_t* a, poly_t* b, int level = 1);
void poly_xi_ckks(Context* ctx, poly_t* c, poly_t* a);
void poly_rho_ckks(Context* ctx, poly_t* c, poly_t* a);

std::string poly_to_string(Context* ctx, poly_t* a);
void poly_set_coeff(Context* ctx, poly_t* a, unsigned int index, NTL::ZZ c);
NTL::ZZ poly_get_coeff(Context* ctx, poly_t* a, int index);
bool poly_are_equal(Context* ctx, poly_t* a, poly_t* b);
NTL::ZZ poly_infty_norm(Context* ctx, poly_t* p);

// Text forms (cuPoly polynomial.cu:1291-1437) and the binary wire form of the C ABI.
std::string poly_export(Context* ctx, poly_t* p);
poly_t* poly_import(Context* ctx, std::string v);
std::string poly_export_residues(Context* ctx, poly_t* p);
poly_t* poly_import_residues(Context* ctx, std::string v, int base = QBase);
std::vector<unsigned char> poly_export_binary(Context* ctx, poly_t* p);
poly_t* poly_import_binary(Context* ctx, const std::vector<unsigned char>& data, int base = QBase);

// Residue access (coefficient domain, host): residue `id` as nphi words.
std::string poly_residue_to_string(Context* ctx, poly_t* a, int id);
uint64_t* poly_get_residue(Context* ctx, uint64_t* b, poly_t* a, int id);
uint64_t* poly_get_residues(Context* ctx, poly_t* a);  // malloc'd, nres x nphi words
void poly_select_residue(Context* ctx, poly_t* p, int id);
void poly_discard_qbase(Context* ctx, poly_t* p);

#include <cuPoly/arithmetic/context.h>
#include <cuPoly/cuda/cudaengine.h>
#include <cuPoly/cuda/dgt.h>
#endif
