// C ABI (include/cupoly_b200.h): argument checking, engine lifecycle and the
// composite polynomial calls built from the kernels.
#include <cstring>
#include <new>

#include "../../include/cupoly_b200.h"
#include "launch.cuh"
#include "pointwise.cuh"
#include "prime_table.h"
#include "prime_table_ckks.h"


using namespace cpoly;

namespace {

cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

bool valid_base(const cp_engine* e, int base) { return e && base >= 0 && base <= 3; }

#define CP_REQUIRE(cond, msg)      \
  do {                             \
    if (!(cond)) {                 \
      set_error(msg);              \
      return CP_ERR_INVALID;       \
    }                              \
  } while (0)

// The exact BFV base conversions and scalings need the 63-bit prime form.
#define CP_BFV_ONLY(h, name)                                                     \
  do {                                                                           \
    if ((h) && (h)->e.ckks_prec) {                                               \
      set_error(name ": not available on a CKKS engine (BFV base conversions)"); \
      return CP_ERR_UNSUPPORTED;                                                 \
    }                                                                            \
  } while (0)

// canonical xi with xi^N = i (see cp_engine_set_nthroot)
std::pair<uint64_t, uint64_t> canonical_xi(uint64_t p, uint64_t g, uint64_t N) {
  const uint64_t s = h_powmod(g, (p - 1) / 4, p);
  const uint64_t u = h_powmod(g, (p - 1) / (4 * N), p);
  const uint64_t ui = h_invmod(u, p);
  const uint64_t inv2 = (p + 1) / 2;
  const uint64_t re = h_mulmod((u + ui) % p, inv2, p);
  const uint64_t im = h_mulmod(h_mulmod((u + p - ui) % p, inv2, p), h_invmod(s, p), p);
  return {re, im};
}

size_t ws_elems(const Engine& e) { return (size_t)(5 * e.k + 10 * e.kl) * e.N; }

}  // namespace

extern "C" {

const char* cp_version(void) { return "cupoly_b200 0.1.0 (sm_100a)"; }
const char* cp_last_error(void) { return last_error(); }

}  // extern "C"

namespace {

// build_tables with host allocation failures turned into a status (no exception may cross
// the C ABI).
int build_tables_nothrow(Engine& e) {
  try {
    return build_tables(e);
  } catch (const std::bad_alloc&) {
    set_error("engine tables: host allocation failed");
    return CP_ERR_OOM;
  } catch (...) {
    set_error("engine tables: unexpected host error");
    return CP_ERR_INVALID;
  }
}

// Shared tail of the two creation calls: tables for the given primes.
int finish_engine(cp_engine** out, cp_engine* h, int log_radix) {
  Engine& e = h->e;
  for (size_t i = 0; i < e.primes.size(); ++i) {
    const uint64_t p = e.primes[i];
    e.mconst.push_back(h_modconst(p));
    if ((p - 1) % (2 * (uint64_t)e.nphi) != 0) {  // xi is a root of unity of order 2 nphi
      delete h;
      set_error("engine create: a prime of the bases has no root of unity of order 2 nphi");
      return CP_ERR_UNSUPPORTED;
    }
    e.xi.push_back(canonical_xi(p, e.roots[i], (uint64_t)e.N));
  }
  // Default main plan, the fastest measured on B200 (forward + inverse of 2048 residues): the
  // whole transform in one CTA up to N = 4096; from N = 8192 on, the top 2 bits in the split
  // stage (nphi 16384: 0.969 ms against 1.030 ms whole; nphi 32768: 2.082 against 2.312 ms
  // with 1 split bit).
  e.plan = make_plan(e.logN, log_radix ? log_radix : 3, e.logN >= 13 ? e.logN - 2 : kMaxLogNc);
  // Default small-launch plan: radix 4 over 2^(log N - 2) elements per CTA, the top 2 bits in
  // the split stage.  Where the main plan keeps more of the transform in one CTA (N = 2048 and
  // 4096) it takes launches of up to 96 residue transforms: a single BFV multiplication went
  // from 133 to 77 us at nphi 8192.  At N = 8192, where the main plan has the same split, only
  // launches of up to 16 (0.027 against 0.031 ms at 16, slower from 96 on); none above.
  // cp_engine_set_narrow_plan replaces or removes it.
  if (e.logN >= 11 && e.logN - 2 < e.plan.logNc) {
    e.plan_narrow = make_plan(e.logN, 2, e.logN - 2);
    e.narrow_units = 96;
  } else if (e.logN == 13 && e.plan.logR != 2) {
    e.plan_narrow = make_plan(e.logN, 2, e.logN - 2);
    e.narrow_units = 16;
  }
  int rc = build_tables_nothrow(e);
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return CP_OK;
}

cp_engine* new_engine(int k, int kl, int nphi, uint64_t t) {
  cp_engine* h = new (std::nothrow) cp_engine();
  if (!h) {
    set_error("engine create: host allocation failed");
    return nullptr;
  }
  Engine& e = h->e;
  cudaGetDevice(&e.device);
  e.k = k;
  e.kl = kl;
  e.nphi = nphi;
  e.N = nphi / 2;
  e.logN = 0;
  while ((1 << e.logN) < e.N) ++e.logN;
  e.t = t;
  return h;
}

}  // namespace

extern "C" {

int cp_engine_create(cp_engine** out, int k, int kl, int nphi, uint64_t t, int log_radix) {
  CP_REQUIRE(out, "cp_engine_create: out is NULL");
  *out = nullptr;
  if (kl <= 0) kl = k + 1;
  CP_REQUIRE(k >= 1 && k <= 24, "cp_engine_create: k must be in [1, 24]");
  CP_REQUIRE(kl >= 1 && kl <= 24, "cp_engine_create: kl must be in [1, 24]");
  CP_REQUIRE(k + kl <= kNumPrimes, "cp_engine_create: k + kl exceeds the prime table");
  CP_REQUIRE(nphi >= 4 && nphi <= 65536 && (nphi & (nphi - 1)) == 0,
             "cp_engine_create: nphi must be a power of two in [4, 65536]");
  CP_REQUIRE(t >= 2 && t < kPrimes[kNumPrimes - 1], "cp_engine_create: t must be in [2, min prime)");
  CP_REQUIRE(log_radix == 0 || (log_radix >= 2 && log_radix <= 4), "cp_engine_create: log_radix must be 0, 2, 3 or 4");
  cp_engine* h = new_engine(k, kl, nphi, t);
  if (!h) return CP_ERR_OOM;
  Engine& e = h->e;
  for (int i = 0; i < k + kl; ++i) {
    const uint64_t p = kPrimes[i];
    // the BFV base conversions rely on 2^64 mod p < 2^32 and p = 2^63 - c, c < 2^31 - 1
    if ((uint64_t)(((unsigned __int128)1 << 64) % p) >> 32 || (p >> 63) || (1ull << 63) - p >= (1ull << 31) - 1) {
      delete h;
      set_error("cp_engine_create: prime outside the supported 63-bit form");
      return CP_ERR_UNSUPPORTED;
    }
    e.primes.push_back(p);
    e.roots.push_back(kPrimitiveRoots[i]);
  }
  return finish_engine(out, h, log_radix);
}

int cp_ckks_engine_create(cp_engine** out, int k, int kl, int nphi, int prec, int log_radix) {
  CP_REQUIRE(out, "cp_ckks_engine_create: out is NULL");
  *out = nullptr;
  if (kl <= 0) kl = k + 1;
  CP_REQUIRE(prec == 45 || prec == 48 || prec == 52 || prec == 55,
             "cp_ckks_engine_create: prec must be 45, 48, 52 or 55");
  CP_REQUIRE(k >= 1 && k <= 24, "cp_ckks_engine_create: k must be in [1, 24]");
  CP_REQUIRE(kl >= 1 && kl <= 24, "cp_ckks_engine_create: kl must be in [1, 24]");
  CP_REQUIRE(nphi >= 4 && nphi <= 65536 && (nphi & (nphi - 1)) == 0,
             "cp_ckks_engine_create: nphi must be a power of two in [4, 65536]");
  CP_REQUIRE(log_radix == 0 || (log_radix >= 2 && log_radix <= 4),
             "cp_ckks_engine_create: log_radix must be 0, 2, 3 or 4");
  // Q = the first 63-bit prime, then k - 1 primes of the precision bucket; B = kl primes of
  // the 45-bit (prec 45) or 55-bit bucket from index k - 1 (cuPoly cudaengine.cu:1192-1232)
  const uint64_t* qb = prec == 45 ? kPrimes45 : prec == 48 ? kPrimes48 : prec == 52 ? kPrimes52 : kPrimes55;
  const uint32_t* qr = prec == 45 ? kRoots45 : prec == 48 ? kRoots48 : prec == 52 ? kRoots52 : kRoots55;
  const int qn = prec == 45 ? kNumPrimes45 : prec == 48 ? kNumPrimes48 : prec == 52 ? kNumPrimes52 : kNumPrimes55;
  const uint64_t* bb = prec == 45 ? kPrimes45 : kPrimes55;
  const uint32_t* br = prec == 45 ? kRoots45 : kRoots55;
  const int bn = prec == 45 ? kNumPrimes45 : kNumPrimes55;
  CP_REQUIRE(k - 1 <= qn && k - 1 + kl <= bn, "cp_ckks_engine_create: k, kl exceed the precision bucket");
  cp_engine* h = new_engine(k, kl, nphi, 2);
  if (!h) return CP_ERR_OOM;
  Engine& e = h->e;
  e.ckks_prec = prec;
  e.primes.push_back(kPrimes[0]);
  e.roots.push_back(kPrimitiveRoots[0]);
  for (int i = 0; i < k - 1; ++i) {
    e.primes.push_back(qb[i]);
    e.roots.push_back(qr[i]);
  }
  for (int j = 0; j < kl; ++j) {
    e.primes.push_back(bb[k - 1 + j]);
    e.roots.push_back(br[k - 1 + j]);
  }
  return finish_engine(out, h, log_radix);
}

int cp_engine_ckks_prec(const cp_engine* h) { return h ? h->e.ckks_prec : -1; }

int cp_engine_set_plan(cp_engine* h, int log_radix, int log_cta) {
  CP_REQUIRE(h, "cp_engine_set_plan: NULL engine");
  CP_REQUIRE(log_radix == 0 || (log_radix >= 2 && log_radix <= 4), "cp_engine_set_plan: log_radix must be 0, 2, 3 or 4");
  Engine& e = h->e;
  const int lc = log_cta ? log_cta : kMaxLogNc;
  CP_REQUIRE(lc >= 8 && lc <= kMaxLogNc, "cp_engine_set_plan: log_cta must be 0 or in [8, 13]");
  CP_REQUIRE(e.logN - (e.logN < lc ? e.logN : lc) <= 2, "cp_engine_set_plan: at most 2 split bits (log N - log_cta)");
  cudaDeviceSynchronize();
  free_tables(e);
  const int cluster = e.plan.cluster;  // the split-stage form survives a plan change
  e.plan = make_plan(e.logN, log_radix ? log_radix : 3, lc);
  e.plan.cluster = cluster;
  return build_tables_nothrow(e);
}

int cp_engine_set_narrow_plan(cp_engine* h, int log_radix, int log_cta, long long max_units) {
  CP_REQUIRE(h, "cp_engine_set_narrow_plan: NULL engine");
  CP_REQUIRE(max_units >= 0, "cp_engine_set_narrow_plan: max_units must be >= 0");
  Engine& e = h->e;
  if (max_units > 0) {
    CP_REQUIRE(log_radix == 0 || (log_radix >= 2 && log_radix <= 4),
               "cp_engine_set_narrow_plan: log_radix must be 0, 2, 3 or 4");
    const int lc = log_cta ? log_cta : kMaxLogNc;
    CP_REQUIRE(lc >= 8 && lc <= kMaxLogNc, "cp_engine_set_narrow_plan: log_cta must be 0 or in [8, 13]");
    CP_REQUIRE(e.logN - (e.logN < lc ? e.logN : lc) <= 2,
               "cp_engine_set_narrow_plan: at most 2 split bits (log N - log_cta)");
  }
  cudaDeviceSynchronize();
  free_tables(e);
  if (max_units > 0) {
    e.plan_narrow = make_plan(e.logN, log_radix ? log_radix : 3, log_cta ? log_cta : kMaxLogNc);
    e.plan_narrow.cluster = 0;
  } else {
    e.plan_narrow = DgtPlan{};
  }
  e.narrow_units = max_units;
  return build_tables_nothrow(e);
}

int cp_engine_get_narrow_plan(const cp_engine* h, int* log_radix, int* log_cta, long long* max_units) {
  CP_REQUIRE(h, "cp_engine_get_narrow_plan: NULL engine");
  const Engine& e = h->e;
  if (log_radix) *log_radix = e.narrow_units > 0 ? e.plan_narrow.logR : 0;
  if (log_cta) *log_cta = e.narrow_units > 0 ? e.plan_narrow.logNc : 0;
  if (max_units) *max_units = e.narrow_units;
  return CP_OK;
}

int cp_engine_set_split_mode(cp_engine* h, int mode) {
  CP_REQUIRE(h, "cp_engine_set_split_mode: NULL engine");
  CP_REQUIRE(mode == 0 || mode == 1, "cp_engine_set_split_mode: mode must be 0 (split kernel) or 1 (cluster)");
  cudaDeviceSynchronize();  // transforms in flight keep the form they were launched with
  h->e.plan.cluster = mode;
  return CP_OK;
}

int cp_engine_get_split_mode(const cp_engine* h) { return h ? h->e.plan.cluster : -1; }

int cp_engine_set_hps_force_exact(cp_engine* h, int on) {
  CP_REQUIRE(h, "cp_engine_set_hps_force_exact: NULL engine");
  CP_REQUIRE(on == 0 || on == 1, "cp_engine_set_hps_force_exact: on must be 0 or 1");
  cudaDeviceSynchronize();  // conversions in flight keep the form they were launched with
  h->e.hps_force_exact = on;
  return CP_OK;
}

int cp_engine_get_plan(const cp_engine* h, int* log_radix, int* log_cta, int* split_bits) {
  CP_REQUIRE(h, "cp_engine_get_plan: NULL engine");
  if (log_radix) *log_radix = h->e.plan.logR;
  if (log_cta) *log_cta = h->e.plan.logNc;
  if (split_bits) *split_bits = h->e.plan.S;
  return CP_OK;
}

int cp_engine_destroy(cp_engine* h) {
  if (!h) return CP_OK;
  cudaDeviceSynchronize();
  free_tables(h->e);
  delete h;
  return CP_OK;
}

int cp_engine_n_residues(const cp_engine* h, int base) {
  if (!valid_base(h, base)) {
    set_error("cp_engine_n_residues: bad engine or base");
    return -1;
  }
  return h->e.n_residues(base);
}

int cp_engine_nphi(const cp_engine* h) { return h ? h->e.nphi : -1; }

int cp_engine_primes(const cp_engine* h, uint64_t* out, int capacity) {
  CP_REQUIRE(h && out, "cp_engine_primes: NULL argument");
  const int n = (int)h->e.primes.size();
  CP_REQUIRE(capacity >= n, "cp_engine_primes: capacity too small");
  std::memcpy(out, h->e.primes.data(), n * sizeof(uint64_t));
  return n;
}

int cp_engine_set_nthroot(cp_engine* h, const uint64_t* xi) {
  CP_REQUIRE(h && xi, "cp_engine_set_nthroot: NULL argument");
  Engine& e = h->e;
  const int n = e.k + e.kl;
  std::vector<std::pair<uint64_t, uint64_t>> nx(n);
  for (int r = 0; r < n; ++r) {
    const uint64_t p = e.primes[r];
    nx[r] = {xi[2 * r], xi[2 * r + 1]};
    CP_REQUIRE(nx[r].first < p && nx[r].second < p, "cp_engine_set_nthroot: value not reduced");
    // verify xi^N == i
    uint64_t ar = 1, ai = 0, br = nx[r].first, bi = nx[r].second;
    uint64_t ex = (uint64_t)e.N;
    while (ex) {
      if (ex & 1) {
        const uint64_t nr = (h_mulmod(ar, br, p) + p - h_mulmod(ai, bi, p)) % p;
        const uint64_t ni = (h_mulmod(ar, bi, p) + h_mulmod(ai, br, p)) % p;
        ar = nr;
        ai = ni;
      }
      const uint64_t sr = (h_mulmod(br, br, p) + p - h_mulmod(bi, bi, p)) % p;
      const uint64_t si = 2 * h_mulmod(br, bi, p) % p;
      br = sr;
      bi = si;
      ex >>= 1;
    }
    CP_REQUIRE(ar == 0 && ai == 1, "cp_engine_set_nthroot: xi^N != i for some residue");
  }
  cudaDeviceSynchronize();
  free_tables(e);
  e.xi = nx;
  return build_tables_nothrow(e);
}

int cp_engine_get_nthroot(const cp_engine* h, uint64_t* xi_out) {
  CP_REQUIRE(h && xi_out, "cp_engine_get_nthroot: NULL argument");
  for (size_t r = 0; r < h->e.xi.size(); ++r) {
    xi_out[2 * r] = h->e.xi[r].first;
    xi_out[2 * r + 1] = h->e.xi[r].second;
  }
  return CP_OK;
}

size_t cp_workspace_bytes(const cp_engine* h) { return h ? ws_elems(h->e) * 16 : 0; }

int cp_engine_check(const cp_engine* h, void* stream) {
  CP_REQUIRE(h, "cp_engine_check: NULL engine");
  int flag = 0;
  cudaError_t err = cudaMemcpyAsync(&flag, h->e.d_err, sizeof(int), cudaMemcpyDeviceToHost, S(stream));
  if (err == cudaSuccess) err = cudaStreamSynchronize(S(stream));
  if (err != cudaSuccess) return cuda_fail("cp_engine_check", err);
  if (flag) {
    cudaMemsetAsync(h->e.d_err, 0, sizeof(int), S(stream));
    cudaStreamSynchronize(S(stream));
    set_error("a kernel reported an error (sampler rejection limit reached)");
    return CP_ERR_DEVICE;
  }
  return CP_OK;
}

int cp_engine_check_async(const cp_engine* h, int* flag_host, void* stream) {
  CP_REQUIRE(h && flag_host, "cp_engine_check_async: NULL engine or flag");
  const cudaError_t err = cudaMemcpyAsync(flag_host, h->e.d_err, sizeof(int), cudaMemcpyDeviceToHost, S(stream));
  if (err != cudaSuccess) return cuda_fail("cp_engine_check_async", err);
  return CP_OK;
}

int cp_dgt(const cp_engine* h, void* data, int base, int direction, int npolys, int64_t poly_stride, void* stream) {
  CP_REQUIRE(valid_base(h, base) && data, "cp_dgt: bad engine, base or data");
  CP_REQUIRE(direction == CP_FORWARD || direction == CP_INVERSE, "cp_dgt: bad direction");
  CP_REQUIRE(npolys >= 0 && poly_stride >= 0, "cp_dgt: bad npolys or stride");
  return launch_dgt(h->e, data, base, npolys, poly_stride, direction == CP_INVERSE, S(stream));
}

int cp_dgt_list(const cp_engine* h, void* data, const int* rid_list, int nlist, int direction, void* stream) {
  CP_REQUIRE(h && data && rid_list && nlist >= 0, "cp_dgt_list: bad argument");
  CP_REQUIRE(direction == CP_FORWARD || direction == CP_INVERSE, "cp_dgt_list: bad direction");
  return launch_dgt_list(h->e, data, rid_list, nlist, direction == CP_INVERSE, S(stream));
}

int cp_mul_list(const cp_engine* h, void* c, const void* a, const void* b, const int* rid_list, int nlist,
                void* stream) {
  CP_REQUIRE(h && c && a && b && rid_list && nlist >= 0, "cp_mul_list: bad argument");
  if (nlist == 0) return CP_OK;
  return pw_mul_list(h->e, c, a, b, rid_list, nlist, S(stream));
}

size_t cp_polymul_workspace_bytes(const cp_engine* h, int base, int npolys) {
  if (!valid_base(h, base) || base == CP_TBASE || npolys < 0) return 0;
  return (size_t)2 * npolys * h->e.n_residues(base) * h->e.N * 16;
}

int cp_polymul(const cp_engine* h, void* c, const void* a, const void* b, int base, int npolys, void* workspace,
               void* stream) {
  CP_REQUIRE(valid_base(h, base) && base != CP_TBASE, "cp_polymul: bad engine or base");
  CP_REQUIRE(c && a && b && workspace && npolys >= 0, "cp_polymul: bad argument");
  if (npolys == 0) return CP_OK;
  NvtxRange range("cp_polymul");
  const Engine& e = h->e;
  ulonglong2* wa = reinterpret_cast<ulonglong2*>(workspace);
  ulonglong2* wb = wa + (size_t)npolys * e.n_residues(base) * e.N;
  cudaStream_t st = S(stream);
  if (int rc = launch_dgt_ex(e, wa, a, nullptr, base, npolys, 0, false, st)) return rc;
  if (int rc = launch_dgt_ex(e, wb, b, nullptr, base, npolys, 0, false, st)) return rc;
  InvSrc is{};
  is.p[0] = wa;
  is.p[1] = wb;
  is.mode = 3;
  is.npairs = 1;
  return launch_dgt_ex(e, c, nullptr, &is, base, npolys, 0, true, st);
}

int cp_polymul_list(const cp_engine* h, void* c, const void* a, const void* b, void* wa, void* wb,
                    const int* rid_list, int nlist, void* stream) {
  CP_REQUIRE(h && c && a && b && wa && wb && rid_list && nlist >= 0, "cp_polymul_list: bad argument");
  if (nlist == 0) return CP_OK;
  const Engine& e = h->e;
  cudaStream_t st = S(stream);
  if (int rc = launch_dgt_list_ex(e, wa, a, nullptr, rid_list, nlist, false, st)) return rc;
  if (int rc = launch_dgt_list_ex(e, wb, b, nullptr, rid_list, nlist, false, st)) return rc;
  InvSrc is{};
  is.p[0] = reinterpret_cast<const ulonglong2*>(wa);
  is.p[1] = reinterpret_cast<const ulonglong2*>(wb);
  is.mode = 3;
  is.npairs = 1;
  return launch_dgt_list_ex(e, c, nullptr, &is, rid_list, nlist, true, st);
}

#define PW_CHECK(name) CP_REQUIRE(valid_base(h, base) && base != CP_TBASE, name ": bad engine or base")

int cp_add(const cp_engine* h, void* c, const void* a, const void* b, int base, void* stream) {
  PW_CHECK("cp_add");
  CP_REQUIRE(c && a && b, "cp_add: NULL buffer");
  return pw_add(h->e, c, a, b, base, S(stream));
}
int cp_sub(const cp_engine* h, void* c, const void* a, const void* b, int base, void* stream) {
  PW_CHECK("cp_sub");
  CP_REQUIRE(c && a && b, "cp_sub: NULL buffer");
  return pw_sub(h->e, c, a, b, base, S(stream));
}
int cp_double_add(const cp_engine* h, void* c1, const void* a1, const void* b1, void* c2, const void* a2,
                  const void* b2, int base, void* stream) {
  PW_CHECK("cp_double_add");
  CP_REQUIRE(c1 && a1 && b1 && c2 && a2 && b2, "cp_double_add: NULL buffer");
  return pw_double_add(h->e, c1, a1, b1, c2, a2, b2, base, S(stream));
}
int cp_mul(const cp_engine* h, void* c, const void* a, const void* b, int base, void* stream) {
  PW_CHECK("cp_mul");
  CP_REQUIRE(c && a && b, "cp_mul: NULL buffer");
  return pw_mul(h->e, c, a, b, base, S(stream));
}
int cp_mul_batch(const cp_engine* h, void* c, const void* a, const void* b, int base, int npolys, void* stream) {
  PW_CHECK("cp_mul_batch");
  CP_REQUIRE(c && a && b && npolys >= 0, "cp_mul_batch: bad argument");
  return pw_mul(h->e, c, a, b, base, S(stream), npolys);
}
int cp_mul_u64(const cp_engine* h, void* c, const void* a, const uint64_t* b, int base, void* stream) {
  PW_CHECK("cp_mul_u64");
  CP_REQUIRE(c && a && b, "cp_mul_u64: NULL buffer");
  return pw_mul_u64(h->e, c, a, b, base, S(stream));
}
int cp_muladd(const cp_engine* h, void* d, const void* a, const void* b, const void* c, int base, void* stream) {
  PW_CHECK("cp_muladd");
  CP_REQUIRE(d && a && b && c, "cp_muladd: NULL buffer");
  return pw_muladd(h->e, d, a, b, c, base, S(stream));
}
int cp_dot(const cp_engine* h, void* c, const void* const* a, const void* const* b, int n, int base,
           void* stream) {
  PW_CHECK("cp_dot");
  CP_REQUIRE(c && a && b && n >= 1, "cp_dot: NULL buffer or n < 1");
  for (int t = 0; t < n; ++t) CP_REQUIRE(a[t] && b[t], "cp_dot: NULL operand");
  NvtxRange range("cp_dot");
  return pw_dot(h->e, c, a, b, n, base, S(stream));
}
int cp_dot_batch(const cp_engine* h, void* c, const void* a, const void* b, int n, int npolys, int b_shared, int base,
                 void* stream) {
  PW_CHECK("cp_dot_batch");
  CP_REQUIRE(c && a && b && n >= 1 && npolys >= 0, "cp_dot_batch: NULL buffer, n < 1 or npolys < 0");
  NvtxRange range("cp_dot_batch");
  return pw_dot_batch(h->e, c, a, b, n, npolys, b_shared != 0, base, S(stream));
}
int cp_dr2(const cp_engine* h, void* c21, void* c22, void* c23, const void* c01, const void* c02, const void* c11,
           const void* c12, int base, void* stream) {
  PW_CHECK("cp_dr2");
  CP_REQUIRE(c21 && c22 && c23 && c01 && c02 && c11 && c12, "cp_dr2: NULL buffer");
  return pw_dr2(h->e, c21, c22, c23, c01, c02, c11, c12, base, S(stream));
}
int cp_negate(const cp_engine* h, void* b, const void* a, int base, void* stream) {
  PW_CHECK("cp_negate");
  CP_REQUIRE(b && a, "cp_negate: NULL buffer");
  return pw_negate(h->e, b, a, base, S(stream));
}
int cp_op_by_int(const cp_engine* h, void* b, const void* a, int base, uint64_t x, int op, void* stream) {
  PW_CHECK("cp_op_by_int");
  CP_REQUIRE(b && a, "cp_op_by_int: NULL buffer");
  return pw_op_by_int(h->e, b, a, base, x, op, S(stream));
}
int cp_double_op_by_int(const cp_engine* h, void* b1, const void* a1, void* b2, const void* a2, int base, uint64_t x1,
                        uint64_t x2, int op, void* stream) {
  PW_CHECK("cp_double_op_by_int");
  CP_REQUIRE(b1 && a1 && b2 && a2, "cp_double_op_by_int: NULL buffer");
  return pw_double_op_by_int(h->e, b1, a1, b2, a2, base, x1, x2, op, S(stream));
}

int cp_basis_ext_q_to_b(const cp_engine* h, void* out_b, const void* in_q, int npolys, void* stream) {
  CP_BFV_ONLY(h, "cp_basis_ext_q_to_b");
  CP_REQUIRE(h && out_b && in_q && npolys >= 0, "cp_basis_ext_q_to_b: bad argument");
  if (npolys == 0) return CP_OK;
  return hps_basis_ext(h->e, out_b, in_q, true, npolys, S(stream));
}
int cp_basis_ext_b_to_q(const cp_engine* h, void* out_q, const void* in_b, int npolys, void* stream) {
  CP_BFV_ONLY(h, "cp_basis_ext_b_to_q");
  CP_REQUIRE(h && out_q && in_b && npolys >= 0, "cp_basis_ext_b_to_q: bad argument");
  if (npolys == 0) return CP_OK;
  return hps_basis_ext(h->e, out_q, in_b, false, npolys, S(stream));
}
int cp_complex_scaling(const cp_engine* h, void* out_b, const void* in_q, const void* in_b, int npolys,
                       void* stream) {
  CP_BFV_ONLY(h, "cp_complex_scaling");
  CP_REQUIRE(h && out_b && in_q && in_b && npolys >= 0, "cp_complex_scaling: bad argument");
  if (npolys == 0) return CP_OK;
  return hps_complex_scaling(h->e, out_b, in_q, in_b, npolys, S(stream));
}
int cp_simple_scaling(const cp_engine* h, void* out_t, const void* in_q, void* stream) {
  CP_BFV_ONLY(h, "cp_simple_scaling");
  CP_REQUIRE(h && out_t && in_q, "cp_simple_scaling: bad argument");
  return hps_simple_scaling(h->e, out_t, in_q, S(stream));
}
int cp_xi(const cp_engine* h, void* out, const void* in, void* stream) {
  CP_BFV_ONLY(h, "cp_xi");
  CP_REQUIRE(h && out && in, "cp_xi: bad argument");
  return rns_xi_rho(h->e, out, in, false, S(stream));
}
int cp_rho(const cp_engine* h, void* out, const void* in, void* stream) {
  CP_BFV_ONLY(h, "cp_rho");
  CP_REQUIRE(h && out && in, "cp_rho: bad argument");
  return rns_xi_rho(h->e, out, in, true, S(stream));
}
int cp_xi_batch(const cp_engine* h, void* out, const void* in, int npolys, void* stream) {
  CP_BFV_ONLY(h, "cp_xi_batch");
  CP_REQUIRE(h && out && in && npolys >= 0, "cp_xi_batch: bad argument");
  return rns_xi_rho(h->e, out, in, false, S(stream), npolys);
}
int cp_rho_batch(const cp_engine* h, void* out, const void* in, int npolys, void* stream) {
  CP_BFV_ONLY(h, "cp_rho_batch");
  CP_REQUIRE(h && out && in && npolys >= 0, "cp_rho_batch: bad argument");
  return rns_xi_rho(h->e, out, in, true, S(stream), npolys);
}

// ---------------- composite calls ----------------

static int d2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (dst == src || bytes == 0) return CP_OK;
  cudaError_t err = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st);
  return err == cudaSuccess ? CP_OK : cuda_fail("cudaMemcpyAsync", err);
}

#define CP_TRY(x)            \
  do {                       \
    int rc_ = (x);           \
    if (rc_) return rc_;     \
  } while (0)

// Inverse DGT of one polynomial over `base` from `src` into `dst` (out of place: the
// kernel reads the source directly, no copy first).
static int inv_dgt_from(const Engine& e, void* dst, const void* src, int base, cudaStream_t st) {
  InvSrc is{};
  is.p[0] = reinterpret_cast<const ulonglong2*>(src);
  is.mode = 0;
  is.npairs = 1;
  return launch_dgt_ex(e, dst, nullptr, &is, base, 1, 0, true, st);
}

int cp_poly_basis_extension_q_to_b(const cp_engine* h, void* out_b, const void* in_q, void* ws, void* stream) {
  CP_BFV_ONLY(h, "cp_poly_basis_extension_q_to_b");
  CP_REQUIRE(h && out_b && in_q && ws, "cp_poly_basis_extension_q_to_b: bad argument");
  const Engine& e = h->e;
  cudaStream_t st = S(stream);
  CP_TRY(inv_dgt_from(e, ws, in_q, CP_QBASE, st));
  CP_TRY(hps_basis_ext(e, out_b, ws, true, 1, st));
  return launch_dgt(e, out_b, CP_BBASE, 1, 0, false, st);
}

int cp_poly_basis_extension_q_to_qb(const cp_engine* h, void* out_qb, const void* in_q, void* ws, void* stream) {
  CP_BFV_ONLY(h, "cp_poly_basis_extension_q_to_qb");
  CP_REQUIRE(h && out_qb && in_q && ws, "cp_poly_basis_extension_q_to_qb: bad argument");
  const Engine& e = h->e;
  cudaStream_t st = S(stream);
  const size_t qb = (size_t)e.k * e.N * 16;
  char* ob = reinterpret_cast<char*>(out_qb) + qb;
  CP_TRY(inv_dgt_from(e, ws, in_q, CP_QBASE, st));
  CP_TRY(hps_basis_ext(e, ob, ws, true, 1, st));
  CP_TRY(launch_dgt(e, ob, CP_BBASE, 1, 0, false, st));
  return d2d(out_qb, in_q, qb, st);
}

int cp_poly_basis_extension_b_to_q(const cp_engine* h, void* out_q, const void* in_b, void* ws, void* stream) {
  CP_BFV_ONLY(h, "cp_poly_basis_extension_b_to_q");
  CP_REQUIRE(h && out_q && in_b && ws, "cp_poly_basis_extension_b_to_q: bad argument");
  const Engine& e = h->e;
  cudaStream_t st = S(stream);
  CP_TRY(inv_dgt_from(e, ws, in_b, CP_BBASE, st));
  CP_TRY(hps_basis_ext(e, out_q, ws, false, 1, st));
  return launch_dgt(e, out_q, CP_QBASE, 1, 0, false, st);
}

int cp_poly_complex_scaling_tdivq(const cp_engine* h, void* out_q, void* in_q, void* in_b, unsigned flags, void* ws,
                                  void* stream) {
  CP_BFV_ONLY(h, "cp_poly_complex_scaling_tdivq");
  CP_REQUIRE(h && out_q && in_q && in_b && ws, "cp_poly_complex_scaling_tdivq: bad argument");
  const Engine& e = h->e;
  cudaStream_t st = S(stream);
  const size_t qe = (size_t)e.k * e.N, be = (size_t)e.kl * e.N;
  ulonglong2* w = reinterpret_cast<ulonglong2*>(ws);
  void* xq = in_q;
  void* xb = in_b;
  if (!(flags & CP_DESTROY_INPUTS)) {  // inputs kept: transform out of place into the workspace
    xq = w;
    xb = w + qe;
  }
  void* u = w + qe + be;
  CP_TRY(inv_dgt_from(e, xq, in_q, CP_QBASE, st));
  CP_TRY(inv_dgt_from(e, xb, in_b, CP_BBASE, st));
  CP_TRY(hps_scale_to_q(e, out_q, xq, xb, u, 1, st));
  return launch_dgt(e, out_q, CP_QBASE, 1, 0, false, st);
}

int cp_poly_simple_scaling_tdivq(const cp_engine* h, void* out_t, const void* in_q, void* ws, void* stream) {
  CP_BFV_ONLY(h, "cp_poly_simple_scaling_tdivq");
  CP_REQUIRE(h && out_t && in_q && ws, "cp_poly_simple_scaling_tdivq: bad argument");
  const Engine& e = h->e;
  cudaStream_t st = S(stream);
  CP_TRY(inv_dgt_from(e, ws, in_q, CP_QBASE, st));
  return hps_simple_scaling(e, out_t, ws, st);
}

int cp_bfv_mul(const cp_engine* h, void* c0, void* c1, void* c2, const void* a0, const void* a1, const void* b0,
               const void* b1, void* ws, void* stream) {
  CP_BFV_ONLY(h, "cp_bfv_mul");
  CP_REQUIRE(h && c0 && c1 && c2 && a0 && a1 && b0 && b1 && ws, "cp_bfv_mul: bad argument");
  NvtxRange range("cp_bfv_mul");
  const Engine& e = h->e;
  cudaStream_t st = S(stream);
  const size_t qe = (size_t)e.k * e.N, be = (size_t)e.kl * e.N;
  ulonglong2* w = reinterpret_cast<ulonglong2*>(ws);
  // layout: xb[4] (B), cb[3] (B), cq[3] (Q), scratch (k + 2 kl)
  ulonglong2* xb = w;
  ulonglong2* cb = xb + 4 * be;
  ulonglong2* cq = cb + 3 * be;
  ulonglong2* scratch = cq + 3 * qe;
  const void* in[4] = {a0, a1, b0, b1};
  for (int i = 0; i < 4; ++i) CP_TRY(cp_poly_basis_extension_q_to_b(h, xb + i * be, in[i], scratch, stream));
  CP_TRY(pw_dr2(e, cq, cq + qe, cq + 2 * qe, a0, a1, b0, b1, CP_QBASE, st));
  CP_TRY(pw_dr2(e, cb, cb + be, cb + 2 * be, xb, xb + be, xb + 2 * be, xb + 3 * be, CP_BBASE, st));
  void* outs[3] = {c0, c1, c2};
  for (int i = 0; i < 3; ++i)
    CP_TRY(cp_poly_complex_scaling_tdivq(h, outs[i], cq + i * qe, cb + i * be, CP_DESTROY_INPUTS, scratch, stream));
  return CP_OK;
}

size_t cp_bfv_mul_batch_workspace_bytes(const cp_engine* h, int npairs) {
  if (!h || npairs <= 0) return 0;
  const Engine& e = h->e;
  // X[4P][k] + XB[4P][kl] + CQ[3P][k] + CB[3P][kl] + U[3P][kl]
  return (size_t)npairs * (7 * e.k + 10 * e.kl) * e.N * 16;
}

int cp_bfv_mul_batch(const cp_engine* h, void* c, const void* a0, const void* a1, const void* b0, const void* b1,
                     int npairs, void* ws, void* stream) {
  CP_BFV_ONLY(h, "cp_bfv_mul_batch");
  CP_REQUIRE(h && c && a0 && a1 && b0 && b1 && ws && npairs >= 0, "cp_bfv_mul_batch: bad argument");
  if (npairs == 0) return CP_OK;
  NvtxRange range("cp_bfv_mul_batch");
  const Engine& e = h->e;
  cudaStream_t st = S(stream);
  const size_t P = (size_t)npairs;
  const size_t qe = (size_t)e.k * e.N, be = (size_t)e.kl * e.N;
  ulonglong2* X = reinterpret_cast<ulonglong2*>(ws);  // [4][P][k]
  ulonglong2* XB = X + 4 * P * qe;                     // [4][P][kl]
  ulonglong2* CQ = XB + 4 * P * be;                    // [3][P][k]
  ulonglong2* CB = CQ + 3 * P * qe;                    // [3][P][kl]
  ulonglong2* U = CB + 3 * P * be;                     // [3][P][kl]
  // Every inverse DGT below untwists with a prescaled table (off_untwist_pre), so that it
  // also applies the first constant product of the conversion that reads its output.
  // 1. inverse DGT of the four inputs over Q, gathered into X (no copies):
  //    X = x_i (Q/q_i)^-1 mod q_i
  InvSrc gather{};
  gather.p[0] = reinterpret_cast<const ulonglong2*>(a0);
  gather.p[1] = reinterpret_cast<const ulonglong2*>(a1);
  gather.p[2] = reinterpret_cast<const ulonglong2*>(b0);
  gather.p[3] = reinterpret_cast<const ulonglong2*>(b1);
  gather.mode = 2;
  gather.npairs = npairs;
  gather.untwist = 1;
  {
    NvtxRange r("inverse DGT over Q (4P)");
    CP_TRY(launch_dgt_ex(e, X, nullptr, &gather, CP_QBASE, 4 * npairs, 0, true, st));
  }
  // 2. exact Q -> B extension, forward DGT over B
  {
    NvtxRange r("Q -> B, forward DGT over B (4P)");
    CP_TRY(hps_basis_ext_pre(e, XB, X, true, 4 * npairs, st));
    CP_TRY(launch_dgt(e, XB, CP_BBASE, 4 * npairs, 0, false, st));
  }
  // 3. tensor product computed inside the inverse DGTs (Q side from the inputs, B side from
  //    XB): CQ = t c_i (Q/q_i)^-1 mod q_i, CB = t Q^-1 (B/b_j)^-1 c_j mod b_j
  InvSrc tq = gather;
  tq.mode = 1;
  tq.untwist = 2;
  NvtxRange r3("tensor products + inverse DGTs (3P over Q and B)");
  CP_TRY(launch_dgt_ex(e, CQ, nullptr, &tq, CP_QBASE, 3 * npairs, 0, true, st));
  InvSrc tb{};
  for (int v = 0; v < 4; ++v) tb.p[v] = XB + v * P * be;
  tb.mode = 1;
  tb.npairs = npairs;
  tb.untwist = 1;
  CP_TRY(launch_dgt_ex(e, CB, nullptr, &tb, CP_BBASE, 3 * npairs, 0, true, st));
  // 4. round(t X / Q) and B -> Q, then forward DGT of the outputs
  NvtxRange r4("scale t/Q, B -> Q, forward DGT over Q (3P)");
  CP_TRY(hps_scale_to_q_pre(e, c, CQ, CB, U, 3 * npairs, st));
  return launch_dgt(e, c, CP_QBASE, 3 * npairs, 0, false, st);
}

int cp_sample(const cp_engine* h, void* out, int base, int kind, uint64_t seed, uint32_t stream_id, int npolys,
              int to_dgt, void* stream) {
  CP_REQUIRE(valid_base(h, base) && out && npolys >= 0, "cp_sample: bad argument");
  if (npolys == 0) return CP_OK;
  CP_TRY(sample_poly(h->e, out, base, kind, seed, stream_id, npolys, S(stream)));
  if (to_dgt) return launch_dgt(h->e, out, base, npolys, 0, false, S(stream));
  return CP_OK;
}

int cp_sample_ids(const cp_engine* h, void* out, int base, int kind, uint64_t seed, const uint32_t* stream_ids,
                  int npolys, int to_dgt, void* stream) {
  CP_REQUIRE(valid_base(h, base) && out && stream_ids && npolys >= 0, "cp_sample_ids: bad argument");
  if (npolys == 0) return CP_OK;
  CP_TRY(sample_poly(h->e, out, base, kind, seed, 0, npolys, S(stream), stream_ids));
  if (to_dgt) return launch_dgt(h->e, out, base, npolys, 0, false, S(stream));
  return CP_OK;
}

}  // extern "C"
