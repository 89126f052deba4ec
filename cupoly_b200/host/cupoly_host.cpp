// C++ host layer: cuPoly's CUDAEngine / Context / poly_t / DGTEngine / Sampler
// API (include/cuPoly/...) implemented over the cupoly_b200 C ABI
// (include/cupoly_b200.h).  Built as cupoly_b200/lib/libcupoly.so (linked with
// libcupoly_b200.so and libcudart); see cupoly_b200/build.py.
//
// Follows cuPoly's src/arithmetic/polynomial.cu (state machine :45-188,
// operations :310-1153, text I/O :1181-1437, residue access :1489-1660),
// src/arithmetic/context.cpp and src/cuda/cudaengine.cu:1186-1779, with the
// kernels replaced by C-ABI calls and the host NTL CRT replaced by the device
// cp_crt / cp_icrt.  Every ABI status other than CP_OK becomes a
// std::runtime_error carrying cp_last_error().
#include <cuPoly/arithmetic/polynomial.h>
#include <cuPoly/cuda/sampler.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
namespace {

void check(int rc, const char* what) {
  if (rc != CP_OK) throw std::runtime_error(std::string(what) + ": " + cp_last_error());
}

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

void require(bool ok, const char* msg) {
  if (!ok) throw std::runtime_error(msg);
}

cp_engine* E() { return CUDAEngine::handle(); }
void* S(Context* ctx) { return (void*)ctx->get_stream(); }
int nres(int base) { return CUDAEngine::get_n_residues(base); }
int nphi() { return 2 * CUDAEngine::N; }
size_t res_bytes(int base) { return (size_t)CUDAEngine::N * (size_t)nres(base) * sizeof(GaussianInteger); }
size_t alloc_bytes() { return res_bytes(QBBase); }  // every poly_t buffer holds a QB polynomial

NTL::ZZ product(const std::vector<uint64_t>& ps) {
  NTL::ZZ r = NTL::conv<NTL::ZZ>(1L);
  for (uint64_t p : ps) r *= NTL::conv<NTL::ZZ>((unsigned long)p);
  return r;
}

NTL::ZZ base_product(int base) {
  switch (base) {
    case QBase: return CUDAEngine::RNSProduct;
    case BBase: return CUDAEngine::RNSBProduct;
    case QBBase: return CUDAEngine::RNSProduct * CUDAEngine::RNSBProduct;
    case TBase: return NTL::conv<NTL::ZZ>((unsigned long)CUDAEngine::t);
    default: throw std::runtime_error("Unknown base");
  }
}

uint64_t inv_mod(uint64_t a, uint64_t p) {  // a^-1 mod p by the extended Euclidean algorithm
  __int128 t0 = 0, t1 = 1, r0 = p, r1 = a % p;
  while (r1 != 0) {
    const __int128 q = r0 / r1;
    __int128 tmp = r0 - q * r1;
    r0 = r1;
    r1 = tmp;
    tmp = t0 - q * t1;
    t0 = t1;
    t1 = tmp;
  }
  require(r0 == 1, "inv_mod: not invertible");
  return (uint64_t)(t0 < 0 ? t0 + p : t0);
}

// ZZ <-> machine words and little-endian 64-bit limbs.
NTL::ZZ zz_u64(uint64_t v) { return NTL::conv<NTL::ZZ>((unsigned long)v); }
#ifdef CUPOLY_WITH_NTL
size_t zz_nlimbs(const NTL::ZZ& x) { return (size_t)((NTL::NumBits(x) + 63) / 64); }
void zz_to_limbs(const NTL::ZZ& x, uint64_t* w, size_t n) {
  std::memset(w, 0, n * 8);
  NTL::BytesFromZZ(reinterpret_cast<unsigned char*>(w), x, (long)(n * 8));
}
NTL::ZZ zz_from_limbs(const uint64_t* w, size_t n) {
  return NTL::ZZFromBytes(reinterpret_cast<const unsigned char*>(w), (long)(n * 8));
}
#else
size_t zz_nlimbs(const NTL::ZZ& x) { return x.limbs().size(); }
void zz_to_limbs(const NTL::ZZ& x, uint64_t* w, size_t n) {
  const auto& l = x.limbs();
  std::memset(w, 0, n * 8);
  std::copy(l.begin(), l.begin() + std::min(l.size(), n), w);
}
NTL::ZZ zz_from_limbs(const uint64_t* w, size_t n) { return NTL::ZZ::from_limbs(w, n); }
#endif

NTL::ZZ zz_from_decimal(const std::string& s) { return NTL::conv<NTL::ZZ>(s.c_str()); }

// x mod m in [0, m) for m > 0 (NTL's % takes the sign of the divisor).
NTL::ZZ floor_mod(const NTL::ZZ& x, const NTL::ZZ& m) { return x % m; }

// ---- cuPoly's tabulated roots of i, read from its own data files ----
//
// cuPoly's NTHROOT[p][N] (src/arithmetic/coprimes.cu:868, used by
// src/cuda/dgt.cu:1610-1692) is generated from the JSON files of
// src/arithmetic/coprimes/: qis_<bits>.json maps each prime p of that bit
// length to [ {N: {"re": ..., "imag": ...}, ...}, ... ], the first element
// holding xi with xi^N = i.  A minimal reader of that format follows: objects,
// arrays, strings and unsigned integers (the only value types those files use).
struct RootFileReader {
  const std::string& s;
  size_t i = 0;
  explicit RootFileReader(const std::string& text) : s(text) {}
  void ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
  }
  bool eat(char c) {
    ws();
    if (i < s.size() && s[i] == c) {
      ++i;
      return true;
    }
    return false;
  }
  void expect(char c) {
    if (!eat(c)) throw std::runtime_error(std::string("cuPoly root table: expected '") + c + "'");
  }
  std::string str() {
    expect('"');
    const size_t b = i;
    while (i < s.size() && s[i] != '"') ++i;
    require(i < s.size(), "cuPoly root table: unterminated string");
    return s.substr(b, i++ - b);
  }
  uint64_t num() {
    ws();
    const size_t b = i;
    while (i < s.size() && std::isdigit((unsigned char)s[i])) ++i;
    require(i > b && i - b <= 20, "cuPoly root table: expected an unsigned integer");
    errno = 0;
    const unsigned long long v = std::strtoull(s.c_str() + b, nullptr, 10);
    require(errno == 0, "cuPoly root table: integer out of range");
    return (uint64_t)v;
  }
  void skip() {  // any value
    ws();
    require(i < s.size(), "cuPoly root table: truncated");
    if (s[i] == '{') {
      ++i;
      if (eat('}')) return;
      do {
        str();
        expect(':');
        skip();
      } while (eat(','));
      expect('}');
    } else if (s[i] == '[') {
      ++i;
      if (eat(']')) return;
      do skip();
      while (eat(','));
      expect(']');
    } else if (s[i] == '"') {
      str();
    } else {
      num();
    }
  }
  // {"re": a, "imag": b}
  std::pair<uint64_t, uint64_t> gauss() {
    uint64_t re = 0, im = 0;
    int seen = 0;
    expect('{');
    do {
      const std::string k = str();
      expect(':');
      if (k == "re") re = num(), seen |= 1;
      else if (k == "imag") im = num(), seen |= 2;
      else skip();
    } while (eat(','));
    expect('}');
    require(seen == 3, "cuPoly root table: a root lacks re or imag");
    return {re, im};
  }
  // Whole file: p -> (N -> xi) from the first element of each prime's array.
  void read(std::map<uint64_t, std::map<int, std::pair<uint64_t, uint64_t>>>& out) {
    expect('{');
    if (eat('}')) return;
    do {
      const uint64_t p = std::strtoull(str().c_str(), nullptr, 10);
      expect(':');
      expect('[');
      auto& roots = out[p];
      if (!eat(']')) {
        expect('{');
        if (!eat('}')) {
          do {
            const int n = std::atoi(str().c_str());
            expect(':');
            roots[n] = gauss();
          } while (eat(','));
          expect('}');
        }
        while (eat(',')) skip();
        expect(']');
      }
    } while (eat(','));
    expect('}');
  }
};

// Load xi = NTHROOT[p][N] for every prime of the engine from cuPoly's
// coprimes directory and install it (cp_engine_set_nthroot).
void load_cupoly_roots(cp_engine* e, const std::string& dir, int N) {
  const int n = cp_engine_n_residues(e, CP_QBBASE);
  std::vector<uint64_t> ps(n), xi(2 * (size_t)n);
  require(cp_engine_primes(e, ps.data(), n) == n, "cp_engine_primes failed");
  std::map<int, std::map<uint64_t, std::map<int, std::pair<uint64_t, uint64_t>>>> files;  // by bit length
  for (int r = 0; r < n; ++r) {
    const int bits = 64 - __builtin_clzll(ps[r]);
    if (!files.count(bits)) {
      const std::string path = dir + "/qis_" + std::to_string(bits) + ".json";
      std::FILE* f = std::fopen(path.c_str(), "rb");
      if (!f) throw std::runtime_error("cuPoly root table: cannot open " + path);
      std::string text;
      char buf[1 << 16];
      size_t got;
      while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
      std::fclose(f);
      RootFileReader(text).read(files[bits]);
    }
    const auto& tab = files[bits];
    const auto pi = tab.find(ps[r]);
    const bool found = pi != tab.end() && pi->second.count(N);
    if (!found)
      throw std::runtime_error("cuPoly root table in " + dir + " has no root for prime " + std::to_string(ps[r]) +
                               " and N = " + std::to_string(N));
    const auto x = pi->second.at(N);
    xi[2 * (size_t)r] = x.first;
    xi[2 * (size_t)r + 1] = x.second;
  }
  check(cp_engine_set_nthroot(e, xi.data()), "cp_engine_set_nthroot (cuPoly's root table)");
}

// With CUPOLY_COPRIMES_DIR set, engines take cuPoly's roots; otherwise the
// library's canonical root, said once on stderr (coefficient-domain results
// are the same either way; only the DGT-domain bytes of poly_t::d_coefs differ).
void apply_root_table(cp_engine* e, int N) {
  const char* dir = std::getenv("CUPOLY_COPRIMES_DIR");
  if (dir && *dir) {
    load_cupoly_roots(e, dir, N);
    return;
  }
  static bool said = false;
  if (!said) {
    said = true;
    std::fprintf(stderr,
                 "cupoly_b200: DGT-domain bytes use the library's canonical root of i; set CUPOLY_COPRIMES_DIR to "
                 "cuPoly's src/arithmetic/coprimes directory for cuPoly's own (coefficient-domain results do not "
                 "depend on it)\n");
  }
}

void d2d(void* dst, const void* src, size_t bytes, Context* ctx) {
  if (dst == src || bytes == 0) return;
  cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->get_stream()), "cudaMemcpyAsync");
}

void sync(Context* ctx) { cuda_check(cudaStreamSynchronize(ctx->get_stream()), "cudaStreamSynchronize"); }

// Inputs to the device; output initialised for `base` (cuPoly's lazy poly_init of outputs).
void prep_out(Context* ctx, poly_t* out, int base) {
  poly_init(ctx, out, base);
  out->base = base;
}
void done(poly_t* out, int base) {
  out->status = RNSSTATE;
  out->base = base;
}
void same_base(const poly_t* a, const poly_t* b) { require(a->base == b->base, "operands lie in different bases"); }

// Coefficient-domain copy of a's residues in the context's aux buffer.
GaussianInteger* coefficient_residues(Context* ctx, poly_t* a) {
  poly_copy_to_device(ctx, a);
  GaussianInteger* aux = ctx->aux();
  d2d(aux, a->d_coefs, res_bytes(a->base), ctx);
  DGTEngine::execute_dgt(aux, a->base, INVERSE, ctx);
  return aux;
}

}  // namespace

// ---------------------------------------------------------------------------
// CUDAEngine (cudaengine.cu:1186-1779)
// ---------------------------------------------------------------------------
int CUDAEngine::is_init = 0;
int CUDAEngine::N = 0;
uint64_t CUDAEngine::t = 0;
int CUDAEngine::scalingfactor = 0;
int CUDAEngine::dnum = 0;
std::vector<uint64_t> CUDAEngine::RNSPrimes;
std::vector<uint64_t> CUDAEngine::RNSBPrimes;
NTL::ZZ CUDAEngine::RNSProduct;
NTL::ZZ CUDAEngine::RNSBProduct;
std::vector<NTL::ZZ> CUDAEngine::RNSMpi;
std::vector<uint64_t> CUDAEngine::RNSInvMpi;
cp_engine* CUDAEngine::engine = nullptr;
bool DGTEngine::is_init = false;

static void fill_statics(int M) {
  cp_engine* e = CUDAEngine::engine;
  const int k = cp_engine_n_residues(e, CP_QBASE), kl = cp_engine_n_residues(e, CP_BBASE);
  std::vector<uint64_t> ps(k + kl);
  if (cp_engine_primes(e, ps.data(), k + kl) != k + kl)  // returns the count written
    throw std::runtime_error(std::string("cp_engine_primes: ") + cp_last_error());
  CUDAEngine::N = M / 2;
  CUDAEngine::RNSPrimes.assign(ps.begin(), ps.begin() + k);
  CUDAEngine::RNSBPrimes.assign(ps.begin() + k, ps.end());
  CUDAEngine::RNSProduct = product(CUDAEngine::RNSPrimes);
  CUDAEngine::RNSBProduct = product(CUDAEngine::RNSBPrimes);
  CUDAEngine::RNSMpi.clear();
  CUDAEngine::RNSInvMpi.clear();
  for (uint64_t q : CUDAEngine::RNSPrimes) {
    const NTL::ZZ m = CUDAEngine::RNSProduct / zz_u64(q);
    CUDAEngine::RNSMpi.push_back(m);
    const uint64_t r = (uint64_t)NTL::conv<unsigned long>(m % zz_u64(q));
    CUDAEngine::RNSInvMpi.push_back(inv_mod(r, q));
  }
  apply_root_table(e, M / 2);
  DGTEngine::init();
  CUDAEngine::is_init = 1;
}

void CUDAEngine::load_nthroot_table(const std::string& coprimes_dir) {
  load_cupoly_roots(handle(), coprimes_dir, N);
}

void CUDAEngine::init_bfv(int k, int kl, int M, uint64_t t_) {
  if (is_init) destroy();
  check(cp_engine_create(&engine, k, kl < 0 ? k + 1 : kl, M, t_, 0), "CUDAEngine::init");
  t = t_;
  scalingfactor = 0;
  fill_statics(M);
}

void CUDAEngine::init_ckks(int k, int kl, int M, int prec) {
  if (is_init) destroy();
  check(cp_ckks_engine_create(&engine, k, kl < 0 ? k + 1 : kl, M, prec, 0), "CUDAEngine::init (CKKS)");
  t = (uint64_t)prec;
  scalingfactor = prec;
  fill_statics(M);
}

void CUDAEngine::destroy() {
  if (engine) {
    cudaDeviceSynchronize();
    cp_engine_destroy(engine);
  }
  engine = nullptr;
  is_init = 0;
  N = 0;
  RNSPrimes.clear();
  RNSBPrimes.clear();
  RNSMpi.clear();
  RNSInvMpi.clear();
  RNSProduct = NTL::ZZ(0);
  RNSBProduct = NTL::ZZ(0);
  DGTEngine::destroy();
}

cp_engine* CUDAEngine::handle() {
  require(is_init && engine, "CUDAEngine is not initialised");
  return engine;
}

int CUDAEngine::get_n_residues(int base) {
  const int n = cp_engine_n_residues(handle(), base);
  require(n > 0, "Unknown base");
  return n;
}

void CUDAEngine::execute_polynomial_negate(GaussianInteger* b, const GaussianInteger* a, const int base,
                                           Context* ctx) {
  check(cp_negate(E(), b, a, base, S(ctx)), "execute_polynomial_negate");
}

void CUDAEngine::execute_polynomial_op_by_int(GaussianInteger* b, GaussianInteger* a, const int base, uint64_t x,
                                              int OP, Context* ctx) {
  check(cp_op_by_int(E(), b, a, base, x, OP, S(ctx)), "execute_polynomial_op_by_int");
}

void CUDAEngine::execute_polynomial_double_op_by_int(GaussianInteger* b1, GaussianInteger* a1, GaussianInteger* b2,
                                                     GaussianInteger* a2, const int base, uint64_t x1, uint64_t x2,
                                                     int OP, Context* ctx) {
  check(cp_double_op_by_int(E(), b1, a1, b2, a2, base, x1, x2, OP, S(ctx)), "execute_polynomial_double_op_by_int");
}

size_t poly_get_residues_size(int base) { return res_bytes(base); }

// ---------------------------------------------------------------------------
// DGTEngine (dgt.cu:1069-1499)
// ---------------------------------------------------------------------------
void DGTEngine::execute_dgt(GaussianInteger* data, const int base, const int direction, Context* ctx) {
  check(cp_dgt(E(), data, base, direction, 1, 0, S(ctx)), "execute_dgt");
}
void DGTEngine::execute_add_dgt(GaussianInteger* c, const GaussianInteger* a, const GaussianInteger* b,
                                const int base, const cudaStream_t stream) {
  check(cp_add(E(), c, a, b, base, (void*)stream), "execute_add_dgt");
}
void DGTEngine::execute_sub_dgt(GaussianInteger* c, const GaussianInteger* a, const GaussianInteger* b,
                                const int base, const cudaStream_t stream) {
  check(cp_sub(E(), c, a, b, base, (void*)stream), "execute_sub_dgt");
}
void DGTEngine::execute_double_add_dgt(GaussianInteger* c1, const GaussianInteger* a1, const GaussianInteger* b1,
                                       GaussianInteger* c2, const GaussianInteger* a2, const GaussianInteger* b2,
                                       const int base, const cudaStream_t stream) {
  check(cp_double_add(E(), c1, a1, b1, c2, a2, b2, base, (void*)stream), "execute_double_add_dgt");
}
void DGTEngine::execute_dr2_dgt(GaussianInteger* ct21, GaussianInteger* ct22, GaussianInteger* ct23,
                                const GaussianInteger* ct01, const GaussianInteger* ct02, const GaussianInteger* ct11,
                                const GaussianInteger* ct12, const int base, const cudaStream_t stream) {
  check(cp_dr2(E(), ct21, ct22, ct23, ct01, ct02, ct11, ct12, base, (void*)stream), "execute_dr2_dgt");
}
void DGTEngine::execute_mul_dgt_gi(GaussianInteger* c, const GaussianInteger* a, const GaussianInteger* b,
                                   const int base, const cudaStream_t stream) {
  check(cp_mul(E(), c, a, b, base, (void*)stream), "execute_mul_dgt_gi");
}
void DGTEngine::execute_mul_dgt_u64(GaussianInteger* c, const GaussianInteger* a, const uint64_t* b,
                                    const int base, const cudaStream_t stream) {
  check(cp_mul_u64(E(), c, a, b, base, (void*)stream), "execute_mul_dgt_u64");
}
void DGTEngine::execute_muladd_dgt(GaussianInteger* d, const GaussianInteger* a, const GaussianInteger* b,
                                   const GaussianInteger* c, const int base, const cudaStream_t stream) {
  check(cp_muladd(E(), d, a, b, c, base, (void*)stream), "execute_muladd_dgt");
}

// ---------------------------------------------------------------------------
// Context (context.cpp:19-67)
// ---------------------------------------------------------------------------
Context::Context() {
  require(CUDAEngine::is_init, "Context: CUDAEngine is not initialised");
  cuda_check(cudaStreamCreate(&stream), "cudaStreamCreate");
  aux();
}

Context::~Context() {
  if (stream) cudaStreamSynchronize(stream);
  cudaFree(d_workspace);
  cudaFree(d_aux_coefs);
  cudaFree(d_scratch);
  if (stream) cudaStreamDestroy(stream);
}

void Context::grow(void** p, size_t* have, size_t need) {
  if (need <= *have && *p) return;
  if (*p) {
    cuda_check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    cudaFree(*p);
    *p = nullptr;
    *have = 0;
  }
  cuda_check(cudaMalloc(p, need ? need : 16), "cudaMalloc");
  *have = need;
}

void* Context::workspace() {
  grow(&d_workspace, &workspace_bytes, cp_workspace_bytes(E()));
  return d_workspace;
}

GaussianInteger* Context::aux() {
  void* p = d_aux_coefs;
  grow(&p, &aux_bytes, alloc_bytes());
  d_aux_coefs = reinterpret_cast<GaussianInteger*>(p);
  return d_aux_coefs;
}

void* Context::scratch(size_t bytes) {
  grow(&d_scratch, &scratch_bytes, bytes);
  return d_scratch;
}

uint64_t* Context::host_scratch(size_t words) {
  if (h_scratch.size() < words) h_scratch.resize(words);
  return h_scratch.data();
}

// ---------------------------------------------------------------------------
// state machine and coefficient I/O (polynomial.cu:45-308)
// ---------------------------------------------------------------------------
void poly_init(Context* ctx, poly_t* a, int base) {
  if (a->init) return;
  require(ctx != nullptr, "poly_init: null context");
  nres(base);  // validates the base
  void* p = nullptr;
  cuda_check(cudaMalloc(&p, alloc_bytes()), "cudaMalloc");
  a->d_coefs = reinterpret_cast<GaussianInteger*>(p);
  cuda_check(cudaMemsetAsync(a->d_coefs, 0, alloc_bytes(), ctx->get_stream()), "cudaMemsetAsync");
  a->coefs.assign(nphi(), NTL::ZZ(0));
  a->base = base;
  a->status = BOTHSTATE;
  a->init = true;
}

void poly_free(Context* ctx, poly_t* a) {
  if (!a || !a->init) return;
  if (ctx) sync(ctx);
  cudaFree(a->d_coefs);
  a->d_coefs = NULL;
  a->coefs.clear();
  a->init = false;
}

void poly_clear(Context* ctx, poly_t* a) {
  poly_init(ctx, a);
  a->coefs.assign(nphi(), NTL::ZZ(0));
  cuda_check(cudaMemsetAsync(a->d_coefs, 0, alloc_bytes(), ctx->get_stream()), "cudaMemsetAsync");
  a->status = BOTHSTATE;
}

GaussianInteger* poly_crt(Context* ctx, poly_t* a) {
  require(a->init, "poly_crt: polynomial not initialised");
  require(a->base == QBase || a->base == BBase || a->base == QBBase, "poly_crt: base must be Q, B or QB");
  const NTL::ZZ m = base_product(a->base);
  const int n = nphi();
  std::vector<NTL::ZZ> c(n, NTL::ZZ(0));
  size_t nl = 1;
  bool reduce = false;
  for (int i = 0; i < n && i < (int)a->coefs.size(); ++i) {
    c[i] = a->coefs[i];
    if (c[i] < NTL::ZZ(0)) c[i] = floor_mod(c[i], m);
    nl = std::max(nl, zz_nlimbs(c[i]));
  }
  if (nl > 64) reduce = true;  // beyond the device limb limit: same residues after reduction
  if (reduce) {
    nl = 1;
    for (auto& x : c) {
      x = floor_mod(x, m);
      nl = std::max(nl, zz_nlimbs(x));
    }
  }
  uint64_t* h = ctx->host_scratch((size_t)n * nl);
  for (int i = 0; i < n; ++i) zz_to_limbs(c[i], h + (size_t)i * nl, nl);
  uint64_t* d = reinterpret_cast<uint64_t*>(ctx->scratch((size_t)n * nl * 8));
  cuda_check(cudaMemcpyAsync(d, h, (size_t)n * nl * 8, cudaMemcpyHostToDevice, ctx->get_stream()),
             "cudaMemcpyAsync");
  GaussianInteger* out = ctx->aux();
  check(cp_crt(E(), out, d, (int)nl, a->base, 1, S(ctx)), "poly_crt");
  sync(ctx);  // the host staging is reused by the next call
  return out;
}

void poly_icrt(Context* ctx, poly_t* a) {
  require(a->base == QBase || a->base == BBase || a->base == TBase, "Unknown base");
  GaussianInteger* aux = coefficient_residues(ctx, a);
  const int n = nphi(), nl = nres(a->base);
  uint64_t* d = reinterpret_cast<uint64_t*>(ctx->scratch((size_t)n * nl * 8));
  check(cp_icrt(E(), d, nl, aux, a->base, 1, S(ctx)), "poly_icrt");
  uint64_t* h = ctx->host_scratch((size_t)n * nl);
  cuda_check(cudaMemcpyAsync(h, d, (size_t)n * nl * 8, cudaMemcpyDeviceToHost, ctx->get_stream()),
             "cudaMemcpyAsync");
  sync(ctx);
  a->coefs.resize(n);
  for (int i = 0; i < n; ++i) a->coefs[i] = zz_from_limbs(h + (size_t)i * nl, nl);
}

void poly_copy_to_device(Context* ctx, poly_t* a) {
  require(a->init, "poly_copy_to_device: polynomial not initialised");
  if (a->status == RNSSTATE || a->status == BOTHSTATE) return;
  GaussianInteger* r = poly_crt(ctx, a);
  d2d(a->d_coefs, r, res_bytes(a->base), ctx);
  DGTEngine::execute_dgt(a->d_coefs, a->base, FORWARD, ctx);
  sync(ctx);
  a->status = BOTHSTATE;
}

void poly_copy_to_host(Context* ctx, poly_t* a) {
  require(a->init, "poly_copy_to_host: polynomial not initialised");
  if (a->status == HOSTSTATE || a->status == BOTHSTATE) return;
  poly_icrt(ctx, a);
  a->status = BOTHSTATE;
}

void poly_copy(Context* ctx, poly_t* b, poly_t* a) {
  poly_init(ctx, b, a->base);
  b->base = a->base;
  if (a->status == RNSSTATE || a->status == BOTHSTATE) {
    d2d(b->d_coefs, a->d_coefs, res_bytes(a->base), ctx);
    b->status = RNSSTATE;
  } else {
    b->coefs = a->coefs;
    b->status = HOSTSTATE;
  }
}

int poly_get_deg(Context* ctx, poly_t* a) {
  if (a->status == RNSSTATE) poly_copy_to_host(ctx, a);
  int d = (int)a->coefs.size() - 1;
  while (d >= 0 && IsZero(a->coefs[d])) --d;
  return d;
}

// ---------------------------------------------------------------------------
// arithmetic (polynomial.cu:802-1153)
// ---------------------------------------------------------------------------
void poly_add(Context* ctx, poly_t* c, poly_t* a, poly_t* b) {
  same_base(a, b);
  poly_copy_to_device(ctx, a);
  poly_copy_to_device(ctx, b);
  prep_out(ctx, c, a->base);
  DGTEngine::execute_add_dgt(c->d_coefs, a->d_coefs, b->d_coefs, a->base, ctx->get_stream());
  done(c, a->base);
}

void poly_double_add(Context* ctx, poly_t* c1, poly_t* a1, poly_t* b1, poly_t* c2, poly_t* a2, poly_t* b2) {
  same_base(a1, b1);
  same_base(a1, a2);
  same_base(a1, b2);
  for (poly_t* x : {a1, b1, a2, b2}) poly_copy_to_device(ctx, x);
  prep_out(ctx, c1, a1->base);
  prep_out(ctx, c2, a1->base);
  DGTEngine::execute_double_add_dgt(c1->d_coefs, a1->d_coefs, b1->d_coefs, c2->d_coefs, a2->d_coefs, b2->d_coefs,
                                    a1->base, ctx->get_stream());
  done(c1, a1->base);
  done(c2, a1->base);
}

void poly_sub(Context* ctx, poly_t* c, poly_t* a, poly_t* b) {
  same_base(a, b);
  poly_copy_to_device(ctx, a);
  poly_copy_to_device(ctx, b);
  prep_out(ctx, c, a->base);
  DGTEngine::execute_sub_dgt(c->d_coefs, a->d_coefs, b->d_coefs, a->base, ctx->get_stream());
  done(c, a->base);
}

void poly_mul(Context* ctx, poly_t* c, poly_t* a, poly_t* b) {
  same_base(a, b);
  poly_copy_to_device(ctx, a);
  poly_copy_to_device(ctx, b);
  prep_out(ctx, c, a->base);
  DGTEngine::execute_mul_dgt_gi(c->d_coefs, a->d_coefs, b->d_coefs, a->base, ctx->get_stream());
  done(c, a->base);
}

void poly_mul_add(Context* ctx, poly_t* d, poly_t* a, poly_t* b, poly_t* c) {
  same_base(a, b);
  same_base(a, c);
  for (poly_t* x : {a, b, c}) poly_copy_to_device(ctx, x);
  prep_out(ctx, d, a->base);
  DGTEngine::execute_muladd_dgt(d->d_coefs, a->d_coefs, b->d_coefs, c->d_coefs, a->base, ctx->get_stream());
  done(d, a->base);
}

void poly_dr2(Context* ctx, poly_t* ct21, poly_t* ct22, poly_t* ct23, poly_t* ct01, poly_t* ct02, poly_t* ct11,
              poly_t* ct12) {
  same_base(ct01, ct02);
  same_base(ct01, ct11);
  same_base(ct01, ct12);
  const int base = ct01->base;
  for (poly_t* x : {ct01, ct02, ct11, ct12}) poly_copy_to_device(ctx, x);
  for (poly_t* x : {ct21, ct22, ct23}) prep_out(ctx, x, base);
  DGTEngine::execute_dr2_dgt(ct21->d_coefs, ct22->d_coefs, ct23->d_coefs, ct01->d_coefs, ct02->d_coefs,
                             ct11->d_coefs, ct12->d_coefs, base, ctx->get_stream());
  for (poly_t* x : {ct21, ct22, ct23}) done(x, base);
}

static void op_int(Context* ctx, poly_t* b, poly_t* a, uint64_t x, int op) {
  poly_copy_to_device(ctx, a);
  prep_out(ctx, b, a->base);
  CUDAEngine::execute_polynomial_op_by_int(b->d_coefs, a->d_coefs, a->base, x, op, ctx);
  done(b, a->base);
}
void poly_mul_int(Context* ctx, poly_t* c, poly_t* a, uint64_t x) { op_int(ctx, c, a, x, MUL); }
void poly_add_int(Context* ctx, poly_t* c, poly_t* a, uint64_t x) { op_int(ctx, c, a, x, ADD); }
void poly_sub_int(Context* ctx, poly_t* c, poly_t* a, uint64_t x) { op_int(ctx, c, a, x, SUB); }

static void double_op_int(Context* ctx, poly_t* b1, poly_t* a1, poly_t* b2, poly_t* a2, uint64_t x1, uint64_t x2,
                          int op) {
  same_base(a1, a2);
  poly_copy_to_device(ctx, a1);
  poly_copy_to_device(ctx, a2);
  prep_out(ctx, b1, a1->base);
  prep_out(ctx, b2, a1->base);
  CUDAEngine::execute_polynomial_double_op_by_int(b1->d_coefs, a1->d_coefs, b2->d_coefs, a2->d_coefs, a1->base, x1,
                                                  x2, op, ctx);
  done(b1, a1->base);
  done(b2, a1->base);
}
void poly_double_mul_int(Context* ctx, poly_t* b1, poly_t* a1, poly_t* b2, poly_t* a2, uint64_t x1, uint64_t x2) {
  double_op_int(ctx, b1, a1, b2, a2, x1, x2, MULMUL);
}
void poly_double_add_int(Context* ctx, poly_t* b1, poly_t* a1, poly_t* b2, poly_t* a2, uint64_t x1, uint64_t x2) {
  double_op_int(ctx, b1, a1, b2, a2, x1, x2, ADDADD);
}

void poly_div_by_ZZ(Context* ctx, poly_t* c, poly_t* a, NTL::ZZ x) {
  const int deg = poly_get_deg(ctx, a);
  for (int i = 0; i <= deg; ++i) poly_set_coeff(ctx, c, i, poly_get_coeff(ctx, a, i) / x);
}

void poly_mod_by_ZZ(Context* ctx, poly_t* c, poly_t* a, NTL::ZZ x) {
  const int deg = poly_get_deg(ctx, a);
  for (int i = 0; i <= deg; ++i) poly_set_coeff(ctx, c, i, poly_get_coeff(ctx, a, i) % x);
}

void poly_negate(Context* ctx, poly_t* a) {
  require(a->init, "poly_negate: polynomial not initialised");
  poly_copy_to_device(ctx, a);
  CUDAEngine::execute_polynomial_negate(a->d_coefs, a->d_coefs, a->base, ctx);
  a->status = RNSSTATE;
}

void poly_right_shift(Context* ctx, poly_t* b, poly_t* a, int bits) {
  require(a->init, "poly_right_shift: polynomial not initialised");
  poly_init(ctx, b);
  const int deg = poly_get_deg(ctx, a);
  for (int i = 0; i <= deg; ++i) poly_set_coeff(ctx, b, i, poly_get_coeff(ctx, a, i) >> bits);
}

// cuPoly composes one poly_mul and k - 1 poly_mul_add calls (polynomial.cu:1439-1451),
// so when c is also an operand of a later term those calls read the partial sum; that
// case keeps the composition and gives the same bytes.  Otherwise one fused pass.
void poly_dot(Context* ctx, poly_t* c, poly_t* a, poly_t* b, const int k) {
  require(k >= 1, "poly_dot: k must be at least 1");
  bool later_alias = false;
  for (int i = 1; i < k; ++i) later_alias = later_alias || &a[i] == c || &b[i] == c;
  if (later_alias) {
    poly_mul(ctx, c, &a[0], &b[0]);
    for (int i = 1; i < k; ++i) poly_mul_add(ctx, c, &a[i], &b[i], c);
    return;
  }
  const int base = a[0].base;
  std::vector<const void*> pa(k), pb(k);
  for (int i = 0; i < k; ++i) {
    same_base(&a[0], &a[i]);
    same_base(&a[0], &b[i]);
    poly_copy_to_device(ctx, &a[i]);
    poly_copy_to_device(ctx, &b[i]);
  }
  prep_out(ctx, c, base);
  for (int i = 0; i < k; ++i) {
    pa[i] = a[i].d_coefs;
    pb[i] = b[i].d_coefs;
  }
  check(cp_dot(E(), c->d_coefs, pa.data(), pb.data(), k, base, S(ctx)), "poly_dot");
  done(c, base);
}

// ---------------------------------------------------------------------------
// HPS and decomposition (polynomial.cu:310-693)
// ---------------------------------------------------------------------------
void poly_simple_scaling_tDivQ(Context* ctx, poly_t* b, poly_t* a) {
  require(a->base == QBase, "poly_simple_scaling_tDivQ: input must lie in Q");
  poly_copy_to_device(ctx, a);
  prep_out(ctx, b, TBase);
  check(cp_poly_simple_scaling_tdivq(E(), b->d_coefs, a->d_coefs, ctx->workspace(), S(ctx)),
        "poly_simple_scaling_tDivQ");
  done(b, TBase);
}

void poly_complex_scaling_tDivQ(Context* ctx, poly_t* b, poly_t* a_Q, poly_t* a_B) {
  require(a_Q->base == QBase && a_B->base == BBase, "poly_complex_scaling_tDivQ: inputs must lie in Q and B");
  poly_copy_to_device(ctx, a_Q);
  poly_copy_to_device(ctx, a_B);
  prep_out(ctx, b, QBase);
  check(cp_poly_complex_scaling_tdivq(E(), b->d_coefs, a_Q->d_coefs, a_B->d_coefs, 0u, ctx->workspace(), S(ctx)),
        "poly_complex_scaling_tDivQ");
  done(b, QBase);
}

void poly_basis_extension_Q_to_B(Context* ctx, poly_t* a_B, poly_t* a_Q) {
  require(a_Q->base == QBase, "poly_basis_extension_Q_to_B: input must lie in Q");
  poly_copy_to_device(ctx, a_Q);
  prep_out(ctx, a_B, BBase);
  check(cp_poly_basis_extension_q_to_b(E(), a_B->d_coefs, a_Q->d_coefs, ctx->workspace(), S(ctx)),
        "poly_basis_extension_Q_to_B");
  done(a_B, BBase);
}

void poly_basis_extension_Q_to_QB(Context* ctx, poly_t* b, poly_t* a) {
  require(a->base == QBase, "poly_basis_extension_Q_to_QB: input must lie in Q");
  poly_copy_to_device(ctx, a);
  prep_out(ctx, b, QBBase);
  check(cp_poly_basis_extension_q_to_qb(E(), b->d_coefs, a->d_coefs, ctx->workspace(), S(ctx)),
        "poly_basis_extension_Q_to_QB");
  done(b, QBBase);
}

void poly_basis_extension_B_to_Q(Context* ctx, poly_t* a_Q, poly_t* a_B) {
  require(a_B->base == BBase, "poly_basis_extension_B_to_Q: input must lie in B");
  poly_copy_to_device(ctx, a_B);
  prep_out(ctx, a_Q, QBase);
  check(cp_poly_basis_extension_b_to_q(E(), a_Q->d_coefs, a_B->d_coefs, ctx->workspace(), S(ctx)),
        "poly_basis_extension_B_to_Q");
  done(a_Q, QBase);
}

static void xi_rho(Context* ctx, poly_t* c, poly_t* a, bool rho) {
  require(a->base == QBase, "xi / rho: input must lie in Q");
  poly_copy_to_device(ctx, a);
  const int k = nres(QBase);
  const size_t qb = res_bytes(QBase);
  void* out = ctx->scratch(qb * k);
  check((rho ? cp_rho : cp_xi)(E(), out, a->d_coefs, S(ctx)), rho ? "poly_rho_bfv" : "poly_xi_bfv");
  for (int i = 0; i < k; ++i) {
    prep_out(ctx, &c[i], QBase);
    d2d(c[i].d_coefs, static_cast<char*>(out) + qb * i, qb, ctx);
    done(&c[i], QBase);
  }
  sync(ctx);  // the scratch is reused by the next call
}
void poly_xi_bfv(Context* ctx, poly_t* c, poly_t* a) { xi_rho(ctx, c, a, false); }
void poly_rho_bfv(Context* ctx, poly_t* c, poly_t* a) { xi_rho(ctx, c, a, true); }

// ---------------------------------------------------------------------------
// CKKS (polynomial.cu:530-608, 696-800)
// ---------------------------------------------------------------------------
void poly_approx_basis_raising_Q_to_QB(Context* ctx, poly_t* a, poly_t* b, int level) {
  require(b->base == QBase, "poly_approx_basis_raising_Q_to_QB: input must lie in Q");
  poly_copy_to_device(ctx, b);
  prep_out(ctx, a, QBBase);
  check(cp_ckks_modulus_raising(E(), a->d_coefs, b->d_coefs, level, ctx->workspace(), S(ctx)),
        "poly_approx_basis_raising_Q_to_QB");
  done(a, QBBase);
}

void poly_approx_basis_reduction_QB_to_Q(Context* ctx, poly_t* a, poly_t* b, int level) {
  require(b->base == QBBase, "poly_approx_basis_reduction_QB_to_Q: input must lie in QB");
  poly_copy_to_device(ctx, b);
  prep_out(ctx, a, QBase);
  poly_copy_to_device(ctx, a);
  check(cp_ckks_modulus_reduction(E(), a->d_coefs, b->d_coefs, level, ctx->workspace(), S(ctx)),
        "poly_approx_basis_reduction_QB_to_Q");
  done(a, QBase);
}

void poly_ckks_rescale(Context* ctx, poly_t* a, poly_t* b, int level) {
  require(a->init && a->base == QBase, "poly_ckks_rescale: input must lie in Q");
  poly_copy_to_device(ctx, a);
  if (b) poly_copy_to_device(ctx, b);
  check(cp_ckks_rescale(E(), a->d_coefs, b ? b->d_coefs : nullptr, level, S(ctx)), "poly_ckks_rescale");
  a->status = RNSSTATE;
  if (b) b->status = RNSSTATE;
}

void poly_xi_ckks(Context* ctx, poly_t* c, poly_t* a) {
  require(a->init && a->base == QBase, "poly_xi_ckks: input must lie in Q");
  poly_copy_to_device(ctx, a);
  prep_out(ctx, c, QBase);
  check(cp_ckks_xi(E(), c->d_coefs, a->d_coefs, S(ctx)), "poly_xi_ckks");
  done(c, QBase);
}

void poly_rho_ckks(Context* ctx, poly_t* c, poly_t* a) {
  require(a->init && (a->base == QBase || a->base == QBBase), "poly_rho_ckks: input must lie in Q or QB");
  poly_copy_to_device(ctx, a);
  prep_out(ctx, c, QBase);
  check(cp_ckks_rho(E(), c->d_coefs, a->d_coefs, S(ctx)), "poly_rho_ckks");
  done(c, QBase);
}

// ---------------------------------------------------------------------------
// coefficients and text forms (polynomial.cu:1181-1437)
// ---------------------------------------------------------------------------
std::string poly_to_string(Context* ctx, poly_t* a) {
  std::ostringstream oss;
  const int deg = poly_get_deg(ctx, a);
  for (int i = 0; i <= deg; ++i) oss << poly_get_coeff(ctx, a, i) << ", ";
  return oss.str();
}

void poly_set_coeff(Context* ctx, poly_t* a, unsigned int index, NTL::ZZ c) {
  if (!a->init) poly_init(ctx, a);
  require((int)index < nphi(), "poly_set_coeff: index out of range");
  poly_copy_to_host(ctx, a);
  if (c < NTL::ZZ(0)) c = CUDAEngine::RNSProduct + c;  // negatives as Q + c
  if (index >= a->coefs.size()) a->coefs.resize(index + 1, NTL::ZZ(0));
  a->coefs[index] = c;
  a->status = HOSTSTATE;
}

NTL::ZZ poly_get_coeff(Context* ctx, poly_t* a, int index) {
  require(a->init, "poly_get_coeff: polynomial not initialised");
  poly_copy_to_host(ctx, a);
  if (index < 0 || (size_t)index >= a->coefs.size()) return NTL::ZZ(0);
  return a->coefs[index];
}

bool poly_are_equal(Context* ctx, poly_t* a, poly_t* b) {
  require(a->init && b->init, "poly_are_equal: polynomial not initialised");
  const int deg = poly_get_deg(ctx, a);
  if (deg != poly_get_deg(ctx, b)) return false;
  const NTL::ZZ& q = CUDAEngine::RNSProduct;
  for (int i = 0; i <= deg; ++i)
    if (poly_get_coeff(ctx, a, i) % q != poly_get_coeff(ctx, b, i) % q) return false;
  return true;
}

NTL::ZZ poly_infty_norm(Context* ctx, poly_t* p) {
  NTL::ZZ x(0);
  const int deg = poly_get_deg(ctx, p);
  for (int i = 0; i <= deg; ++i) {
    const NTL::ZZ c = poly_get_coeff(ctx, p, i);
    if (c > x) x = c;
  }
  return x;
}

std::string poly_export(Context* ctx, poly_t* p) {
  std::ostringstream oss;
  const int deg = poly_get_deg(ctx, p);
  for (int i = 0; i <= deg; ++i) oss << poly_get_coeff(ctx, p, i) << (i < deg ? "," : "");
  return oss.str();
}

poly_t* poly_import(Context* ctx, std::string s) {
  poly_t* p = new poly_t;
  poly_init(ctx, p);
  if (!s.empty()) {
    std::vector<NTL::ZZ> v;
    std::string cur;
    for (size_t i = 0; i <= s.size(); ++i) {
      if (i == s.size() || s[i] == ',') {
        v.push_back(zz_from_decimal(cur.empty() ? std::string("0") : cur));
        cur.clear();
      } else if (s[i] != ' ') {
        cur += s[i];
      }
    }
    for (size_t i = 0; i < v.size(); ++i) poly_set_coeff(ctx, p, (unsigned)i, v[i]);
  }
  return p;
}

// Coefficient-domain residues of a on the host: word (r, j) at r * nphi + j.
static void host_residues(Context* ctx, poly_t* a, std::vector<uint64_t>& out) {
  require(a->init, "residue access: polynomial not initialised");
  GaussianInteger* aux = coefficient_residues(ctx, a);
  const int nr = nres(a->base), N = CUDAEngine::N;
  std::vector<GaussianInteger> h((size_t)nr * N);
  cuda_check(cudaMemcpyAsync(h.data(), aux, res_bytes(a->base), cudaMemcpyDeviceToHost, ctx->get_stream()),
             "cudaMemcpyAsync");
  sync(ctx);
  out.assign((size_t)nr * 2 * N, 0);
  for (int r = 0; r < nr; ++r)
    for (int j = 0; j < N; ++j) {
      out[(size_t)r * 2 * N + j] = h[(size_t)r * N + j].re;
      out[(size_t)r * 2 * N + N + j] = h[(size_t)r * N + j].imag;
    }
}

std::string poly_export_residues(Context* ctx, poly_t* p) {
  std::vector<uint64_t> v;
  host_residues(ctx, p, v);
  std::ostringstream oss;
  for (size_t i = 0; i < v.size(); ++i) oss << (int64_t)v[i] << (i + 1 < v.size() ? " " : "");
  return oss.str();
}

poly_t* poly_import_residues(Context* ctx, std::string s, int base) {
  const int nr = nres(base), N = CUDAEngine::N;
  std::vector<GaussianInteger> h((size_t)nr * N, GaussianInteger{0, 0});
  std::istringstream iss(s);
  long long val;
  size_t i = 0;
  while (iss >> val && i < (size_t)nr * 2 * N) {
    const size_t cid = i % (2 * N), rid = i / (2 * N);
    if (cid < (size_t)N)
      h[rid * N + cid].re = (uint64_t)val;
    else
      h[rid * N + cid - N].imag = (uint64_t)val;
    ++i;
  }
  poly_t* a = new poly_t;
  poly_init(ctx, a, base);
  cuda_check(cudaMemcpyAsync(a->d_coefs, h.data(), res_bytes(base), cudaMemcpyHostToDevice, ctx->get_stream()),
             "cudaMemcpyAsync");
  DGTEngine::execute_dgt(a->d_coefs, base, FORWARD, ctx);
  sync(ctx);
  a->base = base;
  a->status = RNSSTATE;
  return a;
}

std::vector<unsigned char> poly_export_binary(Context* ctx, poly_t* p) {
  poly_copy_to_device(ctx, p);
  std::vector<unsigned char> out(cp_wire_bytes(E(), p->base, 1));
  check(cp_export_residues(E(), out.data(), out.size(), p->d_coefs, p->base, 1, 1, S(ctx)), "poly_export_binary");
  return out;
}

poly_t* poly_import_binary(Context* ctx, const std::vector<unsigned char>& data, int base) {
  poly_t* a = new poly_t;
  poly_init(ctx, a, base);
  int domain = -1;
  const int rc = cp_import_residues(E(), a->d_coefs, data.data(), data.size(), base, 1, &domain, S(ctx));
  if (rc != CP_OK) {
    poly_free(ctx, a);
    delete a;
    check(rc, "poly_import_binary");
  }
  if (domain == 0) DGTEngine::execute_dgt(a->d_coefs, base, FORWARD, ctx);
  sync(ctx);
  a->base = base;
  a->status = RNSSTATE;
  return a;
}

std::string poly_residue_to_string(Context* ctx, poly_t* a, int id) {
  require(id >= 0 && id < nres(a->base), "poly_residue_to_string: bad residue index");
  std::vector<uint64_t> v;
  host_residues(ctx, a, v);
  std::ostringstream oss;
  for (int j = 0; j < nphi(); ++j) oss << v[(size_t)id * nphi() + j] << ",";
  return oss.str();
}

uint64_t* poly_get_residue(Context* ctx, uint64_t* b, poly_t* a, int id) {
  require(id >= 0 && id < nres(a->base), "poly_get_residue: bad residue index");
  std::vector<uint64_t> v;
  host_residues(ctx, a, v);
  uint64_t* r = b ? b : static_cast<uint64_t*>(std::malloc((size_t)nphi() * sizeof(uint64_t)));
  require(r != nullptr, "poly_get_residue: out of host memory");
  std::copy(v.begin() + (size_t)id * nphi(), v.begin() + (size_t)(id + 1) * nphi(), r);
  return r;
}

uint64_t* poly_get_residues(Context* ctx, poly_t* a) {
  std::vector<uint64_t> v;
  host_residues(ctx, a, v);
  uint64_t* r = static_cast<uint64_t*>(std::malloc(v.size() * sizeof(uint64_t)));
  require(r != nullptr, "poly_get_residues: out of host memory");
  std::copy(v.begin(), v.end(), r);
  return r;
}

void poly_select_residue(Context* ctx, poly_t* p, int id) {
  require(p->init && id >= 0 && id < nres(p->base), "poly_select_residue: bad polynomial or residue index");
  poly_copy_to_device(ctx, p);
  const int nr = nres(p->base), N = CUDAEngine::N;
  DGTEngine::execute_dgt(p->d_coefs, p->base, INVERSE, ctx);
  for (int i = 0; i < nr; ++i)
    if (i != id) d2d(p->d_coefs + (size_t)i * N, p->d_coefs + (size_t)id * N, (size_t)N * sizeof(GaussianInteger), ctx);
  // residue id's values may exceed a smaller prime: reduce every residue (x * 1 mod q_i)
  CUDAEngine::execute_polynomial_op_by_int(p->d_coefs, p->d_coefs, p->base, 1, MUL, ctx);
  DGTEngine::execute_dgt(p->d_coefs, p->base, FORWARD, ctx);
  p->status = RNSSTATE;
}

void poly_discard_qbase(Context* ctx, poly_t* p) {
  poly_copy_to_device(ctx, p);
  if (p->base == BBase) return;
  require(p->base == QBBase, "poly_discard_qbase: polynomial must lie in QB");
  const size_t off = (size_t)nres(QBase) * CUDAEngine::N;
  // overlapping ranges when kl > k: move through the aux buffer
  GaussianInteger* aux = ctx->aux();
  d2d(aux, p->d_coefs + off, res_bytes(BBase), ctx);
  d2d(p->d_coefs, aux, res_bytes(BBase), ctx);
  p->base = BBase;
  p->status = RNSSTATE;
}

// ---------------------------------------------------------------------------
// Sampler (sampler.cu:576-645)
// ---------------------------------------------------------------------------
uint64_t Sampler::seed = SEED;
uint32_t Sampler::counter = 0;

void Sampler::init(Context*) { counter = 0; }
void Sampler::reset(Context*) { counter = 0; }

// cuPoly's names keep cuPoly's meanings; the layer-only kinds select the
// library's independent forms.  cuPoly's CKKS UNIFORM is per residue already.
static int device_kind(int kind) {
  switch (kind) {
    case UNIFORM: return CUDAEngine::scalingfactor ? CP_UNIFORM : CP_UNIFORM_U32;
    case ZO: return CP_ZO_HALF;
    case UNIFORM_MOD_Q: return CP_UNIFORM;
    case ZO_IID: return CP_ZO;
    default: return kind;
  }
}

void Sampler::sample(Context* ctx, poly_t* p, int kind) {
  poly_init(ctx, p);
  check(cp_sample(E(), p->d_coefs, p->base, device_kind(kind), seed, counter++, 1, 1, S(ctx)), "Sampler::sample");
  p->status = RNSSTATE;
}

poly_t* Sampler::sample(Context* ctx, int kind) {
  poly_t* p = new poly_t;
  sample(ctx, p, kind);
  return p;
}
