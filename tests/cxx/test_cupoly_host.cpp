// C++ tests of the cuPoly host layer (libcupoly.so over libcupoly_b200.so), written
// the way cuPoly's own gtests are (tests/unit_tests/test_bfv_mode.cu:243-1487): the
// same fixtures (CUDAEngine::init(k, k + 1, nphi, 256), a Context, Sampler::init),
// the same test names and the same (log2 q, nphi) grid (:1492-1508, k = ceil(log2 q / 63)).
// cuPoly checks against NTL (ZZX products mod x^nphi + 1, ZZ arithmetic); here the
// check is big-integer arithmetic on the in-repo ZZ: every coefficient for the
// elementwise operations, and the negacyclic convolution for every coefficient when
// nphi <= 256 and for 24 sampled coefficients above.  No gtest in this image, so a
// small registry stands in for TEST_P.
//
//   test_cupoly_host [--quick] [substring]
// Exit status 0 when every test passes.
#include <cuPoly/arithmetic/polynomial.h>
#include <cuPoly/cuda/sampler.h>

#include <cmath>
#include <cstdio>
#include <functional>
#include <random>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct Params {
  int logq2;
  int nphi;
};

struct Failure {
  std::string msg;
};

#define CHECK(cond, what)                                                                 \
  do {                                                                                    \
    if (!(cond)) {                                                                        \
      std::ostringstream oss_;                                                            \
      oss_ << __FILE__ << ":" << __LINE__ << ": " << #cond << " -- " << what;             \
      throw Failure{oss_.str()};                                                          \
    }                                                                                     \
  } while (0)

struct Fixture {
  int k, nphi;
  uint64_t t = 256;
  ZZ q;
  Context* ctx = nullptr;
  std::mt19937_64 rng{0};
  explicit Fixture(const Params& p) : k((p.logq2 + 62) / 63), nphi(p.nphi) {
    CUDAEngine::init(k, k + 1, nphi, t);
    q = CUDAEngine::RNSProduct;
    ctx = new Context();
    Sampler::init(ctx);
  }
  ~Fixture() {
    delete ctx;
    Sampler::destroy();
    CUDAEngine::destroy();
  }
  ZZ random_below(const ZZ& m) {
    ZZ x(0);
    for (long b = 0; b < NumBits(m) + 64; b += 64) x = (x << 64) + ZZ((unsigned long)rng());
    return x % m;
  }
  void random_poly(poly_t* a, int base = QBase, const ZZ* bound = nullptr) {
    poly_init(ctx, a, base);
    const ZZ m = bound ? *bound : q;
    for (int i = 0; i < nphi; ++i) poly_set_coeff(ctx, a, i, random_below(m));
  }
  std::vector<ZZ> coeffs(poly_t* a) {
    std::vector<ZZ> v(nphi);
    for (int i = 0; i < nphi; ++i) v[i] = poly_get_coeff(ctx, a, i);
    return v;
  }
  // coefficient j of a b mod (x^nphi + 1, m)
  ZZ negacyclic(const std::vector<ZZ>& a, const std::vector<ZZ>& b, int j, const ZZ& m) {
    ZZ s(0);
    for (int i = 0; i <= j; ++i) s += a[i] * b[j - i];
    for (int i = j + 1; i < nphi; ++i) s -= a[i] * b[nphi + j - i];
    return s % m;
  }
  std::vector<int> check_indices() {
    std::vector<int> idx;
    if (nphi <= 256) {
      for (int i = 0; i < nphi; ++i) idx.push_back(i);
    } else {
      idx = {0, 1, nphi / 2 - 1, nphi / 2, nphi - 1};
      while (idx.size() < 24) idx.push_back((int)(rng() % nphi));
    }
    return idx;
  }
};

using TestFn = std::function<void(Fixture&)>;
std::vector<std::pair<std::string, TestFn>>& registry() {
  static std::vector<std::pair<std::string, TestFn>> r;
  return r;
}
struct Reg {
  Reg(const char* name, TestFn f) { registry().emplace_back(name, std::move(f)); }
};
#define TEST_F(suite, name)                                  \
  void suite##_##name(Fixture& F);                           \
  static Reg reg_##suite##_##name(#suite "." #name, suite##_##name); \
  void suite##_##name(Fixture& F)

uint64_t as_u64(const ZZ& x) { return (uint64_t)to_ulong(x); }

// ---------------------------------------------------------------------------
// TestDGT
// ---------------------------------------------------------------------------
TEST_F(TestDGT, RoundTrip) {
  poly_t a;
  Sampler::sample(F.ctx, &a, UNIFORM);
  const size_t bytes = poly_get_residues_size(QBase);
  std::vector<GaussianInteger> before(bytes / 16), after(bytes / 16);
  cudaMemcpy(before.data(), a.d_coefs, bytes, cudaMemcpyDeviceToHost);
  DGTEngine::execute_dgt(a.d_coefs, QBase, INVERSE, F.ctx);
  DGTEngine::execute_dgt(a.d_coefs, QBase, FORWARD, F.ctx);
  cudaStreamSynchronize(F.ctx->get_stream());
  cudaMemcpy(after.data(), a.d_coefs, bytes, cudaMemcpyDeviceToHost);
  for (size_t i = 0; i < before.size(); ++i) CHECK(before[i] == after[i], "element " << i);
  poly_free(F.ctx, &a);
}

TEST_F(TestDGT, MulByDGTEngine) {
  // DGTEngine::execute_mul_dgt_gi on raw buffers is the negacyclic product
  poly_t a, b, c;
  F.random_poly(&a);
  F.random_poly(&b);
  poly_copy_to_device(F.ctx, &a);
  poly_copy_to_device(F.ctx, &b);
  poly_init(F.ctx, &c);
  DGTEngine::execute_mul_dgt_gi(c.d_coefs, a.d_coefs, b.d_coefs, QBase, F.ctx->get_stream());
  c.status = RNSSTATE;
  const auto va = F.coeffs(&a), vb = F.coeffs(&b), vc = F.coeffs(&c);
  for (int j : F.check_indices()) CHECK(vc[j] == F.negacyclic(va, vb, j, F.q), "index " << j);
  for (poly_t* x : {&a, &b, &c}) poly_free(F.ctx, x);
}

// ---------------------------------------------------------------------------
// TestRNS
// ---------------------------------------------------------------------------
TEST_F(TestRNS, RNS) {
  // coefficients up to twice the width of Q come back reduced mod Q
  poly_t a;
  poly_init(F.ctx, &a);
  const ZZ big = F.q * F.q;
  std::vector<ZZ> v(F.nphi);
  for (int i = 0; i < F.nphi; ++i) {
    v[i] = F.random_below(big);
    poly_set_coeff(F.ctx, &a, i, v[i]);
  }
  poly_copy_to_device(F.ctx, &a);
  a.status = RNSSTATE;  // force the device -> host path
  for (int i = 0; i < F.nphi; ++i) CHECK(poly_get_coeff(F.ctx, &a, i) == v[i] % F.q, "index " << i);
  poly_free(F.ctx, &a);
}

TEST_F(TestRNS, Serializing) {
  poly_t a;
  F.random_poly(&a);
  poly_t* b = poly_import(F.ctx, poly_export(F.ctx, &a));
  CHECK(poly_are_equal(F.ctx, &a, b), "poly_export / poly_import");
  poly_t* c = poly_import_residues(F.ctx, poly_export_residues(F.ctx, &a));
  CHECK(poly_are_equal(F.ctx, &a, c), "poly_export_residues / poly_import_residues");
  poly_t* d = poly_import_binary(F.ctx, poly_export_binary(F.ctx, &a));
  CHECK(poly_are_equal(F.ctx, &a, d), "binary wire form");
  for (poly_t* x : {&a, b, c, d}) poly_free(F.ctx, x);
  delete b;
  delete c;
  delete d;
}

TEST_F(TestRNS, SimpleBasisExtensionUniformQtoB) {
  poly_t a, ab;
  F.random_poly(&a);
  const auto va = F.coeffs(&a);
  poly_basis_extension_Q_to_B(F.ctx, &ab, &a);
  CHECK(ab.base == BBase, "output base");
  for (size_t j = 0; j < CUDAEngine::RNSBPrimes.size(); ++j) {
    uint64_t* r = poly_get_residue(F.ctx, NULL, &ab, (int)j);
    const ZZ bj((unsigned long)CUDAEngine::RNSBPrimes[j]);
    for (int i = 0; i < F.nphi; ++i) CHECK(r[i] == as_u64(va[i] % bj), "residue " << j << " index " << i);
    free(r);
  }
  poly_free(F.ctx, &a);
  poly_free(F.ctx, &ab);
}

TEST_F(TestRNS, SimpleBasisExtensionUniformQtoQB) {
  poly_t a, aqb;
  F.random_poly(&a);
  const auto va = F.coeffs(&a);
  poly_basis_extension_Q_to_QB(F.ctx, &aqb, &a);
  CHECK(aqb.base == QBBase, "output base");
  const int k = (int)CUDAEngine::RNSPrimes.size();
  for (int j = 0; j < CUDAEngine::get_n_residues(QBBase); ++j) {
    uint64_t* r = poly_get_residue(F.ctx, NULL, &aqb, j);
    const uint64_t m = j < k ? CUDAEngine::RNSPrimes[j] : CUDAEngine::RNSBPrimes[j - k];
    for (int i = 0; i < F.nphi; ++i) CHECK(r[i] == as_u64(va[i] % ZZ((unsigned long)m)), "residue " << j);
    free(r);
  }
  poly_free(F.ctx, &a);
  poly_free(F.ctx, &aqb);
}

TEST_F(TestRNS, SimpleBasisExtensionUniformBtoQ) {
  poly_t ab, aq;
  const ZZ B = CUDAEngine::RNSBProduct;
  F.random_poly(&ab, BBase, &B);
  const auto vb = F.coeffs(&ab);
  poly_basis_extension_B_to_Q(F.ctx, &aq, &ab);
  for (int i = 0; i < F.nphi; ++i) CHECK(poly_get_coeff(F.ctx, &aq, i) == vb[i] % F.q, "index " << i);
  poly_free(F.ctx, &ab);
  poly_free(F.ctx, &aq);
}

TEST_F(TestRNS, SimpleScalingtDivQ) {
  poly_t a, b;
  F.random_poly(&a);
  const auto va = F.coeffs(&a);
  poly_simple_scaling_tDivQ(F.ctx, &b, &a);
  CHECK(b.base == TBase, "output base");
  const ZZ t((unsigned long)F.t);
  for (int i = 0; i < F.nphi; ++i) {
    const ZZ want = ((va[i] * t * 2 + F.q) / (F.q * 2)) % t;  // round(t X / Q) mod t
    CHECK(poly_get_coeff(F.ctx, &b, i) == want, "index " << i);
  }
  poly_free(F.ctx, &a);
  poly_free(F.ctx, &b);
}

TEST_F(TestRNS, ComplexBasisScalingUniform) {
  // X uniform in [0, QB) given by its Q and B residues; b = (round(t X / Q) mod B) mod Q
  const ZZ B = CUDAEngine::RNSBProduct, QB = F.q * B, t((unsigned long)F.t);
  poly_t x, aq, ab, b;
  F.random_poly(&x, QBBase, &QB);
  const auto vx = [&] {  // host coefficients of the QB polynomial, as set
    std::vector<ZZ> v(F.nphi);
    for (int i = 0; i < F.nphi; ++i) v[i] = x.coefs[i];
    return v;
  }();
  poly_init(F.ctx, &aq);
  for (int i = 0; i < F.nphi; ++i) poly_set_coeff(F.ctx, &aq, i, vx[i] % F.q);
  poly_copy(F.ctx, &ab, &x);
  poly_discard_qbase(F.ctx, &ab);
  poly_complex_scaling_tDivQ(F.ctx, &b, &aq, &ab);
  for (int i = 0; i < F.nphi; ++i) {
    const ZZ want = (((vx[i] * t * 2 + F.q) / (F.q * 2)) % B) % F.q;
    CHECK(poly_get_coeff(F.ctx, &b, i) == want, "index " << i);
  }
  for (poly_t* p : {&x, &aq, &ab, &b}) poly_free(F.ctx, p);
}

TEST_F(TestRNS, XiRho) {
  poly_t a;
  F.random_poly(&a);
  const auto va = F.coeffs(&a);
  const int k = F.k;
  std::vector<poly_t> xi(k), rho(k);
  poly_xi_bfv(F.ctx, xi.data(), &a);
  poly_rho_bfv(F.ctx, rho.data(), &a);
  for (int i = 0; i < k; ++i) {
    const ZZ qi((unsigned long)CUDAEngine::RNSPrimes[i]);
    const ZZ inv((unsigned long)CUDAEngine::RNSInvMpi[i]);
    const ZZ mpi = CUDAEngine::RNSMpi[i] % qi;
    for (int j = 0; j < k; ++j) {
      uint64_t* rx = poly_get_residue(F.ctx, NULL, &xi[i], j);
      uint64_t* rr = poly_get_residue(F.ctx, NULL, &rho[i], j);
      for (int c = 0; c < F.nphi; ++c) {
        CHECK(rx[c] == (j == i ? as_u64((va[c] % qi) * inv % qi) : 0), "xi " << i << " residue " << j);
        CHECK(rr[c] == (j == i ? as_u64((va[c] % qi) * mpi % qi) : 0), "rho " << i << " residue " << j);
      }
      free(rx);
      free(rr);
    }
    poly_free(F.ctx, &xi[i]);
    poly_free(F.ctx, &rho[i]);
  }
  poly_free(F.ctx, &a);
}

// ---------------------------------------------------------------------------
// TestArithmetic
// ---------------------------------------------------------------------------
TEST_F(TestArithmetic, SetCoeff) {
  poly_t a;
  poly_init(F.ctx, &a);
  std::vector<ZZ> v(F.nphi);
  for (int i = 0; i < F.nphi; ++i) {
    v[i] = F.random_below(F.q);
    poly_set_coeff(F.ctx, &a, i, v[i]);
  }
  poly_set_coeff(F.ctx, &a, 0, to_ZZ(-5));
  v[0] = F.q - 5;
  poly_copy_to_device(F.ctx, &a);
  a.status = RNSSTATE;
  for (int i = 0; i < F.nphi; ++i) CHECK(poly_get_coeff(F.ctx, &a, i) == v[i], "index " << i);
  CHECK(poly_get_coeff(F.ctx, &a, F.nphi + 3) == ZZ(0), "beyond the degree");
  poly_free(F.ctx, &a);
}

TEST_F(TestArithmetic, Add) {
  poly_t a, b, c;
  Sampler::sample(F.ctx, &a, UNIFORM);
  Sampler::sample(F.ctx, &b, UNIFORM);
  poly_add(F.ctx, &c, &a, &b);
  for (int i = 0; i < F.nphi; ++i)
    CHECK((poly_get_coeff(F.ctx, &a, i) + poly_get_coeff(F.ctx, &b, i)) % F.q == poly_get_coeff(F.ctx, &c, i),
          "index " << i);
  for (poly_t* x : {&a, &b, &c}) poly_free(F.ctx, x);
}

TEST_F(TestArithmetic, Sub) {
  poly_t a, b, c;
  Sampler::sample(F.ctx, &a, UNIFORM);
  Sampler::sample(F.ctx, &b, UNIFORM);
  poly_sub(F.ctx, &c, &a, &b);
  for (int i = 0; i < F.nphi; ++i)
    CHECK((poly_get_coeff(F.ctx, &a, i) - poly_get_coeff(F.ctx, &b, i)) % F.q == poly_get_coeff(F.ctx, &c, i),
          "index " << i);
  for (poly_t* x : {&a, &b, &c}) poly_free(F.ctx, x);
}

TEST_F(TestArithmetic, Mul) {
  poly_t a, b, c;
  Sampler::sample(F.ctx, &a, UNIFORM);
  Sampler::sample(F.ctx, &b, UNIFORM);
  poly_mul(F.ctx, &c, &a, &b);
  const auto va = F.coeffs(&a), vb = F.coeffs(&b), vc = F.coeffs(&c);
  for (int j : F.check_indices()) CHECK(vc[j] == F.negacyclic(va, vb, j, F.q), "index " << j);
  for (poly_t* x : {&a, &b, &c}) poly_free(F.ctx, x);
}

TEST_F(TestArithmetic, MulAdd) {
  poly_t a, b, c, d;
  Sampler::sample(F.ctx, &a, UNIFORM);
  Sampler::sample(F.ctx, &b, UNIFORM);
  Sampler::sample(F.ctx, &c, UNIFORM);
  poly_mul_add(F.ctx, &d, &a, &b, &c);
  const auto va = F.coeffs(&a), vb = F.coeffs(&b), vc = F.coeffs(&c), vd = F.coeffs(&d);
  for (int j : F.check_indices()) CHECK(vd[j] == (F.negacyclic(va, vb, j, F.q) + vc[j]) % F.q, "index " << j);
  for (poly_t* x : {&a, &b, &c, &d}) poly_free(F.ctx, x);
}

TEST_F(TestArithmetic, MulBaseB) {
  // products in the auxiliary base: extend to B, multiply there, compare mod B
  poly_t a, b, ab, bb, cb;
  F.random_poly(&a);
  F.random_poly(&b);
  poly_basis_extension_Q_to_B(F.ctx, &ab, &a);
  poly_basis_extension_Q_to_B(F.ctx, &bb, &b);
  poly_mul(F.ctx, &cb, &ab, &bb);
  const ZZ B = CUDAEngine::RNSBProduct;
  const auto va = F.coeffs(&a), vb = F.coeffs(&b), vc = F.coeffs(&cb);
  for (int j : F.check_indices()) CHECK(vc[j] == F.negacyclic(va, vb, j, B), "index " << j);
  for (poly_t* x : {&a, &b, &ab, &bb, &cb}) poly_free(F.ctx, x);
}

TEST_F(TestArithmetic, DR2) {
  poly_t a0, a1, b0, b1, c0, c1, c2;
  for (poly_t* x : {&a0, &a1, &b0, &b1}) Sampler::sample(F.ctx, x, UNIFORM_MOD_Q);
  poly_dr2(F.ctx, &c0, &c1, &c2, &a0, &a1, &b0, &b1);
  const auto A0 = F.coeffs(&a0), A1 = F.coeffs(&a1), B0 = F.coeffs(&b0), B1 = F.coeffs(&b1);
  const auto C0 = F.coeffs(&c0), C1 = F.coeffs(&c1), C2 = F.coeffs(&c2);
  for (int j : F.check_indices()) {
    CHECK(C0[j] == F.negacyclic(A0, B0, j, F.q), "c0 index " << j);
    CHECK(C1[j] == (F.negacyclic(A0, B1, j, F.q) + F.negacyclic(A1, B0, j, F.q)) % F.q, "c1 index " << j);
    CHECK(C2[j] == F.negacyclic(A1, B1, j, F.q), "c2 index " << j);
  }
  for (poly_t* x : {&a0, &a1, &b0, &b1, &c0, &c1, &c2}) poly_free(F.ctx, x);
}

TEST_F(TestArithmetic, MulByInt) {
  poly_t a, b, c, d, e;
  Sampler::sample(F.ctx, &a, UNIFORM);
  const uint64_t x = F.rng() % 1000003;
  poly_mul_int(F.ctx, &b, &a, x);
  poly_add_int(F.ctx, &c, &a, x);
  poly_sub_int(F.ctx, &d, &a, x);
  poly_copy(F.ctx, &e, &a);
  poly_negate(F.ctx, &e);
  const ZZ X((unsigned long)x);
  for (int i = 0; i < F.nphi; ++i) {
    const ZZ ai = poly_get_coeff(F.ctx, &a, i);
    CHECK(poly_get_coeff(F.ctx, &b, i) == ai * X % F.q, "mul index " << i);
    CHECK(poly_get_coeff(F.ctx, &c, i) == (i == 0 ? (ai + X) % F.q : ai), "add index " << i);
    CHECK(poly_get_coeff(F.ctx, &d, i) == (i == 0 ? (ai - X) % F.q : ai), "sub index " << i);
    CHECK(poly_get_coeff(F.ctx, &e, i) == (F.q - ai) % F.q, "negate index " << i);
  }
  for (poly_t* p : {&a, &b, &c, &d, &e}) poly_free(F.ctx, p);
}

TEST_F(TestArithmetic, Dot) {
  poly_t a[3], b[3], c;
  for (int i = 0; i < 3; ++i) {
    Sampler::sample(F.ctx, &a[i], UNIFORM_MOD_Q);
    Sampler::sample(F.ctx, &b[i], UNIFORM_MOD_Q);
  }
  poly_dot(F.ctx, &c, a, b, 3);
  std::vector<std::vector<ZZ>> va, vb;
  for (int i = 0; i < 3; ++i) {
    va.push_back(F.coeffs(&a[i]));
    vb.push_back(F.coeffs(&b[i]));
  }
  const auto vc = F.coeffs(&c);
  for (int j : F.check_indices()) {
    ZZ s(0);
    for (int i = 0; i < 3; ++i) s += F.negacyclic(va[i], vb[i], j, F.q);
    CHECK(vc[j] == s % F.q, "index " << j);
  }
  // c is also a later operand: the result must be the bytes of cuPoly's
  // poly_mul + poly_mul_add composition, which reads the partial sum
  poly_t x[3], y[3];
  for (int i = 0; i < 3; ++i) {
    poly_copy(F.ctx, &x[i], &a[i]);
    poly_copy(F.ctx, &y[i], &a[i]);
  }
  poly_dot(F.ctx, &x[2], x, b, 3);
  poly_mul(F.ctx, &y[2], &y[0], &b[0]);
  for (int i = 1; i < 3; ++i) poly_mul_add(F.ctx, &y[2], &y[i], &b[i], &y[2]);
  CHECK(F.coeffs(&x[2]) == F.coeffs(&y[2]), "aliased output");
  for (int i = 0; i < 3; ++i) {
    poly_free(F.ctx, &a[i]);
    poly_free(F.ctx, &b[i]);
    poly_free(F.ctx, &x[i]);
    poly_free(F.ctx, &y[i]);
  }
  poly_free(F.ctx, &c);
}

// ---------------------------------------------------------------------------
// TestSampler (support checks as in test_bfv_mode.cu:1405-1487)
// ---------------------------------------------------------------------------
TEST_F(TestSampler, Uniform) {
  poly_t* a = Sampler::sample(F.ctx, UNIFORM);
  for (int i = 0; i < F.nphi; ++i) CHECK(poly_get_coeff(F.ctx, a, i) < F.q, "index " << i);
  CHECK(poly_get_deg(F.ctx, a) > 0, "degree");
  poly_free(F.ctx, a);
  delete a;
}

// cuPoly's BFV UNIFORM (sampler.cu:295-341): one value below 2^32 on every residue.
TEST_F(TestSampler, UniformBelow2To32) {
  poly_t a;
  Sampler::sample(F.ctx, &a, UNIFORM);
  const ZZ lim = ZZ(1) << 32;
  for (int i = 0; i < F.nphi; ++i) CHECK(poly_get_coeff(F.ctx, &a, i) < lim, "index " << i);
  poly_free(F.ctx, &a);
}

// The library's independent form: uniform mod Q, so values far above 2^32 appear.
TEST_F(TestSampler, UniformModQ) {
  poly_t a;
  Sampler::sample(F.ctx, &a, UNIFORM_MOD_Q);
  ZZ mx(0);
  for (int i = 0; i < F.nphi; ++i) {
    const ZZ c = poly_get_coeff(F.ctx, &a, i);
    CHECK(c < F.q, "index " << i);
    if (c > mx) mx = c;
  }
  if (F.nphi >= 128) CHECK(mx > (ZZ(1) << 40), "largest coefficient " << mx);
  poly_free(F.ctx, &a);
}

// cuPoly's ZO (sampler.cu:236-283): exactly nphi/2 coefficients in {-1, +1}.
TEST_F(TestSampler, ZOHalf) {
  poly_t a;
  Sampler::sample(F.ctx, &a, ZO);
  int nz = 0;
  for (int i = 0; i < F.nphi; ++i) {
    const ZZ c = poly_get_coeff(F.ctx, &a, i);
    CHECK(c == ZZ(0) || c == ZZ(1) || c == F.q - 1, "index " << i);
    nz += c != ZZ(0);
  }
  CHECK(nz == F.nphi / 2, "nonzero " << nz);
  poly_free(F.ctx, &a);
}

TEST_F(TestSampler, Narrow) {
  poly_t a;
  Sampler::sample(F.ctx, &a, NARROW);
  int seen[3] = {0, 0, 0};
  for (int i = 0; i < F.nphi; ++i) {
    const ZZ c = poly_get_coeff(F.ctx, &a, i);
    CHECK(c <= ZZ(2), "index " << i << " value " << c);
    seen[to_long(c)]++;
  }
  if (F.nphi >= 128) CHECK(seen[0] && seen[1] && seen[2], "all of {0, 1, 2} drawn");
  poly_free(F.ctx, &a);
}

TEST_F(TestSampler, DiscreteGaussian) {
  poly_t a;
  Sampler::sample(F.ctx, &a, DISCRETE_GAUSSIAN);
  for (int i = 0; i < F.nphi; ++i) CHECK(poly_get_coeff(F.ctx, &a, i) <= ZZ(19), "index " << i);
  poly_free(F.ctx, &a);
}

TEST_F(TestSampler, HammingWeight) {
  poly_t a;
  Sampler::sample(F.ctx, &a, HAMMINGWEIGHT);
  int nz = 0;
  for (int i = 0; i < F.nphi; ++i) {
    const ZZ c = poly_get_coeff(F.ctx, &a, i);
    CHECK(c == ZZ(0) || c == ZZ(1) || c == F.q - 1, "index " << i);
    nz += c != ZZ(0);
  }
  CHECK(nz == std::min(HAMMINGWEIGHT_H, F.nphi), "weight " << nz);
  poly_free(F.ctx, &a);
}

// ---------------------------------------------------------------------------
// CKKS engine (CUDAEngine::init_ckks): xi then rho is the identity; rescale divides
// ---------------------------------------------------------------------------
void ckks_checks() {
  CUDAEngine::init_ckks(3, 4, 4096, 52);
  {
    Context ctx;
    poly_t a, x, r;
    Sampler::sample(&ctx, &a, UNIFORM);
    poly_xi_ckks(&ctx, &x, &a);
    poly_rho_ckks(&ctx, &r, &x);
    for (int j = 0; j < 3; ++j) {
      uint64_t* ra = poly_get_residue(&ctx, NULL, &a, j);
      uint64_t* rr = poly_get_residue(&ctx, NULL, &r, j);
      for (int i = 0; i < 4096; ++i) CHECK(ra[i] == rr[i], "rho(xi(a)) residue " << j << " index " << i);
      free(ra);
      free(rr);
    }
    // rescale at level 2: residues 0, 1 of the result = (x_i - x_2) q_2^-1 mod q_i
    poly_t s;
    poly_copy(&ctx, &s, &a);
    poly_ckks_rescale(&ctx, &s, NULL, 2);
    uint64_t* r2 = poly_get_residue(&ctx, NULL, &a, 2);
    const uint64_t q2 = CUDAEngine::RNSPrimes[2];
    for (int j = 0; j < 2; ++j) {
      const uint64_t qj = CUDAEngine::RNSPrimes[j];
      uint64_t* ra = poly_get_residue(&ctx, NULL, &a, j);
      uint64_t* rs = poly_get_residue(&ctx, NULL, &s, j);
      const ZZ Qj((unsigned long)qj);
      for (int i = 0; i < 4096; ++i) {
        const ZZ d = (ZZ((unsigned long)ra[i]) - ZZ((unsigned long)r2[i])) % Qj;
        CHECK((ZZ((unsigned long)rs[i]) * ZZ((unsigned long)q2)) % Qj == d, "rescale residue " << j << " index " << i);
      }
      free(ra);
      free(rs);
    }
    free(r2);
    for (poly_t* p : {&a, &x, &r, &s}) poly_free(&ctx, p);
  }
  CUDAEngine::destroy();
}

}  // namespace

int main(int argc, char** argv) {
  bool quick = false;
  std::string filter;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--quick")
      quick = true;
    else
      filter = a;
  }
  std::vector<Params> grid = {{30, 32},    {120, 32},   {130, 32},   {340, 32},   {30, 128},
                              {120, 128},  {120, 256},  {30, 2048},  {120, 2048}, {340, 2048},
                              {170, 4096}, {170, 8192}, {250, 8192}, {340, 8192}};
  if (quick) grid = {{120, 32}, {340, 128}, {170, 4096}};
  int passed = 0, failed = 0;
  for (const auto& p : grid) {
    for (auto& [name, fn] : registry()) {
      const std::string full = name + "/" + std::to_string(p.nphi) + "_q" + std::to_string(p.logq2);
      if (!filter.empty() && full.find(filter) == std::string::npos) continue;
      try {
        Fixture f(p);
        fn(f);
        ++passed;
      } catch (const Failure& e) {
        ++failed;
        std::printf("[  FAILED  ] %s: %s\n", full.c_str(), e.msg.c_str());
      } catch (const std::exception& e) {
        ++failed;
        std::printf("[  FAILED  ] %s: exception: %s\n", full.c_str(), e.what());
      }
    }
  }
  if (filter.empty() || std::string("CKKS").find(filter) != std::string::npos) {
    try {
      ckks_checks();
      ++passed;
    } catch (const Failure& e) {
      ++failed;
      std::printf("[  FAILED  ] CKKS: %s\n", e.msg.c_str());
    } catch (const std::exception& e) {
      ++failed;
      std::printf("[  FAILED  ] CKKS: exception: %s\n", e.what());
    }
  }
  std::printf("[==========] %d passed, %d failed\n", passed, failed);
  return failed == 0 ? 0 : 1;
}
