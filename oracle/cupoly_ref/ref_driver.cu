// TEST INFRASTRUCTURE, not product code.
//
// Runs cuPoly's own library (pdroalves/cupoly 0.3.5, compiled unmodified from
// its sources by oracle/cupoly_ref/Makefile into oracle/_ref/) on seeded
// inputs and writes its outputs, so that the oracle and the CUDA path can be
// compared with the reference's bytes.  Every call goes through cuPoly's
// public API: CUDAEngine::init, Context, poly_t, poly_mul, poly_dr2,
// poly_basis_extension_Q_to_B, poly_complex_scaling_tDivQ,
// poly_simple_scaling_tDivQ, poly_xi_bfv, poly_rho_bfv, DGTEngine::execute_dgt
// (include/cuPoly/arithmetic/polynomial.h, include/cuPoly/cuda/dgt.h).
//
//   cupoly_ref_driver OP[,OP...] k kl nphi t IN OUT
//
// With several OPs (one engine initialisation for all of them), OP reads
// IN.<OP> and writes OUT.<OP>.
// IN and OUT are raw little-endian uint64 arrays.  A polynomial is given as
// coefficient-domain residue rows [nres][nphi]; the driver folds them into
// cuPoly's GaussianInteger layout (element j = (a_j, a_{j+N}),
// src/arithmetic/polynomial.cu:206-217), copies them into the poly's device
// buffer and applies cuPoly's forward DGT, which is what poly_copy_to_device
// does after its host CRT (polynomial.cu:105-138).  Outputs are read back the
// way poly_copy_to_host does, through cuPoly's inverse DGT of a copy
// (polynomial.cu:140-188), as coefficient-domain rows.
//
// OPs:
//   tables  IN unused.  OUT: Q primes, B primes, Barrett MU of Q u B, and the
//           BFV HPS constants of cudaengine.cu:1337-1510 read back from
//           constant memory (omega_int, omega_frac lo/hi, lambda,
//           tomega_int, tomega_frac lo/hi).
//   dgt     IN: one poly over Q u B.  OUT: its DGT-domain bytes
//           ([k+kl][N][2]) and then the inverse transform of those bytes.
//   mul     IN: a, b over Q.  OUT: poly_mul(a, b).
//   ext     IN: a over Q.  OUT: poly_basis_extension_Q_to_B(a) over B.
//   cscale  IN: a over Q, a over B.  OUT: poly_complex_scaling_tDivQ over Q.
//   sscale  IN: a over Q.  OUT: poly_simple_scaling_tDivQ: nphi values mod t.
//   bfvmul  IN: a0, a1, b0, b1 over Q.  OUT: c0, c1, c2 over Q: the four
//           extensions Q -> B, poly_dr2 over Q and over B, and one complex
//           scaling per output.
//   bfvtrace  IN as bfvmul.  OUT: the chain stage by stage: the four B
//           extensions, the tensor over Q (3 polys) and over B (3 polys), the
//           scaled B words of c0 (ctx->d_coefs_B) and c0.
//   xirho   IN: a over Q.  OUT: poly_xi_bfv(a) (k polys over Q), then
//           poly_rho_bfv(a) (k polys over Q).
//   time    IN unused; t the iteration count is argv[5] as for the others.
//           OUT (text): milliseconds per call of the polymul (two forward
//           DGTs, poly_mul, one inverse DGT) and of the bfvmul chain above,
//           each timed with CUDA events on the Context's stream.
#include <cuPoly/arithmetic/context.h>
#include <cuPoly/arithmetic/polynomial.h>
#include <cuPoly/cuda/cudaengine.h>
#include <cuPoly/cuda/dgt.h>
#include <cuPoly/settings.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

// cuPoly's constant-memory HPS tables (src/cuda/cudaengine.cu:72-80) and the
// host copy of its Barrett constants (src/cuda/dgt.cu:32).
extern __constant__ uint64_t d_RNSomega_int[MAX_COPRIMES_IN_A_BASE * MAX_COPRIMES_IN_A_BASE];
extern __constant__ uint128_t d_RNSomega_frac[MAX_COPRIMES_IN_A_BASE * MAX_COPRIMES_IN_A_BASE];
extern __constant__ uint64_t d_RNSlambda[MAX_COPRIMES_IN_A_BASE];
extern __constant__ uint64_t d_RNStomega_int[MAX_COPRIMES_IN_A_BASE * MAX_COPRIMES_IN_A_BASE];
extern __constant__ uint128_t d_RNStomega_frac[MAX_COPRIMES_IN_A_BASE * MAX_COPRIMES_IN_A_BASE];
extern uint64_t h_BARRETT_MU[MAX_COPRIMES];

namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "cupoly_ref_driver: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(3);
  }
}

std::vector<uint64_t> read_u64(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    std::fprintf(stderr, "cupoly_ref_driver: cannot read %s\n", path.c_str());
    std::exit(2);
  }
  const std::streamsize n = f.tellg();
  f.seekg(0);
  std::vector<uint64_t> v((size_t)n / 8);
  f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(v.size() * 8));
  return v;
}

void write_u64(const std::string& path, const std::vector<uint64_t>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * 8));
}

int nphi_of() { return 2 * CUDAEngine::N; }

// Every copy goes on the Context's stream and is waited for.  cuPoly builds with
// --default-stream per-thread, so a plain cudaMemcpy runs on the per-thread stream,
// which does not order with the Context's stream: a pageable host-to-device copy may
// still be in flight when the next kernel on the Context's stream reads its target,
// and a device-to-device copy returns before it has run.
void copy(Context* ctx, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, const char* what) {
  check(cudaStreamSynchronize(ctx->get_stream()), what);
  check(cudaMemcpyAsync(dst, src, bytes, kind, ctx->get_stream()), what);
  check(cudaStreamSynchronize(ctx->get_stream()), what);
}

// Rows [nres][nphi] at `rows` -> poly p over `base`, in cuPoly's DGT domain.
void upload(Context* ctx, poly_t* p, int base, const uint64_t* rows) {
  poly_init(ctx, p, base);
  const int N = CUDAEngine::N, nres = CUDAEngine::get_n_residues(base), nphi = nphi_of();
  std::vector<GaussianInteger> h((size_t)nres * N);
  for (int r = 0; r < nres; ++r)
    for (int j = 0; j < N; ++j) {
      h[(size_t)r * N + j].re = rows[(size_t)r * nphi + j];
      h[(size_t)r * N + j].imag = rows[(size_t)r * nphi + j + N];
    }
  copy(ctx, p->d_coefs, h.data(), h.size() * sizeof(GaussianInteger), cudaMemcpyHostToDevice, "upload");
  DGTEngine::execute_dgt(p->d_coefs, base, FORWARD, ctx);
  check(cudaStreamSynchronize(ctx->get_stream()), "forward DGT");
  p->status = RNSSTATE;
  p->base = base;
}

// Coefficient-domain rows of p (DGT domain on the device; p is not changed).
void download(Context* ctx, poly_t* p, std::vector<uint64_t>& out) {
  const int base = p->base;
  const int N = CUDAEngine::N, nres = CUDAEngine::get_n_residues(base), nphi = nphi_of();
  const size_t bytes = (size_t)nres * N * sizeof(GaussianInteger);
  GaussianInteger* tmp = nullptr;
  check(cudaMalloc((void**)&tmp, bytes), "cudaMalloc");
  copy(ctx, tmp, p->d_coefs, bytes, cudaMemcpyDeviceToDevice, "copy");
  DGTEngine::execute_dgt(tmp, base, INVERSE, ctx);
  check(cudaStreamSynchronize(ctx->get_stream()), "inverse DGT");
  std::vector<GaussianInteger> h((size_t)nres * N);
  copy(ctx, h.data(), tmp, bytes, cudaMemcpyDeviceToHost, "download");
  check(cudaFree(tmp), "cudaFree");
  const size_t o = out.size();
  out.resize(o + (size_t)nres * nphi);
  for (int r = 0; r < nres; ++r)
    for (int j = 0; j < N; ++j) {
      out[o + (size_t)r * nphi + j] = h[(size_t)r * N + j].re;
      out[o + (size_t)r * nphi + j + N] = h[(size_t)r * N + j].imag;
    }
}

void raw_download(Context* ctx, poly_t* p, std::vector<uint64_t>& out) {
  const int nres = CUDAEngine::get_n_residues(p->base);
  const size_t words = (size_t)nres * CUDAEngine::N * 2;
  const size_t o = out.size();
  out.resize(o + words);
  copy(ctx, out.data() + o, p->d_coefs, words * 8, cudaMemcpyDeviceToHost, "raw download");
}

void need(const std::vector<uint64_t>& in, size_t words, const char* op) {
  if (in.size() != words) {
    std::fprintf(stderr, "cupoly_ref_driver %s: expected %zu input words, got %zu\n", op, words, in.size());
    std::exit(2);
  }
}

// cuPoly's BFV multiplication chain from DGT-domain Q inputs to DGT-domain Q
// outputs, through its public calls only.
void bfv_chain(Context* ctx, poly_t* c, poly_t* a, poly_t* aB, poly_t* tq, poly_t* tb) {
  for (int v = 0; v < 4; ++v) {
    poly_init(ctx, &aB[v], BBase);
    poly_basis_extension_Q_to_B(ctx, &aB[v], &a[v]);
  }
  for (int o = 0; o < 3; ++o) {
    poly_init(ctx, &tq[o], QBase);
    poly_init(ctx, &tb[o], BBase);
  }
  poly_dr2(ctx, &tq[0], &tq[1], &tq[2], &a[0], &a[1], &a[2], &a[3]);
  poly_dr2(ctx, &tb[0], &tb[1], &tb[2], &aB[0], &aB[1], &aB[2], &aB[3]);
  for (int o = 0; o < 3; ++o) {
    poly_init(ctx, &c[o], QBase);
    poly_complex_scaling_tDivQ(ctx, &c[o], &tq[o], &tb[o]);
  }
}

// One OP on the initialised engine; 0 on success.
int run_op(const std::string& op, int k, int kl, int nphi, uint64_t t, Context* ctx, const std::string& in_path,
           const std::string& out_path) {
  const size_t qw = (size_t)k * nphi, bw = (size_t)kl * nphi;
  std::vector<uint64_t> out;

  if (op == "tables") {
    for (uint64_t p : CUDAEngine::RNSPrimes) out.push_back(p);
    for (uint64_t p : CUDAEngine::RNSBPrimes) out.push_back(p);
    for (int i = 0; i < k + kl; ++i) out.push_back(h_BARRETT_MU[i]);
    const size_t kk = (size_t)k * kl;
    std::vector<uint64_t> oi(kk), l(kl), ti(k);
    std::vector<uint128_t> of(kk), tf(k);
    check(cudaMemcpyFromSymbol(oi.data(), d_RNSomega_int, kk * 8), "omega_int");
    check(cudaMemcpyFromSymbol(of.data(), d_RNSomega_frac, kk * sizeof(uint128_t)), "omega_frac");
    check(cudaMemcpyFromSymbol(l.data(), d_RNSlambda, (size_t)kl * 8), "lambda");
    check(cudaMemcpyFromSymbol(ti.data(), d_RNStomega_int, (size_t)k * 8), "tomega_int");
    check(cudaMemcpyFromSymbol(tf.data(), d_RNStomega_frac, (size_t)k * sizeof(uint128_t)), "tomega_frac");
    out.insert(out.end(), oi.begin(), oi.end());
    for (const uint128_t& v : of) {
      out.push_back(v.lo);
      out.push_back(v.hi);
    }
    out.insert(out.end(), l.begin(), l.end());
    out.insert(out.end(), ti.begin(), ti.end());
    for (const uint128_t& v : tf) {
      out.push_back(v.lo);
      out.push_back(v.hi);
    }
  } else if (op == "dgt") {
    const std::vector<uint64_t> in = read_u64(in_path);
    need(in, qw + bw, "dgt");
    poly_t a;
    upload(ctx, &a, QBBase, in.data());
    raw_download(ctx, &a, out);
    DGTEngine::execute_dgt(a.d_coefs, QBBase, INVERSE, ctx);
    raw_download(ctx, &a, out);
    poly_free(ctx, &a);
  } else if (op == "mul") {
    const std::vector<uint64_t> in = read_u64(in_path);
    need(in, 2 * qw, "mul");
    poly_t a, b, c;
    upload(ctx, &a, QBase, in.data());
    upload(ctx, &b, QBase, in.data() + qw);
    poly_mul(ctx, &c, &a, &b);
    download(ctx, &c, out);
    poly_free(ctx, &a);
    poly_free(ctx, &b);
    poly_free(ctx, &c);
  } else if (op == "ext") {
    const std::vector<uint64_t> in = read_u64(in_path);
    need(in, qw, "ext");
    poly_t a, b;
    upload(ctx, &a, QBase, in.data());
    poly_init(ctx, &b, BBase);
    poly_basis_extension_Q_to_B(ctx, &b, &a);
    download(ctx, &b, out);
    poly_free(ctx, &a);
    poly_free(ctx, &b);
  } else if (op == "cscale") {
    const std::vector<uint64_t> in = read_u64(in_path);
    need(in, qw + bw, "cscale");
    poly_t aq, ab, c;
    upload(ctx, &aq, QBase, in.data());
    upload(ctx, &ab, BBase, in.data() + qw);
    poly_init(ctx, &c, QBase);
    poly_complex_scaling_tDivQ(ctx, &c, &aq, &ab);
    download(ctx, &c, out);
    poly_free(ctx, &aq);
    poly_free(ctx, &ab);
    poly_free(ctx, &c);
  } else if (op == "sscale") {
    const std::vector<uint64_t> in = read_u64(in_path);
    need(in, qw, "sscale");
    poly_t a, b;
    upload(ctx, &a, QBase, in.data());
    poly_init(ctx, &b, QBase);
    poly_simple_scaling_tDivQ(ctx, &b, &a);
    // The result is residue 0 of b's buffer in the coefficient domain
    // (cudaengine.cu:323-362 writes a[cid] for every Gaussian element).
    std::vector<GaussianInteger> h(CUDAEngine::N);
    copy(ctx, h.data(), b.d_coefs, h.size() * sizeof(GaussianInteger), cudaMemcpyDeviceToHost, "download");
    out.resize((size_t)nphi);
    for (int j = 0; j < CUDAEngine::N; ++j) {
      out[j] = h[j].re;
      out[j + CUDAEngine::N] = h[j].imag;
    }
    poly_free(ctx, &a);
    poly_free(ctx, &b);
  } else if (op == "bfvmul") {
    const std::vector<uint64_t> in = read_u64(in_path);
    need(in, 4 * qw, "bfvmul");
    poly_t a[4], aB[4], tq[3], tb[3], c[3];
    for (int v = 0; v < 4; ++v) upload(ctx, &a[v], QBase, in.data() + v * qw);
    bfv_chain(ctx, c, a, aB, tq, tb);
    for (int o = 0; o < 3; ++o) download(ctx, &c[o], out);
    for (poly_t* p : {&a[0], &a[1], &a[2], &a[3], &aB[0], &aB[1], &aB[2], &aB[3], &tq[0], &tq[1], &tq[2], &tb[0],
                      &tb[1], &tb[2], &c[0], &c[1], &c[2]})
      poly_free(ctx, p);
  } else if (op == "bfvtrace") {
    // The chain of bfvmul stage by stage (coefficient domain): the four extensions
    // Q -> B, the tensor over Q and over B, then for c0 the scaled B residues cuPoly
    // leaves in ctx->d_coefs_B ([kl][2N] words) and c0 itself.
    const std::vector<uint64_t> in = read_u64(in_path);
    need(in, 4 * qw, "bfvtrace");
    poly_t a[4], aB[4], tq[3], tb[3], c0;
    for (int v = 0; v < 4; ++v) upload(ctx, &a[v], QBase, in.data() + v * qw);
    for (int v = 0; v < 4; ++v) {
      poly_init(ctx, &aB[v], BBase);
      poly_basis_extension_Q_to_B(ctx, &aB[v], &a[v]);
      download(ctx, &aB[v], out);
    }
    for (int o = 0; o < 3; ++o) {
      poly_init(ctx, &tq[o], QBase);
      poly_init(ctx, &tb[o], BBase);
    }
    poly_dr2(ctx, &tq[0], &tq[1], &tq[2], &a[0], &a[1], &a[2], &a[3]);
    poly_dr2(ctx, &tb[0], &tb[1], &tb[2], &aB[0], &aB[1], &aB[2], &aB[3]);
    for (int o = 0; o < 3; ++o) download(ctx, &tq[o], out);
    for (int o = 0; o < 3; ++o) download(ctx, &tb[o], out);
    poly_init(ctx, &c0, QBase);
    poly_complex_scaling_tDivQ(ctx, &c0, &tq[0], &tb[0]);
    const size_t o0 = out.size();
    out.resize(o0 + bw);
    copy(ctx, out.data() + o0, ctx->d_coefs_B, bw * 8, cudaMemcpyDeviceToHost, "d_coefs_B");
    download(ctx, &c0, out);
    for (poly_t* p : {&a[0], &a[1], &a[2], &a[3], &aB[0], &aB[1], &aB[2], &aB[3], &tq[0], &tq[1], &tq[2], &tb[0],
                      &tb[1], &tb[2], &c0})
      poly_free(ctx, p);
  } else if (op == "xirho") {
    const std::vector<uint64_t> in = read_u64(in_path);
    need(in, qw, "xirho");
    poly_t a;
    upload(ctx, &a, QBase, in.data());
    std::vector<poly_t> xi(k), rho(k);
    for (int i = 0; i < k; ++i) poly_init(ctx, &xi[i], QBase);
    poly_xi_bfv(ctx, xi.data(), &a);
    for (int i = 0; i < k; ++i) download(ctx, &xi[i], out);
    poly_rho_bfv(ctx, rho.data(), &a);
    for (int i = 0; i < k; ++i) download(ctx, &rho[i], out);
    for (int i = 0; i < k; ++i) {
      poly_free(ctx, &xi[i]);
      poly_free(ctx, &rho[i]);
    }
    poly_free(ctx, &a);
  } else if (op == "time") {
    const int iters = (int)t;
    // Operands: zero polynomials are as costly as any other for these kernels.
    std::vector<uint64_t> zeros(4 * qw, 0);
    poly_t a[4], aB[4], tq[3], tb[3], c[3], m;
    for (int v = 0; v < 4; ++v) upload(ctx, &a[v], QBase, zeros.data() + v * qw);
    poly_init(ctx, &m, QBase);
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    cudaStream_t s = ctx->get_stream();
    auto polymul = [&]() {
      DGTEngine::execute_dgt(a[0].d_coefs, QBase, FORWARD, ctx);
      DGTEngine::execute_dgt(a[1].d_coefs, QBase, FORWARD, ctx);
      poly_mul(ctx, &m, &a[0], &a[1]);
      DGTEngine::execute_dgt(m.d_coefs, QBase, INVERSE, ctx);
    };
    for (int i = 0; i < 5; ++i) polymul();
    check(cudaStreamSynchronize(s), "warm-up");
    check(cudaEventRecord(e0, s), "record");
    for (int i = 0; i < iters; ++i) polymul();
    check(cudaEventRecord(e1, s), "record");
    check(cudaEventSynchronize(e1), "sync");
    float ms_mul = 0;
    check(cudaEventElapsedTime(&ms_mul, e0, e1), "elapsed");
    for (int i = 0; i < 3; ++i) bfv_chain(ctx, c, a, aB, tq, tb);
    check(cudaDeviceSynchronize(), "warm-up");
    check(cudaEventRecord(e0, s), "record");
    for (int i = 0; i < iters; ++i) bfv_chain(ctx, c, a, aB, tq, tb);
    check(cudaEventRecord(e1, s), "record");
    check(cudaEventSynchronize(e1), "sync");
    float ms_chain = 0;
    check(cudaEventElapsedTime(&ms_chain, e0, e1), "elapsed");
    check(cudaDeviceSynchronize(), "sync");
    std::ofstream f(out_path);
    f << "{\"polymul_ms\": " << ms_mul / iters << ", \"bfv_mul_ms\": " << ms_chain / iters << ", \"iters\": " << iters
      << "}\n";
    for (poly_t* p : {&a[0], &a[1], &a[2], &a[3], &aB[0], &aB[1], &aB[2], &aB[3], &tq[0], &tq[1], &tq[2], &tb[0],
                      &tb[1], &tb[2], &c[0], &c[1], &c[2], &m})
      poly_free(ctx, p);
    return 0;
  } else {
    std::fprintf(stderr, "cupoly_ref_driver: unknown op %s\n", op.c_str());
    return 2;
  }
  check(cudaDeviceSynchronize(), "final sync");
  write_u64(out_path, out);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 8) {
    std::fprintf(stderr, "usage: %s OP[,OP...] k kl nphi t IN OUT\n", argv[0]);
    return 2;
  }
  std::vector<std::string> ops;
  {
    std::string cur;
    for (const char* c = argv[1];; ++c) {
      if (*c == ',' || *c == 0) {
        if (!cur.empty()) ops.push_back(cur);
        cur.clear();
        if (*c == 0) break;
      } else {
        cur += *c;
      }
    }
  }
  const int k = std::atoi(argv[2]), kl = std::atoi(argv[3]), nphi = std::atoi(argv[4]);
  const uint64_t t = std::strtoull(argv[5], nullptr, 10);
  const std::string in_path = argv[6], out_path = argv[7];
  const bool timing = ops.size() == 1 && ops[0] == "time";
  for (const std::string& op : ops)
    if (op == "time" && !timing) {
      std::fprintf(stderr, "cupoly_ref_driver: time runs alone\n");
      return 2;
    }
  CUDAEngine::init(k, kl, nphi, timing ? 256 : t);
  Context* ctx = new Context();
  int rc = 0;
  for (const std::string& op : ops) {
    // several OPs: IN.<op> and OUT.<op>
    const std::string ip = ops.size() > 1 ? in_path + "." + op : in_path;
    const std::string outp = ops.size() > 1 ? out_path + "." + op : out_path;
    rc = run_op(op, k, kl, nphi, t, ctx, ip, outp);
    if (rc) break;
  }
  delete ctx;
  CUDAEngine::destroy();
  return rc;
}
