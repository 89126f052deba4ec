// Per-call timing of the C++ drop-in layer (libcupoly.so) in the form a cuPoly
// program uses it, one call sequence at a time on the Context's stream:
//  * one polynomial product: two forward DGTs, poly_mul, one inverse DGT
//    (DGTEngine::execute_dgt, cuPoly src/cuda/dgt.cu:107-205; poly_mul,
//    src/arithmetic/polynomial.cu:892-914);
//  * one BFV multiplication: four poly_basis_extension_Q_to_B, poly_dr2 over Q
//    and over B, three poly_complex_scaling_tDivQ (polynomial.cu:350-470,
//    951-1000).
// Each is timed with CUDA events over ITERS calls after five warm-up calls.
// Operands are zero polynomials: the kernels' cost does not depend on the values.
//
//   cupoly_percall k kl nphi iters      -> one JSON line on stdout
#include <cuPoly/arithmetic/context.h>
#include <cuPoly/arithmetic/polynomial.h>
#include <cuPoly/cuda/cudaengine.h>
#include <cuPoly/cuda/dgt.h>

#include <cstdio>
#include <cstdlib>

namespace {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "cupoly_percall: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(3);
  }
}

template <class F>
float time_ms(Context* ctx, int iters, F&& f) {
  for (int i = 0; i < 5; ++i) f();
  check(cudaStreamSynchronize(ctx->get_stream()), "warm-up");
  cudaEvent_t e0, e1;
  check(cudaEventCreate(&e0), "event");
  check(cudaEventCreate(&e1), "event");
  check(cudaEventRecord(e0, ctx->get_stream()), "record");
  for (int i = 0; i < iters; ++i) f();
  check(cudaEventRecord(e1, ctx->get_stream()), "record");
  check(cudaEventSynchronize(e1), "sync");
  float ms = 0.f;
  check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / iters;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s k kl nphi iters\n", argv[0]);
    return 2;
  }
  const int k = std::atoi(argv[1]), kl = std::atoi(argv[2]), nphi = std::atoi(argv[3]), iters = std::atoi(argv[4]);
  if (k < 1 || kl < 1 || nphi < 4 || iters < 1) {
    std::fprintf(stderr, "cupoly_percall: bad arguments\n");
    return 2;
  }
  CUDAEngine::init(k, kl, nphi, 256);
  float ms_mul = 0.f, ms_chain = 0.f;
  {
    Context ctx;
    poly_t a[4], aB[4], tq[3], tb[3], c[3], m;
    for (poly_t& p : a) poly_init(&ctx, &p, QBase);
    for (poly_t& p : aB) poly_init(&ctx, &p, BBase);
    for (int o = 0; o < 3; ++o) {
      poly_init(&ctx, &tq[o], QBase);
      poly_init(&ctx, &tb[o], BBase);
      poly_init(&ctx, &c[o], QBase);
    }
    poly_init(&ctx, &m, QBase);
    ms_mul = time_ms(&ctx, iters, [&]() {
      DGTEngine::execute_dgt(a[0].d_coefs, QBase, FORWARD, &ctx);
      DGTEngine::execute_dgt(a[1].d_coefs, QBase, FORWARD, &ctx);
      poly_mul(&ctx, &m, &a[0], &a[1]);
      DGTEngine::execute_dgt(m.d_coefs, QBase, INVERSE, &ctx);
    });
    ms_chain = time_ms(&ctx, iters, [&]() {
      for (int v = 0; v < 4; ++v) poly_basis_extension_Q_to_B(&ctx, &aB[v], &a[v]);
      poly_dr2(&ctx, &tq[0], &tq[1], &tq[2], &a[0], &a[1], &a[2], &a[3]);
      poly_dr2(&ctx, &tb[0], &tb[1], &tb[2], &aB[0], &aB[1], &aB[2], &aB[3]);
      for (int o = 0; o < 3; ++o) poly_complex_scaling_tDivQ(&ctx, &c[o], &tq[o], &tb[o]);
    });
    check(cudaDeviceSynchronize(), "final sync");
    for (poly_t* p : {&a[0], &a[1], &a[2], &a[3], &aB[0], &aB[1], &aB[2], &aB[3], &tq[0], &tq[1], &tq[2], &tb[0],
                      &tb[1], &tb[2], &c[0], &c[1], &c[2], &m})
      poly_free(&ctx, p);
  }
  std::printf("{\"polymul_ms\": %.6f, \"bfv_mul_ms\": %.6f, \"iters\": %d}\n", ms_mul, ms_chain, iters);
  CUDAEngine::destroy();
  return 0;
}
