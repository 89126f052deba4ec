// DGT-domain bytes through the C++ host layer, as a cuPoly program would take
// them: CUDAEngine::init(k, kl, nphi, t), coefficient-domain residues copied
// into a poly_t's device buffer (folded GaussianInteger layout), then
// DGTEngine::execute_dgt(..., QBBase, FORWARD, ctx) and the raw d_coefs bytes
// written out.  With CUPOLY_COPRIMES_DIR naming cuPoly's coprimes directory at
// init, the bytes are cuPoly's own.
//
//   dgt_bytes k kl nphi IN OUT    (IN: uint64 rows [k + kl][nphi]; OUT: [k + kl][N][2])
#include <cuPoly/arithmetic/context.h>
#include <cuPoly/arithmetic/polynomial.h>
#include <cuPoly/cuda/dgt.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s k kl nphi IN OUT\n", argv[0]);
    return 2;
  }
  const int k = std::atoi(argv[1]), kl = std::atoi(argv[2]), nphi = std::atoi(argv[3]);
  const int nres = k + kl, N = nphi / 2;
  std::vector<uint64_t> rows((size_t)nres * nphi);
  {
    std::ifstream f(argv[4], std::ios::binary);
    f.read(reinterpret_cast<char*>(rows.data()), (std::streamsize)(rows.size() * 8));
    if (!f) {
      std::fprintf(stderr, "short input\n");
      return 2;
    }
  }
  CUDAEngine::init(k, kl, nphi, 256);
  {
    Context ctx;
    poly_t a;
    poly_init(&ctx, &a, QBBase);
    std::vector<GaussianInteger> h((size_t)nres * N);
    for (int r = 0; r < nres; ++r)
      for (int j = 0; j < N; ++j) {
        h[(size_t)r * N + j].re = rows[(size_t)r * nphi + j];
        h[(size_t)r * N + j].imag = rows[(size_t)r * nphi + j + N];
      }
    cudaMemcpy(a.d_coefs, h.data(), h.size() * sizeof(GaussianInteger), cudaMemcpyHostToDevice);
    DGTEngine::execute_dgt(a.d_coefs, QBBase, FORWARD, &ctx);
    cudaStreamSynchronize(ctx.get_stream());
    cudaMemcpy(h.data(), a.d_coefs, h.size() * sizeof(GaussianInteger), cudaMemcpyDeviceToHost);
    std::ofstream o(argv[5], std::ios::binary);
    o.write(reinterpret_cast<const char*>(h.data()), (std::streamsize)(h.size() * sizeof(GaussianInteger)));
    poly_free(&ctx, &a);
  }
  CUDAEngine::destroy();
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}
