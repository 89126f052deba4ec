// On-device sampler (replaces cuPoly's Sampler: cuRAND XORWOW kernels and the
// host-side ZO / Hamming-weight samplers, src/cuda/sampler.cu:30-645).
//
// Counter-based: every random word comes from Philox4x32-10 (Salmon et al.,
// SC'11) keyed by the 64-bit seed, with counter (coefficient, draw, stream id,
// kind).  There is no generator state in memory, so a polynomial is a pure
// function of (seed, stream id, kind, parameters) and batches of
// polynomials sample in parallel with no setup kernel.
//
// Coefficient c of a polynomial (0 <= c < nphi) is written folded:
// Gaussian element c mod N, real part if c < N, imaginary part otherwise.
// Negative values are stored as p - |v|.
#include "cdt_table.h"
#include "launch.cuh"
#include "pointwise.cuh"

namespace cpoly {

__constant__ uint64_t c_cdt_signed[kCdtLen];
__constant__ uint64_t c_cdt_folded[kCdtLen];

namespace {

struct Philox {
  uint32_t v[4];
};

__device__ __forceinline__ Philox philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  Philox o;
  o.v[0] = c0;
  o.v[1] = c1;
  o.v[2] = c2;
  o.v[3] = c3;
  return o;
}

enum Kind : int {
  DISCRETE_GAUSSIAN = 0,  // cuPoly BFV: |nearbyint(3.2 Z)|, truncated at 6 sigma
  HAMMINGWEIGHT = 1,      // exactly min(64, nphi) coefficients in {-1, +1}
  NARROW = 2,             // uniform {0, 1, 2}
  ZO = 3,                 // i.i.d. {-1: 1/4, 0: 1/2, +1: 1/4}
  BINARY = 4,             // uniform {0, 1}
  UNIFORM = 5,            // uniform mod q_i, independently per residue
  TERNARY = 6,            // uniform {-1, 0, +1}
  GAUSSIAN = 7,           // discrete Gaussian sigma = 3.19, |x| <= 19, signed
  SIGNED_DG = 8,          // CKKS engines' DISCRETE_GAUSSIAN: nearbyint(3.2 Z), signed (internal)
  UNIFORM_U32 = 9,        // cuPoly BFV UNIFORM: one value uniform in [0, 2^32), the same on every residue
  ZO_HALF = 10,           // cuPoly BFV ZO: exactly nphi/2 coefficients nonzero, each +-1 with probability 1/2
};

// A keyed bijection of [0, 2^b) (b = log2 nphi): a 4-round Feistel network whose
// round function is Philox4x32-10 (Luby-Rackoff: a pseudo-random permutation).
// For odd b it runs on b + 1 bits and walks the cycle until the value is back in
// range (at most 64 steps; the chance of more is below 2^-64).  Counter words
// (half, 0x5A000000 + round, stream id, kind) never meet the sign draw's (c, 1, ...).
__device__ __forceinline__ bool zo_half_position(uint32_t c, int b, uint32_t sid, uint32_t k0, uint32_t k1,
                                                 uint32_t& out) {
  const int hb = (b + 1) >> 1;  // half width of the even-width network
  const uint32_t m = (1u << hb) - 1, lim = 1u << b;
  uint32_t x = c;
  for (int walk = 0; walk < 64; ++walk) {
    uint32_t L = x >> hb, R = x & m;
#pragma unroll
    for (uint32_t r = 0; r < 4; ++r) {
      const uint32_t f = philox4x32_10(R, 0x5A000000u + r, sid, (uint32_t)ZO_HALF, k0, k1).v[0] & m;
      const uint32_t nl = R;
      R = L ^ f;
      L = nl;
    }
    x = (L << hb) | R;
    if (x < lim) {
      out = x;
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ uint64_t cdt_lookup(uint64_t u63, const uint64_t* cdt) {
  uint64_t m = 0;
#pragma unroll
  for (int i = 0; i < kCdtLen; ++i) m += (u63 >= cdt[i]) ? 1 : 0;
  return m;
}

// Small signed value of coefficient c for the residue-independent kinds.
// Returns false if all draws were rejected (probability < 2^-250).
__device__ __forceinline__ bool small_value(int kind, uint32_t c, uint32_t sid, uint32_t k0, uint32_t k1,
                                            int nphi_log, int64_t& v) {
  if (kind == NARROW || kind == TERNARY) {
    for (uint32_t d = 0; d < 8; ++d) {
      const Philox r = philox4x32_10(c, d, sid, (uint32_t)kind, k0, k1);
#pragma unroll
      for (int w = 0; w < 4; ++w)
        if (r.v[w] != 0xFFFFFFFFu) {
          const int64_t x = r.v[w] % 3u;
          v = (kind == TERNARY && x == 2) ? -1 : x;
          return true;
        }
    }
    return false;
  }
  if (kind == ZO_HALF) {  // nonzero iff the coefficient's image lies in the first half
    uint32_t pos;
    if (!zo_half_position(c, nphi_log, sid, k0, k1, pos)) return false;
    const Philox sg = philox4x32_10(c, 1, sid, (uint32_t)kind, k0, k1);
    v = (pos >> (nphi_log - 1)) ? 0 : ((sg.v[0] & 1u) ? -1 : 1);
    return true;
  }
  const Philox r = philox4x32_10(c, 0, sid, (uint32_t)kind, k0, k1);
  const uint64_t u63 = ((uint64_t)(r.v[1] & 0x7FFFFFFFu) << 32) | r.v[0];
  switch (kind) {
    case BINARY: v = r.v[0] & 1u; return true;
    case ZO: {
      const uint32_t b = r.v[0] & 3u;
      v = b < 2 ? 0 : (b == 2 ? 1 : -1);
      return true;
    }
    case DISCRETE_GAUSSIAN: v = (int64_t)cdt_lookup(u63, c_cdt_folded); return true;
    case SIGNED_DG: {  // |nearbyint(3.2 Z)| with a symmetric sign is nearbyint(3.2 Z)
      const int64_t m = (int64_t)cdt_lookup(u63, c_cdt_folded);
      v = (r.v[2] & 1u) ? -m : m;
      return true;
    }
    case GAUSSIAN: {
      const int64_t m = (int64_t)cdt_lookup(u63, c_cdt_signed);
      v = (r.v[2] & 1u) ? -m : m;
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ uint64_t lift(int64_t v, uint64_t p) { return v >= 0 ? (uint64_t)v : p - (uint64_t)(-v); }

// One thread per Gaussian element j (coefficients j and j + N) of one polynomial.
__global__ void __launch_bounds__(256) k_sample(ulonglong2* __restrict__ out, const ModConst* __restrict__ mc, int N,
                                                int nres, int rid_off, int kind, uint32_t k0, uint32_t k1,
                                                uint32_t sid0, long long poly_stride, int* __restrict__ err,
                                                const uint32_t* __restrict__ ids) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const uint32_t sid = ids ? ids[blockIdx.y] : sid0 + blockIdx.y;
  out += blockIdx.y * poly_stride;
  if (kind == UNIFORM) {
    // one Philox block per draw serves both coefficients of element j: words 0-1 are
    // the candidate for coefficient j, words 2-3 for j + N; each keeps its first
    // candidate below p (candidates of bitlen(p) bits: every prime of the tables lies
    // within 0.01 % below its power of two, so a draw is accepted with p > 0.9999)
    for (int r = 0; r < nres; ++r) {
      const uint64_t p = mc[rid_off + r].p;
      const uint64_t mask = ~0ull >> __clzll((long long)p);
      uint64_t val[2] = {0, 0};
      bool ok0 = false, ok1 = false;
      for (uint32_t d = 0; d < 16 && !(ok0 && ok1); ++d) {
        const Philox q = philox4x32_10((uint32_t)j, (uint32_t)r * 16u + d, sid, (uint32_t)kind, k0, k1);
        const uint64_t u0 = (((uint64_t)q.v[1] << 32) | q.v[0]) & mask;
        const uint64_t u1 = (((uint64_t)q.v[3] << 32) | q.v[2]) & mask;
        if (!ok0 && u0 < p) {
          val[0] = u0;
          ok0 = true;
        }
        if (!ok1 && u1 < p) {
          val[1] = u1;
          ok1 = true;
        }
      }
      if (!(ok0 && ok1)) atomicExch(err, 1);
      out[(size_t)r * N + j] = make_ulonglong2(val[0], val[1]);
    }
    return;
  }
  if (kind == UNIFORM_U32) {
    // one Philox block per Gaussian element: word 0 for coefficient j, word 1 for
    // j + N; every prime exceeds 2^32, so the value itself is its residue everywhere
    const Philox q = philox4x32_10((uint32_t)j, 0, sid, (uint32_t)kind, k0, k1);
    for (int r = 0; r < nres; ++r) out[(size_t)r * N + j] = make_ulonglong2(q.v[0], q.v[1]);
    return;
  }
  int64_t v0 = 0, v1 = 0;
  const int nphi_log = 31 - __clz(2 * N);
  const bool ok0 = small_value(kind, (uint32_t)j, sid, k0, k1, nphi_log, v0);
  const bool ok1 = small_value(kind, (uint32_t)(j + N), sid, k0, k1, nphi_log, v1);
  if (!(ok0 && ok1)) atomicExch(err, 1);
  for (int r = 0; r < nres; ++r) {
    const uint64_t p = mc[rid_off + r].p;
    out[(size_t)r * N + j] = make_ulonglong2(lift(v0, p), lift(v1, p));
  }
}

// Exactly h = min(64, nphi) nonzero coefficients, values +-1, positions
// uniform without replacement: one block per polynomial, thread 0 draws the
// positions sequentially against a shared bitmap (h is small).
__global__ void __launch_bounds__(256) k_sample_hw(ulonglong2* __restrict__ out, const ModConst* __restrict__ mc,
                                                   int N, int logNphi, int nres, int rid_off, uint32_t k0,
                                                   uint32_t k1, uint32_t sid0, long long poly_stride,
                                                   int* __restrict__ err, const uint32_t* __restrict__ ids) {
  extern __shared__ uint32_t bitmap[];  // nphi bits
  __shared__ int pos[64];
  __shared__ int sgn[64];
  const int nphi = 2 * N;
  const uint32_t sid = ids ? ids[blockIdx.x] : sid0 + blockIdx.x;
  out += blockIdx.x * poly_stride;
  for (int i = threadIdx.x; i < (nphi + 31) / 32; i += blockDim.x) bitmap[i] = 0;
  for (int r = 0; r < nres; ++r)
    for (int i = threadIdx.x; i < N; i += blockDim.x) out[(size_t)r * N + i] = make_ulonglong2(0, 0);
  __syncthreads();
  const int h = nphi < 64 ? nphi : 64;
  if (threadIdx.x == 0) {
    for (int i = 0; i < h; ++i) {
      bool placed = false;
      for (uint32_t d = 0; d < 1024 && !placed; ++d) {
        const Philox q = philox4x32_10((uint32_t)i, d, sid, (uint32_t)HAMMINGWEIGHT, k0, k1);
        const int ps = logNphi == 0 ? 0 : (int)(q.v[0] >> (32 - logNphi));
        if (!(bitmap[ps >> 5] & (1u << (ps & 31)))) {
          bitmap[ps >> 5] |= 1u << (ps & 31);
          pos[i] = ps;
          sgn[i] = (q.v[1] & 1u) ? -1 : 1;
          placed = true;
        }
      }
      if (!placed) {
        atomicExch(err, 1);
        pos[i] = -1;
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < h * nres; t += blockDim.x) {
    const int i = t % h, r = t / h;
    const int ps = pos[i];
    if (ps < 0) continue;
    const uint64_t p = mc[rid_off + r].p;
    const uint64_t v = sgn[i] > 0 ? 1 : p - 1;
    uint64_t* o = reinterpret_cast<uint64_t*>(out + (size_t)r * N + (ps % N));
    o[ps / N] = v;
  }
}

std::atomic<unsigned long long> g_cdt_done{0};

int upload_cdt() {
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ULL << (dev & 63);
  if (g_cdt_done.load() & bit) return CP_OK_;
  if (cudaMemcpyToSymbol(c_cdt_signed, kCdtSigned, sizeof(kCdtSigned)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_cdt_folded, kCdtFolded, sizeof(kCdtFolded)) != cudaSuccess)
    return cuda_fail("cudaMemcpyToSymbol(cdt)");
  g_cdt_done.fetch_or(bit);
  return CP_OK_;
}

}  // namespace

int sample_poly(const Engine& e, void* out_v, int base, int kind, uint64_t seed, uint32_t stream_id, int npolys,
                cudaStream_t st, const uint32_t* ids) {
  if (kind < 0 || kind > ZO_HALF || kind == SIGNED_DG) {
    set_error("sample: unknown distribution");
    return CP_ERR_INVALID_;
  }
  const int nres = e.n_residues(base);
  if (nres <= 0 || base == 3) {
    set_error("sample: base must be Q, B or QB");
    return CP_ERR_INVALID_;
  }
  if (int rc = upload_cdt()) return rc;
  // cuPoly's CKKS build samples the small distributions signed (src/cuda/sampler.cu:
  // 73-106, 459-493): narrow {0, 1, 2} with 2 -> p - 1, i.e. uniform {-1, 0, +1}, and
  // the discrete Gaussian without the absolute value.
  if (e.ckks_prec) {
    if (kind == NARROW) kind = TERNARY;
    else if (kind == DISCRETE_GAUSSIAN) kind = SIGNED_DG;
  }
  int* err = e.d_err;
  auto* out = reinterpret_cast<ulonglong2*>(out_v);
  const long long ps = (long long)nres * e.N;
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  if (kind == HAMMINGWEIGHT) {
    const int words = (e.nphi + 31) / 32;
    k_sample_hw<<<npolys, 256, words * 4, st>>>(out, e.d_mc, e.N, e.logN + 1, nres, e.rid_offset(base), k0, k1,
                                                stream_id, ps, err, ids);
  } else {
    dim3 grid((e.N + 255) / 256, npolys);
    k_sample<<<grid, 256, 0, st>>>(out, e.d_mc, e.N, nres, e.rid_offset(base), kind, k0, k1, stream_id, ps, err,
                                   ids);
  }
  return check_launch("sample");
}

}  // namespace cpoly
