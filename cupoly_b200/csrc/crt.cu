// Coefficient I/O on the device: big-integer coefficients <-> RNS residues,
// and the binary residue wire format.
//
// Replaces cuPoly's host-side NTL conversions poly_crt / poly_icrt
// (src/arithmetic/polynomial.cu:190-296), which reduce every ZZ coefficient
// modulo each prime on the host and recombine with NTL's CRT on read-back,
// and the string forms poly_export_residues / poly_import_residues
// (polynomial.cu:1291-1383).
//
// Coefficient layout: unsigned integers of `nlimbs` 64-bit limbs, least
// significant first, coefficient-major: uint64_t[npolys][nphi][nlimbs].
//  * CRT: residue r of coefficient x = sum_l x_l (2^(64 l) mod q_r), a lazy
//    192-bit dot product with one final reduction.
//  * ICRT: the mixed-radix digits d_i of X (exact, word-size), then
//    X = d_0 + q_0 (d_1 + q_1 (d_2 + ...)) by multi-limb Horner; X in [0, Q).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/cupoly_b200.h"
#include "launch.cuh"

namespace cpoly {

namespace {

constexpr int kMaxIcrt = 24;  // largest base recombined by cp_icrt (|Q|, |B| <= 24)

// One thread per Gaussian element (coefficients j and j + N) of one residue.
__global__ void __launch_bounds__(256) k_crt(ulonglong2* __restrict__ out, const uint64_t* __restrict__ coefs,
                                             int nlimbs, int N, int nres, int rid_off,
                                             const ModConst* __restrict__ mc, const uint64_t* __restrict__ pow64,
                                             const uint64_t* __restrict__ pow64m) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  const int y = blockIdx.y;  // poly * nres + r
  const int r = y % nres, poly = y / nres;
  const int rid = rid_off + r;
  const ModConst m = mc[rid];
  const uint64_t* w = pow64 + (size_t)rid * kMaxLimbs;
  const uint64_t* c0 = coefs + ((size_t)poly * 2 * N + j) * nlimbs;
  const uint64_t* c1 = c0 + (size_t)N * nlimbs;
  if (m.pm) {  // 63-bit primes (2^64 mod p < 2^32): lazy 192-bit sums, one reduction
    uint64_t l0 = 0, h0 = 0, t0 = 0, l1 = 0, h1 = 0, t1 = 0;
    for (int l = 0; l < nlimbs; ++l) {  // each product < 2^127; 64 terms < 2^133
      const uint64_t wl = __ldg(w + l);
      mac192(l0, h0, t0, c0[l], wl);
      mac192(l1, h1, t1, c1[l], wl);
    }
    out[(size_t)y * N + j] =
        make_ulonglong2(red192(l0, h0, t0, m.p, m.r1, m.r2), red192(l1, h1, t1, m.p, m.r1, m.r2));
  } else {  // other primes: one Montgomery product per limb with 2^(64 l) in Montgomery form
    const uint64_t* wm = pow64m + (size_t)rid * kMaxLimbs;
    uint64_t a0 = 0, a1 = 0;
    for (int l = 0; l < nlimbs; ++l) {
      const uint64_t wl = __ldg(wm + l);
      a0 = add_mod(a0, mont_mul(c0[l], wl, m.p, m.pneg), m.p);
      a1 = add_mod(a1, mont_mul(c1[l], wl, m.p, m.pneg), m.p);
    }
    out[(size_t)y * N + j] = make_ulonglong2(a0, a1);
  }
}

// One thread per coefficient (index jj in [0, nphi)) of polynomial blockIdx.y.
__global__ void __launch_bounds__(128) k_icrt(uint64_t* __restrict__ coefs, int nlimbs,
                                              const ulonglong2* __restrict__ in, int N, int ns, int src_off,
                                              const ModConst* __restrict__ mc, const uint64_t* __restrict__ inv,
                                              const uint64_t* __restrict__ inv_s) {
  const int jj = blockIdx.x * blockDim.x + threadIdx.x;
  if (jj >= 2 * N) return;
  const int poly = blockIdx.y;
  const int el = jj < N ? jj : jj - N;
  const bool hi = jj >= N;
  uint64_t d[kMaxIcrt];
  for (int i = 0; i < ns; ++i) {
    const ulonglong2 x = in[((size_t)poly * ns + i) * N + el];
    d[i] = hi ? x.y : x.x;
  }
  // mixed-radix digits: d_i = (x_i - d_0 - d_1 s_0 - ...) / (s_0 ... s_{i-1}) mod s_i
  for (int i = 1; i < ns; ++i) {
    const uint64_t si = mc[src_off + i].p;
    uint64_t y = d[i];
    for (int l = 0; l < i; ++l) {
      uint64_t dl = d[l];  // d_l < s_l: one subtraction for primes of one size, a division otherwise
      if (dl >= si) dl = dl - si < si ? dl - si : dl % si;
      const int c = i * (i - 1) / 2 + l;
      y = shoup_mul(y + si - dl, __ldg(inv + c), __ldg(inv_s + c), si);
    }
    d[i] = y;
  }
  // X = d_{ns-1}; X = X s_i + d_i for i = ns-2 .. 0, in 64-bit limbs
  uint64_t X[kMaxIcrt];
  int n = 1;
  X[0] = d[ns - 1];
  for (int i = ns - 2; i >= 0; --i) {
    const uint64_t si = mc[src_off + i].p;
    uint64_t carry = d[i];
    for (int l = 0; l < n; ++l) {
      const uint64_t lo = X[l] * si, hi2 = mulhi64(X[l], si);
      const uint64_t s = lo + carry;
      carry = hi2 + (s < lo);
      X[l] = s;
    }
    if (carry) X[n++] = carry;
  }
  uint64_t* o = coefs + ((size_t)poly * 2 * N + jj) * nlimbs;
  for (int l = 0; l < nlimbs; ++l) o[l] = l < n ? X[l] : 0;
}

__global__ void __launch_bounds__(256) k_icrt_t(uint64_t* __restrict__ coefs, int nlimbs,
                                                const ulonglong2* __restrict__ in, int N) {
  const int jj = blockIdx.x * blockDim.x + threadIdx.x;
  if (jj >= 2 * N) return;
  const int poly = blockIdx.y;
  const ulonglong2 x = in[(size_t)poly * N + (jj < N ? jj : jj - N)];
  uint64_t* o = coefs + ((size_t)poly * 2 * N + jj) * nlimbs;
  o[0] = jj < N ? x.x : x.y;
  for (int l = 1; l < nlimbs; ++l) o[l] = 0;
}

// Wire header: 16 little-endian 32-bit words.
struct WireHeader {
  uint32_t magic, version, nphi, nres, base, npolys, domain, flags;
  uint32_t reserved[8];
};
static_assert(sizeof(WireHeader) == 64, "wire header is 64 bytes");

const uint64_t* base_primes(const Engine& e, int base, uint64_t* tmp) {
  if (base == CP_TBASE) {
    tmp[0] = e.t;
    return tmp;
  }
  return e.primes.data() + e.rid_offset(base);
}

}  // namespace

}  // namespace cpoly

using namespace cpoly;


#define CRT_REQUIRE(cond, msg) \
  do {                         \
    if (!(cond)) {             \
      set_error(msg);          \
      return CP_ERR_INVALID;   \
    }                          \
  } while (0)

extern "C" {

int cp_crt(const cp_engine* h, void* out, const uint64_t* coefs, int nlimbs, int base, int npolys, void* stream) {
  CRT_REQUIRE(h && out && coefs, "cp_crt: NULL argument");
  CRT_REQUIRE(base == CP_QBASE || base == CP_BBASE || base == CP_QBBASE, "cp_crt: base must be Q, B or QB");
  CRT_REQUIRE(nlimbs >= 1 && nlimbs <= kMaxLimbs, "cp_crt: nlimbs must be in [1, 64]");
  CRT_REQUIRE(npolys >= 0, "cp_crt: npolys < 0");
  const Engine& e = h->e;
  const int nres = e.n_residues(base);
  if (npolys == 0) return CP_OK;
  CRT_REQUIRE((long long)npolys * nres <= 65535, "cp_crt: npolys x residues exceeds 65535");
  dim3 grid((e.N + 255) / 256, npolys * nres);
  k_crt<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<ulonglong2*>(out), coefs, nlimbs, e.N, nres, e.rid_offset(base), e.d_mc,
      e.d_hps + e.ho.pow64, e.d_hps + e.ho.pow64m);
  return check_launch("cp_crt");
}

int cp_icrt(const cp_engine* h, uint64_t* coefs, int nlimbs, const void* in, int base, int npolys, void* stream) {
  CRT_REQUIRE(h && coefs && in, "cp_icrt: NULL argument");
  CRT_REQUIRE(base == CP_QBASE || base == CP_BBASE || base == CP_TBASE, "cp_icrt: base must be Q, B or T");
  CRT_REQUIRE(npolys >= 0 && npolys <= 65535, "cp_icrt: npolys must be in [0, 65535]");
  const Engine& e = h->e;
  const int ns = e.n_residues(base);
  CRT_REQUIRE(nlimbs >= ns && nlimbs <= kMaxLimbs, "cp_icrt: nlimbs must be in [residues of the base, 64]");
  if (npolys == 0) return CP_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const ulonglong2* src = reinterpret_cast<const ulonglong2*>(in);
  if (base == CP_TBASE) {
    dim3 grid((2 * e.N + 255) / 256, npolys);
    k_icrt_t<<<grid, 256, 0, st>>>(coefs, nlimbs, src, e.N);
    return check_launch("cp_icrt");
  }
  CRT_REQUIRE(ns <= kMaxIcrt, "cp_icrt: base larger than 24 primes");
  const uint64_t* inv = e.d_hps + (base == CP_QBASE ? e.ho.qb_inv : e.ho.bq_inv);
  const uint64_t* inv_s = e.d_hps + (base == CP_QBASE ? e.ho.qb_inv_s : e.ho.bq_inv_s);
  dim3 grid((2 * e.N + 127) / 128, npolys);
  k_icrt<<<grid, 128, 0, st>>>(coefs, nlimbs, src, e.N, ns, e.rid_offset(base), e.d_mc, inv, inv_s);
  return check_launch("cp_icrt");
}

size_t cp_wire_bytes(const cp_engine* h, int base, int npolys) {
  if (!h || base < 0 || base > 3 || npolys < 0) return 0;
  const int nres = h->e.n_residues(base);
  return sizeof(WireHeader) + (size_t)nres * 8 + (size_t)npolys * nres * h->e.N * 16;
}

int cp_export_residues(const cp_engine* h, void* host_out, size_t cap, const void* poly, int base, int npolys,
                       int domain, void* stream) {
  CRT_REQUIRE(h && host_out && poly, "cp_export_residues: NULL argument");
  CRT_REQUIRE(base >= 0 && base <= 3 && npolys >= 0, "cp_export_residues: bad base or npolys");
  CRT_REQUIRE(domain == 0 || domain == 1, "cp_export_residues: domain must be 0 (coefficient) or 1 (DGT)");
  const size_t need = cp_wire_bytes(h, base, npolys);
  CRT_REQUIRE(cap >= need, "cp_export_residues: output buffer too small");
  const Engine& e = h->e;
  const int nres = e.n_residues(base);
  WireHeader hd;
  std::memset(&hd, 0, sizeof(hd));
  hd.magic = CP_WIRE_MAGIC;
  hd.version = CP_WIRE_VERSION;
  hd.nphi = (uint32_t)e.nphi;
  hd.nres = (uint32_t)nres;
  hd.base = (uint32_t)base;
  hd.npolys = (uint32_t)npolys;
  hd.domain = (uint32_t)domain;
  unsigned char* o = reinterpret_cast<unsigned char*>(host_out);
  std::memcpy(o, &hd, sizeof(hd));
  uint64_t tmp[1];
  std::memcpy(o + sizeof(hd), base_primes(e, base, tmp), (size_t)nres * 8);
  const size_t body = (size_t)npolys * nres * e.N * 16;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t err = cudaMemcpyAsync(o + sizeof(hd) + (size_t)nres * 8, poly, body, cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) return cuda_fail("cp_export_residues", err);
  return CP_OK;
}

int cp_import_residues(const cp_engine* h, void* poly, const void* host_in, size_t size, int base, int npolys,
                       int* domain_out, void* stream) {
  CRT_REQUIRE(h && poly && host_in, "cp_import_residues: NULL argument");
  CRT_REQUIRE(base >= 0 && base <= 3 && npolys >= 0, "cp_import_residues: bad base or npolys");
  CRT_REQUIRE(size >= sizeof(WireHeader), "cp_import_residues: truncated header");
  const Engine& e = h->e;
  const int nres = e.n_residues(base);
  WireHeader hd;
  const unsigned char* in = reinterpret_cast<const unsigned char*>(host_in);
  std::memcpy(&hd, in, sizeof(hd));
  CRT_REQUIRE(hd.magic == CP_WIRE_MAGIC, "cp_import_residues: bad magic");
  CRT_REQUIRE(hd.version == CP_WIRE_VERSION, "cp_import_residues: unsupported version");
  CRT_REQUIRE(hd.nphi == (uint32_t)e.nphi, "cp_import_residues: ring degree differs from the engine's");
  CRT_REQUIRE(hd.base == (uint32_t)base && hd.nres == (uint32_t)nres, "cp_import_residues: base differs");
  CRT_REQUIRE(hd.npolys == (uint32_t)npolys, "cp_import_residues: polynomial count differs");
  CRT_REQUIRE(hd.domain <= 1 && hd.flags == 0, "cp_import_residues: bad domain or flags");
  CRT_REQUIRE(size == cp_wire_bytes(h, base, npolys), "cp_import_residues: size does not match the header");
  uint64_t tmp[1];
  const uint64_t* primes = base_primes(e, base, tmp);
  CRT_REQUIRE(std::memcmp(in + sizeof(hd), primes, (size_t)nres * 8) == 0,
              "cp_import_residues: primes differ from the engine's");
  const uint64_t* body = reinterpret_cast<const uint64_t*>(in + sizeof(hd) + (size_t)nres * 8);
  // every residue must be canonical: a malformed request is refused before it reaches the GPU.
  // Rows (polynomial, residue) are checked on up to 8 host threads for large payloads.
  const long long rows = (long long)npolys * nres;
  const size_t row_words = (size_t)2 * e.N;
  std::atomic<bool> bad{false};
  auto check_rows = [&](long long lo, long long hi) {
    for (long long y = lo; y < hi && !bad.load(std::memory_order_relaxed); ++y) {
      const uint64_t q = primes[y % nres];
      const uint64_t* row = body + (size_t)y * row_words;
      uint64_t worst = 0;
      for (size_t j = 0; j < row_words; ++j) worst = row[j] > worst ? row[j] : worst;
      if (worst >= q) bad.store(true);
    }
  };
  const size_t bytes = (size_t)rows * row_words * 8;
  const unsigned hw = std::thread::hardware_concurrency();
  // at most 8 threads and half the host's cores: on a 16-core host 8 threads measured best
  // (42 MB: 2.6 ms with the copy; 16 threads 4.5 ms, as the copy then runs at pageable speed)
  const long long nthreads =
      bytes < ((size_t)4 << 20) ? 1 : std::min<long long>(std::min(hw > 1 ? hw / 2 : 1u, 8u), rows);
  if (nthreads <= 1) {
    check_rows(0, rows);
  } else {
    // no exception may cross the C ABI: if a thread cannot be started, the rows it would
    // have checked are checked on this thread
    std::vector<std::thread> pool;
    long long started = 0;
    try {
      for (; started < nthreads; ++started)
        pool.emplace_back(check_rows, rows * started / nthreads, rows * (started + 1) / nthreads);
    } catch (...) {
    }
    if (started < nthreads) check_rows(rows * started / nthreads, rows);
    for (auto& th : pool) th.join();
  }
  if (bad.load()) {
    set_error("cp_import_residues: residue not reduced modulo its prime");
    return CP_ERR_INVALID;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t err = cudaMemcpyAsync(poly, body, (size_t)npolys * nres * e.N * 16, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) return cuda_fail("cp_import_residues", err);
  if (domain_out) *domain_out = (int)hd.domain;
  return CP_OK;
}

}  // extern "C"
