// Pointwise kernels on DGT-domain residues (replaces cuPoly's add_dgt,
// sub_dgt, double_add_dgt, dr2_dgt, mul_dgt<GI>, mul_dgt<u64>, muladd_dgt in
// src/cuda/dgt.cu:1096-1499 and polynomial_negate / polynomial_op_by_int /
// polynomial_double_op_by_int in src/cuda/cudaengine.cu:115-302).
//
// All are HBM-streaming: one 16-byte Gaussian element per thread per step,
// 128-bit loads, grid = (x-chunks, residues) so each block reads its
// residue's constants once.
#include "launch.cuh"
#include "pointwise.cuh"

namespace cpoly {

namespace {

using u2 = ulonglong2;

// blockIdx.y enumerates (polynomial, residue) pairs of a densely packed batch.
template <class F>
__global__ void __launch_bounds__(256)
    k_elementwise(F f, int N, int nres, int rid_off, const ModConst* __restrict__ mc, const int* __restrict__ rid_list) {
  const int y = blockIdx.y + blockIdx.z * gridDim.y;
  const ModConst m = mc[rid_list ? rid_list[y] : rid_off + y % nres];
  const size_t base = (size_t)y * N;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) f(base + j, m);
}

template <class F>
int launch_ew(const Engine& e, F f, int base, cudaStream_t st, int npolys = 1, const int* rid_list = nullptr) {
  const int nres = rid_list ? 1 : e.n_residues(base);
  if (nres <= 0) {
    set_error("pointwise: unknown base");
    return CP_ERR_INVALID_;
  }
  if (npolys <= 0) return CP_OK_;
  const int threads = 256;
  int bx = (e.N + threads - 1) / threads;
  if (bx > 4096) bx = 4096;
  const long long rows = (long long)nres * npolys;
  int gy = (int)rows, gz = 1;
  while (gy > 65535) {  // split rows over z when needed (rows is a multiple of gz)
    gz *= 2;
    if (rows % gz) {
      set_error("pointwise: batch too large");
      return CP_ERR_INVALID_;
    }
    gy = (int)(rows / gz);
  }
  dim3 grid(bx, gy, gz);
  k_elementwise<<<grid, threads, 0, st>>>(f, e.N, nres, rid_list ? 0 : e.rid_offset(base), e.d_mc, rid_list);
  return check_launch("pointwise");
}

struct AddF {
  u2* c;
  const u2 *a, *b;
  __device__ void operator()(size_t i, const ModConst& m) const {
    const u2 x = a[i], y = b[i];
    c[i] = make_ulonglong2(add_mod(x.x, y.x, m.p), add_mod(x.y, y.y, m.p));
  }
};
struct SubF {
  u2* c;
  const u2 *a, *b;
  __device__ void operator()(size_t i, const ModConst& m) const {
    const u2 x = a[i], y = b[i];
    c[i] = make_ulonglong2(sub_mod(x.x, y.x, m.p), sub_mod(x.y, y.y, m.p));
  }
};
struct DoubleAddF {
  u2 *c1, *c2;
  const u2 *a1, *b1, *a2, *b2;
  __device__ void operator()(size_t i, const ModConst& m) const {
    const u2 x = a1[i], y = b1[i], z = a2[i], w = b2[i];
    c1[i] = make_ulonglong2(add_mod(x.x, y.x, m.p), add_mod(x.y, y.y, m.p));
    c2[i] = make_ulonglong2(add_mod(z.x, w.x, m.p), add_mod(z.y, w.y, m.p));
  }
};
struct MulF {
  u2* c;
  const u2 *a, *b;
  __device__ void operator()(size_t i, const ModConst& m) const {
    const u2 x = a[i], y = b[i];
    uint64_t r, im;
    gi_mul(r, im, x.x, x.y, y.x, y.y, m);
    c[i] = make_ulonglong2(r, im);
  }
};
struct MulU64F {
  u2* c;
  const u2* a;
  const uint64_t* b;
  __device__ void operator()(size_t i, const ModConst& m) const {
    const u2 x = a[i];
    const uint64_t y = b[i];
    c[i] = make_ulonglong2(mul_mod(x.x, y, m), mul_mod(x.y, y, m));
  }
};
struct MulAddF {
  u2* d;
  const u2 *a, *b, *c;
  __device__ void operator()(size_t i, const ModConst& m) const {
    const u2 x = a[i], y = b[i], z = c[i];
    uint64_t r, im;
    gi_mul(r, im, x.x, x.y, y.x, y.y, m);
    d[i] = make_ulonglong2(add_mod(r, z.x, m.p), add_mod(im, z.y, m.p));
  }
};
struct Dr2F {
  u2 *c21, *c22, *c23;
  const u2 *c01, *c02, *c11, *c12;
  __device__ void operator()(size_t i, const ModConst& m) const {
    const u2 a0 = c01[i], a1 = c02[i], b0 = c11[i], b1 = c12[i];
    uint64_t r1, i1, r2, i2, r3, i3, r4, i4;
    gi_mul(r1, i1, a0.x, a0.y, b0.x, b0.y, m);
    gi_mul(r2, i2, a0.x, a0.y, b1.x, b1.y, m);
    gi_mul(r3, i3, a1.x, a1.y, b0.x, b0.y, m);
    gi_mul(r4, i4, a1.x, a1.y, b1.x, b1.y, m);
    const uint64_t p = m.p;
    c21[i] = make_ulonglong2(r1, i1);
    c22[i] = make_ulonglong2(add_mod(r2, r3, p), add_mod(i2, i3, p));
    c23[i] = make_ulonglong2(r4, i4);
  }
};
struct NegF {
  u2* b;
  const u2* a;
  __device__ void operator()(size_t i, const ModConst& m) const {
    const u2 x = a[i];
    b[i] = make_ulonglong2(neg_mod(x.x, m.p), neg_mod(x.y, m.p));
  }
};
__device__ __forceinline__ uint64_t red1(uint64_t x, uint64_t p) { return x >= p ? x - p : x; }
__device__ __forceinline__ u2 op_int(u2 x, uint64_t v, int op, const ModConst& m) {
  const uint64_t s = red1(v, m.p);  // v < 2^64 < 2p
  switch (op) {
    case 0: return make_ulonglong2(add_mod(x.x, s, m.p), x.y);
    case 1: return make_ulonglong2(sub_mod(x.x, s, m.p), x.y);
    default: return make_ulonglong2(mul_mod(x.x, s, m), mul_mod(x.y, s, m));
  }
}
struct OpIntF {
  u2* b;
  const u2* a;
  uint64_t x;
  int op;
  __device__ void operator()(size_t i, const ModConst& m) const { b[i] = op_int(a[i], x, op, m); }
};
struct DoubleOpIntF {
  u2 *b1, *b2;
  const u2 *a1, *a2;
  uint64_t x1, x2;
  int op;  // 0 = ADD, 2 = MUL
  __device__ void operator()(size_t i, const ModConst& m) const {
    b1[i] = op_int(a1[i], x1, op, m);
    b2[i] = op_int(a2[i], x2, op, m);
  }
};

// c = sum_t a_t b_t (+ c when `acc`) over up to kDotTerms pairs, one pass,
// one thread per element.  The pseudo-Mersenne primes sum the Karatsuba
// products P1 = a0 b0, P2 = a1 b1, P3 = (a0 + a1)(b0 + b1) (each below 2^128:
// a0 + a1, b0 + b1 < 2^64) in three 192-bit accumulators and reduce once per
// element: re = P1 - P2, im = P3 - P1 - P2.  64 terms stay below 2^134, inside
// red192's t < 2^8 bound, and red192 needs 2^64 mod p < 2^32, which holds for
// these primes.  Other primes reduce every product.  Each element is read
// completely before its output is written, so c may alias any operand of the
// launch.
struct DotArgs {
  const u2* a[kDotTerms];
  const u2* b[kDotTerms];
};

// sum_{t < n} x_t y_t mod p for one element, (x_t, y_t) = load(t).
template <class Load>
__device__ __forceinline__ u2 dot_elem(int n, const ModConst& m, Load load) {
  uint64_t sr = 0, si = 0;
  if (m.pm) {
    uint64_t l1 = 0, h1 = 0, t1 = 0, l2 = 0, h2 = 0, t2 = 0, l3 = 0, h3 = 0, t3 = 0;
#pragma unroll 4
    for (int t = 0; t < n; ++t) {
      u2 x, y;
      load(t, x, y);
      mac192(l1, h1, t1, x.x, y.x);
      mac192(l2, h2, t2, x.y, y.y);
      mac192(l3, h3, t3, x.x + x.y, y.x + y.y);
    }
    const uint64_t p1 = red192(l1, h1, t1, m.p, m.r1, m.r2), p2 = red192(l2, h2, t2, m.p, m.r1, m.r2),
                   p3 = red192(l3, h3, t3, m.p, m.r1, m.r2);
    sr = sub_mod(p1, p2, m.p);
    si = sub_mod(sub_mod(p3, p1, m.p), p2, m.p);
  } else {
    for (int t = 0; t < n; ++t) {
      u2 x, y;
      load(t, x, y);
      uint64_t r, im;
      gi_mul(r, im, x.x, x.y, y.x, y.y, m);
      sr = add_mod(sr, r, m.p);
      si = add_mod(si, im, m.p);
    }
  }
  return make_ulonglong2(sr, si);
}

__global__ void __launch_bounds__(256)
    k_dot(DotArgs args, int n, u2* c, int acc, int N, int rid_off, const ModConst* __restrict__ mc) {
  const ModConst m = mc[rid_off + blockIdx.y];
  const size_t base = (size_t)blockIdx.y * N;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const size_t i = base + j;
    u2 r = dot_elem(n, m, [&](int t, u2& x, u2& y) {
      x = args.a[t][i];
      y = args.b[t][i];
    });
    if (acc) {
      const u2 z = c[i];
      r = make_ulonglong2(add_mod(r.x, z.x, m.p), add_mod(r.y, z.y, m.p));
    }
    c[i] = r;
  }
}

// Batched form: polynomial q of c = sum_t a[q n + t] b[q n + t] (b[t] when b is shared);
// every operand a polynomial of `poly` elements, residue r at offset r N.
__global__ void __launch_bounds__(256)
    k_dot_batch(const u2* __restrict__ a, const u2* __restrict__ b, u2* __restrict__ c, int n, int b_shared, int N,
                int nres, int rid_off, const ModConst* __restrict__ mc) {
  const int r = blockIdx.y % nres;
  const size_t q = blockIdx.y / nres + (size_t)blockIdx.z * (gridDim.y / nres);
  const ModConst m = mc[rid_off + r];
  const size_t poly = (size_t)nres * N;
  const u2* ap = a + q * n * poly + (size_t)r * N;
  const u2* bp = b + (b_shared ? 0 : q * n * poly) + (size_t)r * N;
  u2* cp = c + q * poly + (size_t)r * N;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x)
    cp[j] = dot_elem(n, m, [&](int t, u2& x, u2& y) {
      x = ap[t * poly + j];
      y = bp[t * poly + j];
    });
}

}  // namespace

#define U2(p) reinterpret_cast<u2*>(p)
#define CU2(p) reinterpret_cast<const u2*>(p)

int pw_add(const Engine& e, void* c, const void* a, const void* b, int base, cudaStream_t st) {
  return launch_ew(e, AddF{U2(c), CU2(a), CU2(b)}, base, st);
}
int pw_sub(const Engine& e, void* c, const void* a, const void* b, int base, cudaStream_t st) {
  return launch_ew(e, SubF{U2(c), CU2(a), CU2(b)}, base, st);
}
int pw_double_add(const Engine& e, void* c1, const void* a1, const void* b1, void* c2, const void* a2,
                  const void* b2, int base, cudaStream_t st) {
  return launch_ew(e, DoubleAddF{U2(c1), U2(c2), CU2(a1), CU2(b1), CU2(a2), CU2(b2)}, base, st);
}
int pw_mul(const Engine& e, void* c, const void* a, const void* b, int base, cudaStream_t st, int npolys) {
  return launch_ew(e, MulF{U2(c), CU2(a), CU2(b)}, base, st, npolys);
}
int pw_mul_list(const Engine& e, void* c, const void* a, const void* b, const int* rid_list, int nlist,
                cudaStream_t st) {
  return launch_ew(e, MulF{U2(c), CU2(a), CU2(b)}, 0, st, nlist, rid_list);
}
int pw_mul_u64(const Engine& e, void* c, const void* a, const uint64_t* b, int base, cudaStream_t st) {
  return launch_ew(e, MulU64F{U2(c), CU2(a), b}, base, st);
}
int pw_muladd(const Engine& e, void* d, const void* a, const void* b, const void* c, int base, cudaStream_t st) {
  return launch_ew(e, MulAddF{U2(d), CU2(a), CU2(b), CU2(c)}, base, st);
}
int pw_dot(const Engine& e, void* c, const void* const* a, const void* const* b, int n, int base,
           cudaStream_t st) {
  const int nres = e.n_residues(base);
  if (nres <= 0) {
    set_error("dot: unknown base");
    return CP_ERR_INVALID_;
  }
  // Launches after the first accumulate into c: c must not be an operand of
  // a later launch, whose input the first launch would already have overwritten.
  for (int t = kDotTerms; t < n; ++t)
    if (a[t] == c || b[t] == c) {
      set_error("dot: the output aliases an operand beyond the first 64 terms");
      return CP_ERR_INVALID_;
    }
  const int threads = 256;
  for (int t0 = 0; t0 < n; t0 += kDotTerms) {
    const int m = n - t0 < kDotTerms ? n - t0 : kDotTerms;
    DotArgs args{};
    for (int t = 0; t < m; ++t) {
      args.a[t] = CU2(a[t0 + t]);
      args.b[t] = CU2(b[t0 + t]);
    }
    int bx = (e.N + threads - 1) / threads;
    if (bx > 4096) bx = 4096;
    k_dot<<<dim3(bx, nres), threads, 0, st>>>(args, m, U2(c), t0 > 0, e.N, e.rid_offset(base), e.d_mc);
    const int rc = check_launch("dot");
    if (rc != CP_OK_) return rc;
  }
  return CP_OK_;
}
int pw_dot_batch(const Engine& e, void* c, const void* a, const void* b, int n, int npolys, bool b_shared, int base,
                 cudaStream_t st) {
  const int nres = e.n_residues(base);
  if (nres <= 0) {
    set_error("dot_batch: unknown base");
    return CP_ERR_INVALID_;
  }
  if (n < 1 || n > kDotTerms) {
    set_error("dot_batch: n must be in [1, 64]");
    return CP_ERR_INVALID_;
  }
  if (npolys <= 0) return CP_OK_;
  const int threads = 256;
  int bx = (e.N + threads - 1) / threads;
  if (bx > 4096) bx = 4096;
  // (polynomial, residue) rows over y, split over z in whole polynomials when needed
  long long gz = 1;
  while ((long long)npolys * nres / gz > 65535 || npolys % gz) ++gz;
  if (gz > 65535) {
    set_error("dot_batch: batch too large");
    return CP_ERR_INVALID_;
  }
  const dim3 grid(bx, (unsigned)((long long)npolys / gz * nres), (unsigned)gz);
  k_dot_batch<<<grid, threads, 0, st>>>(CU2(a), CU2(b), U2(c), n, b_shared ? 1 : 0, e.N, nres, e.rid_offset(base),
                                        e.d_mc);
  return check_launch("dot_batch");
}
int pw_dr2(const Engine& e, void* c21, void* c22, void* c23, const void* c01, const void* c02, const void* c11,
           const void* c12, int base, cudaStream_t st, int npolys) {
  return launch_ew(e, Dr2F{U2(c21), U2(c22), U2(c23), CU2(c01), CU2(c02), CU2(c11), CU2(c12)}, base, st, npolys);
}
int pw_negate(const Engine& e, void* b, const void* a, int base, cudaStream_t st) {
  return launch_ew(e, NegF{U2(b), CU2(a)}, base, st);
}
int pw_op_by_int(const Engine& e, void* b, const void* a, int base, uint64_t x, int op, cudaStream_t st) {
  if (op < 0 || op > 2) {
    set_error("op_by_int: op must be ADD, SUB or MUL");
    return CP_ERR_INVALID_;
  }
  return launch_ew(e, OpIntF{U2(b), CU2(a), x, op}, base, st);
}
int pw_double_op_by_int(const Engine& e, void* b1, const void* a1, void* b2, const void* a2, int base, uint64_t x1,
                        uint64_t x2, int op, cudaStream_t st) {
  int k;
  if (op == 3)
    k = 2;  // MULMUL
  else if (op == 4)
    k = 0;  // ADDADD
  else {
    set_error("double_op_by_int: op must be MULMUL or ADDADD");
    return CP_ERR_INVALID_;
  }
  return launch_ew(e, DoubleOpIntF{U2(b1), U2(b2), CU2(a1), CU2(a2), x1, x2, k}, base, st);
}

}  // namespace cpoly
