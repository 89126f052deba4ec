// Elementwise evaluation of the modular primitives every kernel is built from
// (modarith.cuh), for exhaustive-edge and random tests against big-integer
// arithmetic.  cuPoly tests its device functions directly
// (TestDGT.{mod, addmod, submod, mulmod, powmod, GIAdd, GISub, GIMul},
// tests/unit_tests/test_bfv_mode.cu:243-438); this entry point gives the same
// reach to the primitives behind the C ABI.
#include "../../include/cupoly_b200.h"
#include "launch.cuh"

namespace {

using namespace cpoly;

// a ^ e mod p by square-and-multiply on mul_mod (cuPoly's fast_pow, dgt.cu:508-518)
__device__ uint64_t pow_mod(uint64_t a, uint64_t e, const ModConst& m) {
  uint64_t r = 1 % m.p, b = a;
  for (; e; e >>= 1) {
    if (e & 1) r = mul_mod(r, b, m);
    b = mul_mod(b, b, m);
  }
  return r;
}

__global__ void __launch_bounds__(256) k_modarith(int op, const uint64_t* __restrict__ a,
                                                  const uint64_t* __restrict__ b, const uint64_t* __restrict__ c,
                                                  uint64_t* __restrict__ out, long long n, ModConst m) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t p = m.p;
  switch (op) {
    case CP_MODOP_ADD: out[i] = add_mod(a[i], b[i], p); break;
    case CP_MODOP_SUB: out[i] = sub_mod(a[i], b[i], p); break;
    case CP_MODOP_NEG: out[i] = neg_mod(a[i], p); break;
    case CP_MODOP_MULMOD: out[i] = mul_mod(a[i], b[i], m); break;
    case CP_MODOP_SHOUP: out[i] = shoup_mul(a[i], b[i], c[i], p); break;
    case CP_MODOP_RED128: out[i] = red128(a[i], b[i], m); break;
    case CP_MODOP_POW: out[i] = pow_mod(a[i], b[i], m); break;
    case CP_MODOP_GIMUL: {  // element i = (a[2i], a[2i+1]) x (b[2i], b[2i+1])
      uint64_t r, im;
      gi_mul(r, im, a[2 * i], a[2 * i + 1], b[2 * i], b[2 * i + 1], m);
      out[2 * i] = r;
      out[2 * i + 1] = im;
      break;
    }
    case CP_MODOP_GIMUL_CONST3: {  // element i times (b[2i] + b[2i+1] i) by the Karatsuba triple
      // k = (w_re, w_im - w_re, w_re + w_im) with Shoup companions, as the DGT twist tables
      const uint64_t wr = b[2 * i], wi = b[2 * i + 1];
      const uint64_t k1c = sub_mod(wi, wr, p), k2c = add_mod(wr, wi, p);
      const uint64_t xr = a[2 * i], xi = a[2 * i + 1];
      const uint64_t k1 = shoup_mul(xr + xi, wr, c[3 * i], p);
      const uint64_t k2 = shoup_mul(xr, k1c, c[3 * i + 1], p);
      const uint64_t k3 = shoup_mul(xi, k2c, c[3 * i + 2], p);
      out[2 * i] = sub_mod(k1, k3, p);
      out[2 * i + 1] = add_mod(k1, k2, p);
      break;
    }
    default: break;
  }
}

}  // namespace

extern "C" int cp_modarith_eval(int op, const uint64_t* a, const uint64_t* b, const uint64_t* c, uint64_t* out,
                                long long n, uint64_t p, void* stream) {
  if (op < CP_MODOP_ADD || op > CP_MODOP_GIMUL_CONST3 || !a || !out || n < 0 || p < 3 || !(p & 1) || (p >> 63)) {
    set_error("cp_modarith_eval: bad op, pointer, count or modulus (odd, 3 <= p < 2^63)");
    return CP_ERR_INVALID;
  }
  const bool needs_b = op != CP_MODOP_NEG, needs_c = op == CP_MODOP_SHOUP || op == CP_MODOP_GIMUL_CONST3;
  if ((needs_b && !b) || (needs_c && !c)) {
    set_error("cp_modarith_eval: missing operand array");
    return CP_ERR_INVALID;
  }
  if (n == 0) return CP_OK;
  const ModConst m = h_modconst(p);
  const unsigned blocks = (unsigned)((n + 255) / 256);
  k_modarith<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(op, a, b, c, out, n, m);
  return check_launch("cp_modarith_eval");
}
