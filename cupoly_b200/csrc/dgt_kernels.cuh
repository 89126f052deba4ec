// Discrete Galois transform kernels for sm_100a.
//
// Replaces cuPoly's hdgt_tr / hidgt / hidgt_tr / dgt / idgt kernels
// (cuPoly src/cuda/dgt.cu:681-1067).  The transform computed is the same:
// forward = twist by xi^n, then the N-point DFT with w_N = g^((p-1)/N),
// output in bit-reversed order (X[brev(pos)] at pos); inverse = exact
// inverse including N^-1.  cuPoly's two-pass Na x Nb split produces exactly
// this order, so the DGT-domain bytes agree for the same xi.
//
// Structure (one CTA per residue of one polynomial, N <= 8192 GIs):
//  * the residue stays in shared memory for the whole transform: one HBM
//    read and one HBM write per transform (cuPoly: two of each);
//  * each thread keeps 2^LOGR Gaussian elements in registers and runs a
//    radix-2^LOGR DIF (inverse: DIT) over one contiguous bit field of the
//    index per pass; passes exchange through padded shared memory;
//  * between passes the per-element twiddle w_M^(L brev(pos)) comes from a
//    per-pass table laid out in access order, so global reads coalesce;
//  * every constant multiply is a Shoup product with a precomputed quotient.
// For N > 8192 an element-wise radix-2^S stage (twist + top S bits) runs
// first (forward) or last (inverse) and the CTA kernel handles the
// 2^S sub-transforms.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "engine.cuh"

namespace cpoly {

__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }

// pad16(b + (v << F)) = pad16(b) + pad_off<F>(v) whenever the bits of v << F are clear in b
// (the sum is then a bitwise or, and so is its shift right by 4): every unrolled access of a
// pass addresses shared memory at one per-thread base plus a constant.
template <int F>
__host__ __device__ constexpr int pad_off(int v) {
  return (v << F) + ((v << F) >> 4);
}

template <int LOGNC, int LOGR>
struct PassCfg {
  static constexpr int NP = (LOGNC + LOGR - 1) / LOGR;
  static constexpr int W0 = LOGNC - (NP - 1) * LOGR;
  __host__ __device__ static constexpr int width(int i) { return i == 0 ? W0 : LOGR; }
  __host__ __device__ static constexpr int field(int i) { return LOGNC - W0 - i * LOGR; }
  // Passes i >= 1 whose twiddle table (2^(field + LOGR) entries, each read by
  // 2^LOGR - 1 threads of the CTA) is at most 1024 entries are staged in
  // shared memory once per CTA; the first pass reads each entry once and
  // streams it from global memory.
  __host__ __device__ static constexpr bool staged(int i) {
    return i >= 1 && i < NP && field(i) > 0 && field(i) + LOGR <= 10;
  }
  __host__ __device__ static constexpr int soff(int i) {  // entries before pass i's staged table
    int o = 0;
    for (int q = 1; q < i; ++q)
      if (staged(q)) o += 1 << (field(q) + LOGR);
    return o;
  }
  __host__ __device__ static constexpr int stotal() { return soff(NP); }
};

// Copy the staged twiddle tables of the passes (offsets `off` into the residue's
// table block) into shared memory.
template <int LOGNC, int LOGR>
__device__ __forceinline__ void stage_twiddles(ulonglong2* stw, const ulonglong2* tab, const int* off) {
  using C = PassCfg<LOGNC, LOGR>;
  constexpr int T = (1 << LOGNC) >> LOGR;
#pragma unroll
  for (int i = 1; i < C::NP; ++i)
    if (C::staged(i)) {
      const ulonglong2* src = tab + off[i];
      ulonglong2* dst = stw + C::soff(i);
      for (int j = threadIdx.x; j < (1 << (C::field(i) + LOGR)); j += T) dst[j] = __ldg(src + j);
    }
}

// In-register 2^W-point Gentleman-Sande DIF (natural in, bit-reversed out).
// rad[j] = w_R^j, R = 2^LOGR; the 2^W-point root is w_R^(2^(LOGR-W)).
// LAZY: every output but the first goes straight into a Shoup product (the pass
// twiddle), which takes any value below 2^64, so the last stage leaves those in
// [0, 2p) without the final correction.
template <int W, int LOGR, bool LAZY = false>
__device__ __forceinline__ void dif_regs(uint64_t* xr, uint64_t* xi, const ulonglong2* rad, uint64_t p) {
#pragma unroll
  for (int s = 0; s < W; ++s) {
    const int m = (1 << W) >> (s + 1);
#pragma unroll
    for (int i = 0; i < (1 << W); ++i) {
      if ((i & m) == 0) {
        const int j = i & (m - 1);
        const uint64_t ar = xr[i], ai = xi[i], br = xr[i + m], bi = xi[i + m];
        if (LAZY && s == W - 1) {
          xr[i] = i == 0 ? add_mod(ar, br, p) : ar + br;
          xi[i] = i == 0 ? add_mod(ai, bi, p) : ai + bi;
          xr[i + m] = ar + p - br;
          xi[i + m] = ai + p - bi;
          continue;
        }
        xr[i] = add_mod(ar, br, p);
        xi[i] = add_mod(ai, bi, p);
        if (j == 0) {
          xr[i + m] = sub_mod(ar, br, p);
          xi[i + m] = sub_mod(ai, bi, p);
        } else {
          const ulonglong2 w = rad[(j << s) << (LOGR - W)];
          xr[i + m] = shoup_mul(ar + p - br, w.x, w.y, p);
          xi[i + m] = shoup_mul(ai + p - bi, w.x, w.y, p);
        }
      }
    }
  }
}

// In-register 2^W-point Cooley-Tukey DIT with inverse roots (bit-reversed in,
// natural out), unscaled.
// LAZY: the outputs go to the next inverse pass, which reduces the one element it
// does not multiply by a twiddle (lazy_in) and feeds the rest to Shoup products;
// so the last stage leaves every output in [0, 2p) without the final correction.
template <int W, int LOGR, bool LAZY = false>
__device__ __forceinline__ void dit_regs(uint64_t* xr, uint64_t* xi, const ulonglong2* rad, uint64_t p) {
  constexpr int R = 1 << LOGR;
#pragma unroll
  for (int s = W - 1; s >= 0; --s) {
    const int m = (1 << W) >> (s + 1);
#pragma unroll
    for (int i = 0; i < (1 << W); ++i) {
      if ((i & m) == 0) {
        const int j = i & (m - 1);
        const uint64_t ar = xr[i], ai = xi[i];
        uint64_t br = xr[i + m], bi = xi[i + m];
        if (j != 0) {
          const ulonglong2 w = rad[R - ((j << s) << (LOGR - W))];
          br = shoup_mul(br, w.x, w.y, p);
          bi = shoup_mul(bi, w.x, w.y, p);
        }
        if (LAZY && s == 0) {
          xr[i] = ar + br;
          xi[i] = ai + bi;
          xr[i + m] = ar + p - br;
          xi[i + m] = ai + p - bi;
          continue;
        }
        xr[i] = add_mod(ar, br, p);
        xi[i] = add_mod(ai, bi, p);
        xr[i + m] = sub_mod(ar, br, p);
        xi[i + m] = sub_mod(ai, bi, p);
      }
    }
  }
}

// x <- x * (w_re + i w_im) for canonical x, from the Karatsuba triple
// k[0..2] = (w_re, w_im - w_re, w_re + w_im) with Shoup companions:
// re = k1 - k3, im = k1 + k2 for k1 = w_re (x_re + x_im), k2 = x_re (w_im - w_re),
// k3 = x_im (w_re + w_im).  Three constant products instead of four.
__device__ __forceinline__ void gi_mul_const3(uint64_t& xr, uint64_t& xi, const ulonglong2* k, uint64_t p) {
  const ulonglong2 k0 = __ldg(k), k1c = __ldg(k + 1), k2c = __ldg(k + 2);
  const uint64_t k1 = shoup_mul(xr + xi, k0.x, k0.y, p);  // xr + xi < 2p < 2^64
  const uint64_t k2 = shoup_mul(xr, k1c.x, k1c.y, p);
  const uint64_t k3 = shoup_mul(xi, k2c.x, k2c.y, p);
  xr = sub_mod(k1, k3, p);
  xi = add_mod(k1, k2, p);
}

// Bulk prefetch of `bytes` (multiple of 16, 16-byte aligned) into L2 through the
// TMA unit; a hint only, nothing waits on it.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  for (uint32_t o = 0; o < bytes; o += 32768u) {
    const uint32_t n = bytes - o < 32768u ? bytes - o : 32768u;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reinterpret_cast<const char*>(p) + o), "r"(n)
                 : "memory");
  }
}

// One middle/late forward pass (I >= 1), full radix 2^LOGR, data in smem.
template <int LOGNC, int LOGR, int I>
__device__ __forceinline__ void fwd_passes(ulonglong2* sdat, const ulonglong2* srad, const ulonglong2* stw,
                                           const ulonglong2* tab, const DgtTableLayout& L, uint64_t p) {
  using C = PassCfg<LOGNC, LOGR>;
  if constexpr (I < C::NP) {
    constexpr int PF = C::field(I);
    constexpr int R = 1 << LOGR;
    const int c = threadIdx.x;
    const int Lw = c & ((1 << PF) - 1);
    const int base = ((c >> PF) << (PF + LOGR)) + Lw;
    const int pb = pad16(base);
    uint64_t xr[R], xi[R];
#pragma unroll
    for (int v = 0; v < R; ++v) {
      const ulonglong2 a = sdat[pb + pad_off<PF>(v)];
      xr[v] = a.x;
      xi[v] = a.y;
    }
    dif_regs<LOGR, LOGR, (PF > 0)>(xr, xi, srad, p);
    if constexpr (PF > 0) {
      const ulonglong2* tw = C::staged(I) ? stw + C::soff(I) + Lw : tab + L.off_fwd[I] + Lw;
#pragma unroll
      for (int v = 1; v < R; ++v) {
        const ulonglong2 w = C::staged(I) ? tw[v << PF] : __ldg(tw + (v << PF));
        xr[v] = shoup_mul(xr[v], w.x, w.y, p);
        xi[v] = shoup_mul(xi[v], w.x, w.y, p);
      }
    }
#pragma unroll
    for (int v = 0; v < R; ++v) sdat[pb + pad_off<PF>(v)] = make_ulonglong2(xr[v], xi[v]);
    __syncthreads();
    fwd_passes<LOGNC, LOGR, I + 1>(sdat, srad, stw, tab, L, p);
  }
}

template <int LOGNC, int LOGR, int I>
__device__ __forceinline__ void inv_passes(ulonglong2* sdat, const ulonglong2* srad, const ulonglong2* stw,
                                           const ulonglong2* tab, const DgtTableLayout& L, uint64_t p) {
  using C = PassCfg<LOGNC, LOGR>;
  if constexpr (I >= 1) {
    constexpr int PF = C::field(I);
    constexpr int R = 1 << LOGR;
    const int c = threadIdx.x;
    const int Lw = c & ((1 << PF) - 1);
    const int base = ((c >> PF) << (PF + LOGR)) + Lw;
    uint64_t xr[R], xi[R];
#pragma unroll
    for (int v = 0; v < R; ++v) {
      const ulonglong2 a = sdat[pad16(base + (v << PF))];
      xr[v] = a.x;
      xi[v] = a.y;
    }
    if constexpr (PF > 0) {
      const ulonglong2* tw = C::staged(I) ? stw + C::soff(I) + Lw : tab + L.off_inv[I] + Lw;
#pragma unroll
      for (int v = 1; v < R; ++v) {
        const ulonglong2 w = C::staged(I) ? tw[v << PF] : __ldg(tw + (v << PF));
        xr[v] = shoup_mul(xr[v], w.x, w.y, p);
        xi[v] = shoup_mul(xi[v], w.x, w.y, p);
      }
    }
    if constexpr (I < C::NP - 1) {  // written by a lazy pass (I + 1)
      xr[0] = red2p(xr[0], p);
      xi[0] = red2p(xi[0], p);
    }
    dit_regs<LOGR, LOGR, true>(xr, xi, srad, p);
#pragma unroll
    for (int v = 0; v < R; ++v) sdat[pad16(base + (v << PF))] = make_ulonglong2(xr[v], xi[v]);
    __syncthreads();
    inv_passes<LOGNC, LOGR, I - 1>(sdat, srad, stw, tab, L, p);
  }
}

// Split stage inside a thread-block cluster of 2^CL CTAs (one per chunk of 2^LOGNC
// elements of one residue).  Forward: every CTA holds its chunk of the twisted input
// in shared memory; the radix-2^CL DIF over the chunks runs at the positions
// [h SPAN, (h + 1) SPAN) owned by CTA h, reading each chunk's element from its
// owner's shared memory and writing output chunk `pos` back into CTA pos's shared
// memory (distributed shared memory), with the split twiddles -- the arithmetic of
// k_dgt_split, without its HBM pass.  Every thread reads and then rewrites the
// same slot of every peer, and no other thread touches that slot, so the only
// ordering needed is the cluster barrier on each side.
template <int LOGNC, int LOGR, int CL>
__device__ __forceinline__ void cluster_split_fwd(ulonglong2* sdat, int h, const ulonglong2* tab,
                                                  const DgtTableLayout& L, uint64_t p) {
  namespace cg = cooperative_groups;
  constexpr int K = 1 << CL, NC = 1 << LOGNC, T = NC >> LOGR, SPAN = NC / K, R = 1 << LOGR;
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();  // every chunk twisted and in place
  ulonglong2* peer[K];
#pragma unroll
  for (int q = 0; q < K; ++q) peer[q] = cl.map_shared_rank(sdat, q);
  for (int t = threadIdx.x; t < SPAN; t += T) {
    const int Lw = h * SPAN + t;
    uint64_t xr[K], xi[K];
#pragma unroll
    for (int hh = 0; hh < K; ++hh) {
      const ulonglong2 a = peer[hh][pad16(Lw)];
      xr[hh] = a.x;
      xi[hh] = a.y;
    }
#pragma unroll
    for (int s = 0; s < CL; ++s) {
      const int m = K >> (s + 1);
#pragma unroll
      for (int i = 0; i < K; ++i)
        if ((i & m) == 0) {
          const int j = i & (m - 1);
          const uint64_t ar = xr[i], ai = xi[i], br = xr[i + m], bi = xi[i + m];
          xr[i] = add_mod(ar, br, p);
          xi[i] = add_mod(ai, bi, p);
          if (j == 0) {
            xr[i + m] = sub_mod(ar, br, p);
            xi[i + m] = sub_mod(ai, bi, p);
          } else {
            const ulonglong2 w = __ldg(tab + L.off_rad + ((j << s) * (R >> CL)));
            xr[i + m] = shoup_mul(ar + p - br, w.x, w.y, p);
            xi[i + m] = shoup_mul(ai + p - bi, w.x, w.y, p);
          }
        }
    }
#pragma unroll
    for (int pos = 0; pos < K; ++pos) {
      uint64_t ar = xr[pos], ai = xi[pos];
      if (pos) {
        const ulonglong2 w = __ldg(tab + L.off_split_fwd + pos * NC + Lw);
        ar = shoup_mul(ar, w.x, w.y, p);
        ai = shoup_mul(ai, w.x, w.y, p);
      }
      peer[pos][pad16(Lw)] = make_ulonglong2(ar, ai);
    }
  }
  cl.sync();  // every position transformed before the in-CTA passes read them
}

// Inverse: every CTA holds its chunk's sub-transform output in shared memory; CTA h
// combines the chunks at its positions (split twiddles, radix-2^CL DIT, untwist, as
// k_dgt_split) and writes the results to global memory at xg[Lw + hh 2^LOGNC].  The
// closing barrier keeps every CTA's shared memory alive until its peers have read it.
template <int LOGNC, int LOGR, int CL>
__device__ __forceinline__ void cluster_split_inv(ulonglong2* sdat, int h, const ulonglong2* tab,
                                                  const DgtTableLayout& L, uint64_t p, ulonglong2* xg) {
  namespace cg = cooperative_groups;
  constexpr int K = 1 << CL, NC = 1 << LOGNC, T = NC >> LOGR, SPAN = NC / K, R = 1 << LOGR;
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();  // every chunk's sub-transform in place
  const ulonglong2* peer[K];
#pragma unroll
  for (int q = 0; q < K; ++q) peer[q] = cl.map_shared_rank(sdat, q);
  for (int t = threadIdx.x; t < SPAN; t += T) {
    const int Lw = h * SPAN + t;
    uint64_t xr[K], xi[K];
#pragma unroll
    for (int pos = 0; pos < K; ++pos) {
      const ulonglong2 a = peer[pos][pad16(Lw)];
      uint64_t ar = a.x, ai = a.y;
      if (pos) {
        const ulonglong2 w = __ldg(tab + L.off_split_inv + pos * NC + Lw);
        ar = shoup_mul(ar, w.x, w.y, p);
        ai = shoup_mul(ai, w.x, w.y, p);
      }
      xr[pos] = ar;
      xi[pos] = ai;
    }
#pragma unroll
    for (int s = CL - 1; s >= 0; --s) {
      const int m = K >> (s + 1);
#pragma unroll
      for (int i = 0; i < K; ++i)
        if ((i & m) == 0) {
          const int j = i & (m - 1);
          const uint64_t ar = xr[i], ai = xi[i];
          uint64_t br = xr[i + m], bi = xi[i + m];
          if (j != 0) {
            const ulonglong2 w = __ldg(tab + L.off_rad + R - ((j << s) * (R >> CL)));
            br = shoup_mul(br, w.x, w.y, p);
            bi = shoup_mul(bi, w.x, w.y, p);
          }
          xr[i] = add_mod(ar, br, p);
          xi[i] = add_mod(ai, bi, p);
          xr[i + m] = sub_mod(ar, br, p);
          xi[i + m] = sub_mod(ai, bi, p);
        }
    }
#pragma unroll
    for (int hh = 0; hh < K; ++hh) {
      const int n = Lw + hh * NC;
      uint64_t ar = xr[hh], ai = xi[hh];
      gi_mul_const3(ar, ai, tab + L.off_untwist + 3 * n, p);
      xg[n] = make_ulonglong2(ar, ai);
    }
  }
  cl.sync();
}

// Shared-memory bytes of one CTA.
template <int LOGNC, int LOGR>
constexpr int dgt_smem_bytes() {
  return ((1 << LOGNC) + ((1 << LOGNC) >> 4) + (1 << LOGR) + PassCfg<LOGNC, LOGR>::stotal()) * 16;
}

// Forward transform of 2^LOGNC elements per CTA, in place.
// blockIdx.x = (poly * nres + r) * 2^S + h; element block h of residue r.
// Occupancy hint: at most 128 registers per thread for the CTA sizes used.
// Register budget: 64 per thread for radix <= 8 (two 512-thread CTAs per SM),
// 128 for radix 16.
template <int LOGNC, int LOGR>
constexpr int dgt_min_blocks() {
  constexpr int T = (1 << LOGNC) >> LOGR;
  constexpr int regs = LOGR >= 4 ? 128 : 64;
  constexpr int b = 65536 / (T * regs);
  return b < 1 ? 1 : (b > 16 ? 16 : b);
}

// Whether a kernel carries the next-unit L2 prefetch: only the configurations with one
// resident CTA per SM, whose grids the host makes persistent.  Elsewhere the grid is the
// unit count, the prefetch never fires, and its live values only cost registers (the
// radix-8, 4096-element forward kernel spilled 28 bytes per thread with it, 4 without).
template <int LOGNC, int LOGR, int CL>
constexpr bool dgt_prefetches() {
  return CL == 0 && dgt_min_blocks<LOGNC, LOGR>() == 1;
}

// CL > 0: the split stage of 2^CL chunks runs inside the kernel's thread-block
// cluster (launched with cluster dimension 2^CL, one CTA per unit, S = CL); the
// input is read untwisted and the twist applied here (cluster_split_fwd).
template <int LOGNC, int LOGR, int CL = 0>
__global__ void __launch_bounds__((1 << LOGNC) >> LOGR, (dgt_min_blocks<LOGNC, LOGR>()))
    k_dgt_fwd(ulonglong2* __restrict__ data, const ulonglong2* __restrict__ src_base, DgtArgs A, int nres,
              int rid_off, long long poly_stride, int S, int twist, unsigned nunits) {
  constexpr int NC = 1 << LOGNC, R = 1 << LOGR, T = NC >> LOGR;
  using C = PassCfg<LOGNC, LOGR>;
  extern __shared__ ulonglong2 smem[];
  ulonglong2* sdat = smem;
  ulonglong2* srad = smem + NC + (NC >> 4);
  ulonglong2* stw = srad + R;
  const int tid = threadIdx.x;
  // Persistent CTAs: unit ub = (poly * nres + r) * 2^S + h, strided by the grid; each
  // iteration of a one-CTA-per-SM configuration prefetches the next unit's input into L2.
  const ulonglong2* in_base = src_base ? src_base : data;  // out of place when src_base is set
  auto unit_off = [&](unsigned ub) {
    const int pr_ = (int)(ub >> S);
    return (size_t)(pr_ / nres) * poly_stride + ((size_t)(pr_ % nres) << (LOGNC + S)) +
           ((size_t)(ub & ((1u << S) - 1)) << LOGNC);
  };
  for (unsigned ub = blockIdx.x; ub < nunits; ub += gridDim.x) {
  if (dgt_prefetches<LOGNC, LOGR, CL>() && tid == 0 && ub + gridDim.x < nunits)
    prefetch_l2(in_base + unit_off(ub + gridDim.x), NC * 16u);
  const int pr = (int)(ub >> S);
  const int r = pr % nres;
  const int rid = A.rid_list ? A.rid_list[pr] : rid_off + r;
  const uint64_t p = A.mc[rid].p;
  const ulonglong2* tab = A.tab + (size_t)rid * A.stride;
  const size_t off = unit_off(ub);
  ulonglong2* x = data + off;
  const ulonglong2* xs = in_base + off;
  for (int j = tid; j < R; j += T) srad[j] = tab[A.L.off_rad + j];
  stage_twiddles<LOGNC, LOGR>(stw, tab, A.L.off_fwd);
  __syncthreads();
  if constexpr (CL > 0) {  // chunk h of the twisted input, then the split stage across the cluster
    const int h = (int)(ub & ((1u << CL) - 1));
    for (int j = tid; j < NC; j += T) {
      const ulonglong2 a = xs[j];
      uint64_t ar = a.x, ai = a.y;
      gi_mul_const3(ar, ai, tab + A.L.off_twist + 3 * ((size_t)j + ((size_t)h << LOGNC)), p);
      sdat[pad16(j)] = make_ulonglong2(ar, ai);
    }
    cluster_split_fwd<LOGNC, LOGR, CL>(sdat, h, tab, A.L, p);
  }
  {
    constexpr int W = C::W0, PF = LOGNC - C::W0, G = 1 << (LOGR - C::W0);
    uint64_t xr[R], xi[R];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int Lw = tid + g * T;
#pragma unroll
      for (int v = 0; v < (1 << W); ++v) {
        const int idx = Lw + (v << PF);
        const ulonglong2 a = CL > 0 ? sdat[pad16(idx)] : xs[idx];
        uint64_t ar = a.x, ai = a.y;
        if (CL == 0 && twist) gi_mul_const3(ar, ai, tab + A.L.off_twist + 3 * idx, p);
        xr[g * (1 << W) + v] = ar;
        xi[g * (1 << W) + v] = ai;
      }
      dif_regs<W, LOGR, (PF > 0)>(xr + g * (1 << W), xi + g * (1 << W), srad, p);
      if constexpr (PF > 0) {
        const ulonglong2* tw = tab + A.L.off_fwd[0] + Lw;
#pragma unroll
        for (int v = 1; v < (1 << W); ++v) {
          const ulonglong2 w = __ldg(tw + (v << PF));
          xr[g * (1 << W) + v] = shoup_mul(xr[g * (1 << W) + v], w.x, w.y, p);
          xi[g * (1 << W) + v] = shoup_mul(xi[g * (1 << W) + v], w.x, w.y, p);
        }
      }
#pragma unroll
      for (int v = 0; v < (1 << W); ++v)
        sdat[pad16(Lw) + pad_off<PF>(v)] = make_ulonglong2(xr[g * (1 << W) + v], xi[g * (1 << W) + v]);
    }
    __syncthreads();
  }
  fwd_passes<LOGNC, LOGR, 1>(sdat, srad, stw, tab, A.L, p);
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int idx = tid + j * T;
    x[idx] = sdat[pad16(tid) + pad_off<LOGNC - LOGR>(j)];
  }
  __syncthreads();  // shared memory is rewritten by the next unit
  }
}

// src.p[i] by selects: indexing the by-value parameter with a run-time i would copy the
// whole argument to local memory in every thread.
__device__ __forceinline__ const ulonglong2* inv_src_ptr(const InvSrc& s, int i) {
  return i == 0 ? s.p[0] : i == 1 ? s.p[1] : i == 2 ? s.p[2] : s.p[3];
}

// Element `off` of tensor output j from the operands p = {a0, a1, b0, b1}: c0 = a0 b0,
// c1 = a0 b1 + a1 b0, c2 = a1 b1.  Only the operands output j uses are loaded.
__device__ __forceinline__ ulonglong2 tensor_load(const InvSrc& s, int j, size_t off, const ModConst& m) {
  uint64_t r, i;
  if (j == 0) {
    const ulonglong2 a0 = s.p[0][off], b0 = s.p[2][off];
    gi_mul(r, i, a0.x, a0.y, b0.x, b0.y, m);
  } else if (j == 2) {
    const ulonglong2 a1 = s.p[1][off], b1 = s.p[3][off];
    gi_mul(r, i, a1.x, a1.y, b1.x, b1.y, m);
  } else {
    const ulonglong2 a0 = s.p[0][off], a1 = s.p[1][off], b0 = s.p[2][off], b1 = s.p[3][off];
    uint64_t r1, i1, r2, i2;
    gi_mul(r1, i1, a0.x, a0.y, b1.x, b1.y, m);
    gi_mul(r2, i2, a1.x, a1.y, b0.x, b0.y, m);
    r = add_mod(r1, r2, m.p);
    i = add_mod(i1, i2, m.p);
  }
  return make_ulonglong2(r, i);
}

// Inverse transform of 2^LOGNC elements per CTA; untwist (with N^-1) applied
// when `untwist` is set (S == 0).  Input per InvSrc, output to `data`.
// In tensor mode (src.mode 1) the CTAs of c0, c1, c2 of one (pair, residue)
// are adjacent, so each operand residue is fetched from HBM once and served
// from L2 to the other outputs.
// CL > 0: as k_dgt_fwd, the split stage (twiddles, radix-2^CL DIT, untwist) runs
// inside the cluster after the in-CTA passes (cluster_split_inv).
template <int LOGNC, int LOGR, int CL = 0>
__global__ void __launch_bounds__((1 << LOGNC) >> LOGR, (dgt_min_blocks<LOGNC, LOGR>()))
    k_dgt_inv(ulonglong2* __restrict__ data, InvSrc src, DgtArgs A, int nres, int rid_off, long long poly_stride,
              int S, int untwist, unsigned nunits) {
  constexpr int NC = 1 << LOGNC, R = 1 << LOGR, T = NC >> LOGR;
  using C = PassCfg<LOGNC, LOGR>;
  extern __shared__ ulonglong2 smem[];
  ulonglong2* sdat = smem;
  ulonglong2* srad = smem + NC + (NC >> 4);
  ulonglong2* stw = srad + R;
  const int tid = threadIdx.x;
  // Persistent CTAs over units ub = (poly-or-output * nres + r) * 2^S + h (see k_dgt_fwd).
  auto coords = [&](unsigned ub, int& r_, int& poly_) {
    const int pr_ = (int)(ub >> S);
    if (src.mode == 1) {  // c0, c1, c2 of one (pair, residue) in adjacent units
      const int rest = pr_ / 3;
      r_ = rest % nres;
      poly_ = (pr_ % 3) * src.npairs + rest / nres;
    } else {
      r_ = pr_ % nres;
      poly_ = pr_ / nres;
    }
  };
  for (unsigned ub = blockIdx.x; ub < nunits; ub += gridDim.x) {
  if (dgt_prefetches<LOGNC, LOGR, CL>() && tid == 0 && ub + gridDim.x < nunits) {  // the next unit's operands into L2
    int rn, pn;
    coords(ub + gridDim.x, rn, pn);
    const size_t inner_n = ((size_t)rn << (LOGNC + S)) + ((size_t)((ub + gridDim.x) & ((1u << S) - 1)) << LOGNC);
    if (src.mode == 0 || src.mode == 3) {
      prefetch_l2(src.p[0] + pn * poly_stride + inner_n, NC * 16u);
      if (src.mode == 3) prefetch_l2(src.p[1] + pn * poly_stride + inner_n, NC * 16u);
    } else if (src.mode == 2) {
      prefetch_l2(inv_src_ptr(src, pn / src.npairs) + (pn % src.npairs) * poly_stride + inner_n, NC * 16u);
    } else {
      const int jt = pn / src.npairs;
      const size_t bo = (size_t)(pn % src.npairs) * poly_stride + inner_n;
      if (jt != 2) prefetch_l2(src.p[0] + bo, NC * 16u);  // a0: c0, c1
      if (jt != 0) prefetch_l2(src.p[1] + bo, NC * 16u);  // a1: c1, c2
      if (jt != 2) prefetch_l2(src.p[2] + bo, NC * 16u);  // b0: c0, c1
      if (jt != 0) prefetch_l2(src.p[3] + bo, NC * 16u);  // b1: c1, c2
    }
  }
  const int h = (int)(ub & ((1u << S) - 1));
  const int pr = (int)(ub >> S);
  int r, poly;
  coords(ub, r, poly);
  const int rid = A.rid_list ? A.rid_list[pr] : rid_off + r;
  const uint64_t p = A.mc[rid].p;
  const ulonglong2* tab = A.tab + (size_t)rid * A.stride;
  const size_t inner = ((size_t)r << (LOGNC + S)) + ((size_t)h << LOGNC);
  ulonglong2* x = data + poly * poly_stride + inner;
  for (int j = tid; j < R; j += T) srad[j] = tab[A.L.off_rad + j];
  stage_twiddles<LOGNC, LOGR>(stw, tab, A.L.off_inv);
  if (src.mode == 3) {
    const size_t base = poly * poly_stride + inner;
    const ModConst m = A.mc[rid];
#pragma unroll 4
    for (int j = 0; j < R; ++j) {
      const int idx = tid + j * T;
      const ulonglong2 a = src.p[0][base + idx], b = src.p[1][base + idx];
      uint64_t cr, ci;
      gi_mul(cr, ci, a.x, a.y, b.x, b.y, m);
      sdat[pad16(tid) + pad_off<LOGNC - LOGR>(j)] = make_ulonglong2(cr, ci);
    }
  } else if (src.mode != 1) {
    const ulonglong2* xs = src.mode == 0
                               ? src.p[0] + poly * poly_stride + inner
                               : inv_src_ptr(src, poly / src.npairs) + (poly % src.npairs) * poly_stride + inner;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int idx = tid + j * T;
      sdat[pad16(tid) + pad_off<LOGNC - LOGR>(j)] = xs[idx];
    }
  } else {
    const int jt = poly / src.npairs;  // which tensor output
    const size_t base = (size_t)(poly % src.npairs) * poly_stride + inner;
    const ModConst m = A.mc[rid];
    auto load_all = [&](auto out) {  // the output index as a constant: one loop per output
#pragma unroll 4
      for (int j = 0; j < R; ++j) {
        const int idx = tid + j * T;
        sdat[pad16(tid) + pad_off<LOGNC - LOGR>(j)] = tensor_load(src, decltype(out)::value, base + idx, m);
      }
    };
    if (jt == 0)
      load_all(std::integral_constant<int, 0>{});
    else if (jt == 2)
      load_all(std::integral_constant<int, 2>{});
    else
      load_all(std::integral_constant<int, 1>{});
  }
  __syncthreads();
  inv_passes<LOGNC, LOGR, C::NP - 1>(sdat, srad, stw, tab, A.L, p);
  {
    constexpr int W = C::W0, PF = LOGNC - C::W0, G = 1 << (LOGR - C::W0);
    uint64_t xr[1 << W], xi[1 << W];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int Lw = tid + g * T;
#pragma unroll
      for (int v = 0; v < (1 << W); ++v) {
        const ulonglong2 a = sdat[pad16(Lw) + pad_off<PF>(v)];
        xr[v] = a.x;
        xi[v] = a.y;
      }
      if constexpr (PF > 0) {
        const ulonglong2* tw = tab + A.L.off_inv[0] + Lw;
#pragma unroll
        for (int v = 1; v < (1 << W); ++v) {
          const ulonglong2 w = __ldg(tw + (v << PF));
          xr[v] = shoup_mul(xr[v], w.x, w.y, p);
          xi[v] = shoup_mul(xi[v], w.x, w.y, p);
        }
      }
      if constexpr (C::NP > 1) {  // written by the lazy pass 1
        xr[0] = red2p(xr[0], p);
        xi[0] = red2p(xi[0], p);
      }
      dit_regs<W, LOGR>(xr, xi, srad, p);
#pragma unroll
      for (int v = 0; v < (1 << W); ++v) {
        const int idx = Lw + (v << PF);
        uint64_t ar = xr[v], ai = xi[v];
        if constexpr (CL > 0) {
          sdat[pad16(idx)] = make_ulonglong2(ar, ai);  // each thread rewrites the slots it read
        } else {
          if (untwist) gi_mul_const3(ar, ai, tab + A.L.off_untwist + 3 * idx, p);
          x[idx] = make_ulonglong2(ar, ai);
        }
      }
    }
  }
  if constexpr (CL > 0)
    cluster_split_inv<LOGNC, LOGR, CL>(sdat, h, tab, A.L, p, data + poly * poly_stride + ((size_t)r << (LOGNC + CL)));
  __syncthreads();  // shared memory is rewritten by the next unit
  }
}

// Element-wise top stage for N = 2^S * Nc (forward: twist + radix-2^S DIF
// over the top S bits + twiddle; inverse: twiddle + radix-2^S DIT + untwist).
template <int S, bool INV>
__global__ void __launch_bounds__(256)
    k_dgt_split(ulonglong2* __restrict__ data, const ulonglong2* __restrict__ src_base, DgtArgs A, int nres,
                int rid_off, long long poly_stride, int logNc, int logR) {
  const int Nc = 1 << logNc;
  const int chunks = Nc / 256;
  const int pr = blockIdx.x / chunks;
  const int Lw = (blockIdx.x % chunks) * 256 + threadIdx.x;
  const int r = pr % nres;
  const int poly = pr / nres;
  const int rid = A.rid_list ? A.rid_list[pr] : rid_off + r;
  const uint64_t p = A.mc[rid].p;
  const ulonglong2* tab = A.tab + (size_t)rid * A.stride;
  ulonglong2* x = data + poly * poly_stride + ((size_t)r << (logNc + S));
  const ulonglong2* xs = (src_base ? src_base : data) + poly * poly_stride + ((size_t)r << (logNc + S));
  constexpr int K = 1 << S;
  uint64_t xr[K], xi[K];
  const int R = 1 << logR;
  if (!INV) {
#pragma unroll
    for (int hh = 0; hh < K; ++hh) {
      const int n = Lw + hh * Nc;
      const ulonglong2 a = xs[n];
      uint64_t ar = a.x, ai = a.y;
      gi_mul_const3(ar, ai, tab + A.L.off_twist + 3 * n, p);
      xr[hh] = ar;
      xi[hh] = ai;
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int m = K >> (s + 1);
#pragma unroll
      for (int i = 0; i < K; ++i)
        if ((i & m) == 0) {
          const int j = i & (m - 1);
          const uint64_t ar = xr[i], ai = xi[i], br = xr[i + m], bi = xi[i + m];
          xr[i] = add_mod(ar, br, p);
          xi[i] = add_mod(ai, bi, p);
          if (j == 0) {
            xr[i + m] = sub_mod(ar, br, p);
            xi[i + m] = sub_mod(ai, bi, p);
          } else {
            const ulonglong2 w = __ldg(tab + A.L.off_rad + ((j << s) * (R >> S)));
            xr[i + m] = shoup_mul(ar + p - br, w.x, w.y, p);
            xi[i + m] = shoup_mul(ai + p - bi, w.x, w.y, p);
          }
        }
    }
#pragma unroll
    for (int pos = 0; pos < K; ++pos) {
      uint64_t ar = xr[pos], ai = xi[pos];
      if (pos) {
        const ulonglong2 w = __ldg(tab + A.L.off_split_fwd + pos * Nc + Lw);
        ar = shoup_mul(ar, w.x, w.y, p);
        ai = shoup_mul(ai, w.x, w.y, p);
      }
      x[Lw + pos * Nc] = make_ulonglong2(ar, ai);
    }
  } else {
#pragma unroll
    for (int pos = 0; pos < K; ++pos) {
      const ulonglong2 a = x[Lw + pos * Nc];
      uint64_t ar = a.x, ai = a.y;
      if (pos) {
        const ulonglong2 w = __ldg(tab + A.L.off_split_inv + pos * Nc + Lw);
        ar = shoup_mul(ar, w.x, w.y, p);
        ai = shoup_mul(ai, w.x, w.y, p);
      }
      xr[pos] = ar;
      xi[pos] = ai;
    }
#pragma unroll
    for (int s = S - 1; s >= 0; --s) {
      const int m = K >> (s + 1);
#pragma unroll
      for (int i = 0; i < K; ++i)
        if ((i & m) == 0) {
          const int j = i & (m - 1);
          const uint64_t ar = xr[i], ai = xi[i];
          uint64_t br = xr[i + m], bi = xi[i + m];
          if (j != 0) {
            const ulonglong2 w = __ldg(tab + A.L.off_rad + R - ((j << s) * (R >> S)));
            br = shoup_mul(br, w.x, w.y, p);
            bi = shoup_mul(bi, w.x, w.y, p);
          }
          xr[i] = add_mod(ar, br, p);
          xi[i] = add_mod(ai, bi, p);
          xr[i + m] = sub_mod(ar, br, p);
          xi[i + m] = sub_mod(ai, bi, p);
        }
    }
#pragma unroll
    for (int hh = 0; hh < K; ++hh) {
      const int n = Lw + hh * Nc;
      uint64_t ar = xr[hh], ai = xi[hh];
      gi_mul_const3(ar, ai, tab + A.L.off_untwist + 3 * n, p);
      x[n] = make_ulonglong2(ar, ai);
    }
  }
}

}  // namespace cpoly
