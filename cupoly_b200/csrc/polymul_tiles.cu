// Mixed-size negacyclic products in ONE persistent launch.
//
// A batch holds independent products c = a b mod (x^nphi + 1, q) of residues
// of different ring sizes N = nphi / 2 in {1024, 2048, 4096, 8192} (cuPoly
// computes one parameter set per process: poly_mul after two forward DGTs and
// before one inverse, src/arithmetic/polynomial.cu:892-914 with
// src/cuda/dgt.cu:107-205).  Here one grid of one CTA per SM walks a device
// work list of tiles.  A tile is 8192 Gaussian elements' worth of residues of
// one size: 8192 / N residues side by side, each transformed by N / 8 of the
// CTA's 1024 threads with radix-8 register passes in shared memory.  Per tile:
//   1. every residue of a: twist, forward passes; the last pass's registers go
//      to this CTA's slot of the workspace (stays in L2);
//   2. every residue of b: twist, forward passes; in the last pass each
//      thread multiplies its 8 elements by the matching elements of a's
//      transform (the same positions it wrote in step 1), then runs the
//      inverse's first radix-8 pass on them in registers;
//   3. the remaining inverse passes in shared memory, untwist with N^-1, c to
//      HBM.
// So a, b and c cross HBM once each and the two transforms' intermediate
// results never leave the SM / L2.  The arithmetic and the DGT-domain order
// are those of k_dgt_fwd / k_dgt_inv (dgt_kernels.cuh) with the same tables;
// the engines of the batch must use the whole-CTA radix-8 plan (no split).
#include "../../include/cupoly_b200.h"
#include "dgt_kernels.cuh"
#include "launch.cuh"

namespace cpoly {

namespace {

constexpr int kTileElems = 8192;   // Gaussian elements per tile
constexpr int kTileThreads = 1024; // kTileElems / 8
constexpr int kTileLogR = 3;

struct TileGroup {
  const ulonglong2* a;  // rows [rows][N]
  const ulonglong2* b;
  ulonglong2* c;
  const int* rid;       // engine prime of each row
  int rows;
  DgtArgs A;            // the engine's tables
};

struct TileArgs {
  TileGroup g[4];  // index log2(N) - 10
  int* err;        // set when a tile of the list is out of range (it is skipped)
};

struct Tile {
  int lg;     // log2(N) - 10
  int row0;   // first row of the tile in its group
  int count;  // rows in the tile, 1 .. 8192 / N
};

// Barrier of the T threads that transform one residue of a tile (named barrier `id`,
// 1 + the residue's index in the tile).  The residues of a tile are independent, so
// their thread groups run their passes out of step with each other, as separate
// CTAs would; only the end of a tile synchronises the whole CTA.
__device__ __forceinline__ void group_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Threads per named-barrier group of the transition of field f (at least 128, so that a
// tile's groups fit the 15 ids).
constexpr int tile_group(int f) { return (1 << f) > 128 ? (1 << f) : 128; }

// First id of the transition of field f in a tile of residues of 2^LOGN elements: after
// the residues' own ids 1 .. 8192 / N and the ids of every larger field f + 3, f + 6, ...
template <int LOGN>
constexpr int tile_bar_base(int f) {
  constexpr int T = (1 << LOGN) >> kTileLogR;
  int b = 1 + kTileThreads / T;
  for (int g = f + kTileLogR; (1 << g) < T; g += kTileLogR)
    if ((1 << g) > 32 && tile_group(g) < T) b += kTileThreads / tile_group(g);
  return b;
}

// Barrier between two passes of one residue whose exchange spans the 2^F threads that
// share c >> F (F the larger of the two passes' bit fields): a warp barrier when those fit
// in a warp, the residue's barrier when a group spans the residue, else a named barrier
// per group.  Each transition has its own ids, so a thread released early never meets a
// group of another transition at the same id.
template <int LOGN, int F>
__device__ __forceinline__ void tile_pass_sync(int gb) {
  constexpr int T = (1 << LOGN) >> kTileLogR, G = tile_group(F);
  if constexpr ((1 << F) <= 32) {
    __syncwarp();
  } else if constexpr (G >= T) {
    group_sync(gb, T);
  } else {
    constexpr int B = tile_bar_base<LOGN>(F);
    static_assert(B + kTileThreads / G - 1 <= 15, "named barrier ids 1..15");
    group_sync(B + (int)threadIdx.x / G, G);
  }
}

// Forward passes I .. NP - 2 of one residue in shared memory (no staged tables:
// the pass twiddles are read through the read-only cache); thread c of the
// residue's T threads.
// The phases are separate (not inlined) functions: inlined into one body, the
// compiler keeps addresses of every pass live across all of them and spills.
template <int LOGN, int I>
__device__ __noinline__ void tile_fwd_mid(ulonglong2* sdat, const ulonglong2* srad, const ulonglong2* tab,
                                             const DgtTableLayout& L, uint64_t p, int c, int gb) {
  using C = PassCfg<LOGN, kTileLogR>;
  if constexpr (I < C::NP - 1) {
    constexpr int PF = C::field(I), R = 1 << kTileLogR;
    const int Lw = c & ((1 << PF) - 1);
    const int base = ((c >> PF) << (PF + kTileLogR)) + Lw;
    const int pb = pad16(base);
    uint64_t xr[R], xi[R];
#pragma unroll
    for (int v = 0; v < R; ++v) {
      const ulonglong2 x = sdat[pb + pad_off<PF>(v)];
      xr[v] = x.x;
      xi[v] = x.y;
    }
    dif_regs<kTileLogR, kTileLogR, true>(xr, xi, srad, p);
    const ulonglong2* tw = tab + L.off_fwd[I] + Lw;
#pragma unroll
    for (int v = 1; v < R; ++v) {
      const ulonglong2 w = __ldg(tw + (v << PF));
      xr[v] = shoup_mul(xr[v], w.x, w.y, p);
      xi[v] = shoup_mul(xi[v], w.x, w.y, p);
    }
#pragma unroll
    for (int v = 0; v < R; ++v) sdat[pb + pad_off<PF>(v)] = make_ulonglong2(xr[v], xi[v]);
    tile_pass_sync<LOGN, PF>(gb);  // the next pass reads what the threads sharing c >> PF wrote
    tile_fwd_mid<LOGN, I + 1>(sdat, srad, tab, L, p, c, gb);
  }
}

// Inverse passes I .. 1 in shared memory.
template <int LOGN, int I>
__device__ __noinline__ void tile_inv_mid(ulonglong2* sdat, const ulonglong2* srad, const ulonglong2* tab,
                                             const DgtTableLayout& L, uint64_t p, int c, int gb) {
  using C = PassCfg<LOGN, kTileLogR>;
  if constexpr (I >= 1) {
    constexpr int PF = C::field(I), R = 1 << kTileLogR;
    const int Lw = c & ((1 << PF) - 1);
    const int base = ((c >> PF) << (PF + kTileLogR)) + Lw;
    uint64_t xr[R], xi[R];
#pragma unroll
    for (int v = 0; v < R; ++v) {
      const ulonglong2 x = sdat[pad16(base + (v << PF))];
      xr[v] = x.x;
      xi[v] = x.y;
    }
    if constexpr (PF > 0) {
      const ulonglong2* tw = tab + L.off_inv[I] + Lw;
#pragma unroll
      for (int v = 1; v < R; ++v) {
        const ulonglong2 w = __ldg(tw + (v << PF));
        xr[v] = shoup_mul(xr[v], w.x, w.y, p);
        xi[v] = shoup_mul(xi[v], w.x, w.y, p);
      }
    }
    xr[0] = red2p(xr[0], p);  // written by a lazy pass
    xi[0] = red2p(xi[0], p);
    dit_regs<kTileLogR, kTileLogR, true>(xr, xi, srad, p);
#pragma unroll
    for (int v = 0; v < R; ++v) sdat[pad16(base + (v << PF))] = make_ulonglong2(xr[v], xi[v]);
    tile_pass_sync<LOGN, C::field(I - 1)>(gb);  // the next pass reads across c >> field(I - 1)
    tile_inv_mid<LOGN, I - 1>(sdat, srad, tab, L, p, c, gb);
  }
}

// First forward pass of one residue: the input from HBM, twisted, into shared memory.
template <int LOGN>
__device__ __noinline__ void tile_fwd_first(ulonglong2* sdat, const ulonglong2* xs, const ulonglong2* srad,
                                               const ulonglong2* tab, const DgtTableLayout& L, uint64_t p, int c,
                                               bool live, int gb) {
  using C = PassCfg<LOGN, kTileLogR>;
  constexpr int T = (1 << LOGN) >> kTileLogR, W = C::W0, PF = LOGN - C::W0, G = 1 << (kTileLogR - C::W0);
  uint64_t xr[1 << W], xi[1 << W];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    const int Lw = c + g * T;
#pragma unroll
    for (int v = 0; v < (1 << W); ++v) {
      const int idx = Lw + (v << PF);
      uint64_t ar = 0, ai = 0;
      if (live) {
        const ulonglong2 x = xs[idx];
        ar = x.x;
        ai = x.y;
        gi_mul_const3(ar, ai, tab + L.off_twist + 3 * idx, p);
      }
      xr[v] = ar;
      xi[v] = ai;
    }
    static_assert(PF > 0, "the first pass is followed by its twiddles");
    dif_regs<W, kTileLogR, true>(xr, xi, srad, p);
    const ulonglong2* tw = tab + L.off_fwd[0] + Lw;
#pragma unroll
    for (int v = 1; v < (1 << W); ++v) {
      const ulonglong2 w = __ldg(tw + (v << PF));
      xr[v] = shoup_mul(xr[v], w.x, w.y, p);
      xi[v] = shoup_mul(xi[v], w.x, w.y, p);
    }
#pragma unroll
    for (int v = 0; v < (1 << W); ++v) sdat[pad16(Lw) + pad_off<PF>(v)] = make_ulonglong2(xr[v], xi[v]);
  }
  group_sync(gb, T);
}

// Last forward pass of a (lowest index bits, positions c R + v): to the slot.
template <int LOGN>
__device__ __noinline__ void tile_last_a(const ulonglong2* sdat, const ulonglong2* srad, uint64_t p, int c,
                                         ulonglong2* my) {
  constexpr int R = 1 << kTileLogR, T = (1 << LOGN) >> kTileLogR;
  uint64_t xr[R], xi[R];
#pragma unroll
  for (int v = 0; v < R; ++v) {
    const ulonglong2 x = sdat[pad16(c * R) + v];
    xr[v] = x.x;
    xi[v] = x.y;
  }
  dif_regs<kTileLogR, kTileLogR>(xr, xi, srad, p);
#pragma unroll
  for (int v = 0; v < R; ++v) my[v * T] = make_ulonglong2(xr[v], xi[v]);
}

// Last forward pass of b, the Gaussian product with a's transform from the slot,
// and the inverse's first pass (same positions, no twiddles), back to shared memory.
template <int LOGN>
__device__ __noinline__ void tile_last_b(ulonglong2* sdat, const ulonglong2* srad, const ModConst* mc, int c,
                                         const ulonglong2* my) {
  constexpr int R = 1 << kTileLogR, T = (1 << LOGN) >> kTileLogR;
  const ModConst m = *mc;
  uint64_t xr[R], xi[R];
#pragma unroll
  for (int v = 0; v < R; ++v) {
    const ulonglong2 x = sdat[pad16(c * R) + v];
    xr[v] = x.x;
    xi[v] = x.y;
  }
  dif_regs<kTileLogR, kTileLogR>(xr, xi, srad, m.p);
#pragma unroll
  for (int v = 0; v < R; ++v) {
    const ulonglong2 a = my[v * T];
    uint64_t cr, ci;
    gi_mul(cr, ci, a.x, a.y, xr[v], xi[v], m);
    xr[v] = cr;
    xi[v] = ci;
  }
  dit_regs<kTileLogR, kTileLogR, true>(xr, xi, srad, m.p);  // the next inverse pass reduces
  // each thread rewrites only the positions it read
#pragma unroll
  for (int v = 0; v < R; ++v) sdat[pad16(c * R) + v] = make_ulonglong2(xr[v], xi[v]);
}

// Inverse pass 0 (the top W0 bits), untwist with N^-1, c to HBM.
template <int LOGN>
__device__ __noinline__ void tile_inv_last(const ulonglong2* sdat, const ulonglong2* srad, const ulonglong2* tab,
                                           const DgtTableLayout& L, uint64_t p, int c, bool live,
                                           ulonglong2* xc) {
  using C = PassCfg<LOGN, kTileLogR>;
  constexpr int T = (1 << LOGN) >> kTileLogR, W = C::W0, PF = LOGN - C::W0, Gn = 1 << (kTileLogR - C::W0);
  uint64_t xr[1 << W], xi[1 << W];
#pragma unroll
  for (int g = 0; g < Gn; ++g) {
    const int Lw = c + g * T;
#pragma unroll
    for (int v = 0; v < (1 << W); ++v) {
      const ulonglong2 x = sdat[pad16(Lw) + pad_off<PF>(v)];
      xr[v] = x.x;
      xi[v] = x.y;
    }
    const ulonglong2* tw = tab + L.off_inv[0] + Lw;
#pragma unroll
    for (int v = 1; v < (1 << W); ++v) {
      const ulonglong2 w = __ldg(tw + (v << PF));
      xr[v] = shoup_mul(xr[v], w.x, w.y, p);
      xi[v] = shoup_mul(xi[v], w.x, w.y, p);
    }
    xr[0] = red2p(xr[0], p);  // written by a lazy pass
    xi[0] = red2p(xi[0], p);
    dit_regs<W, kTileLogR>(xr, xi, srad, p);
    if (live) {
#pragma unroll
      for (int v = 0; v < (1 << W); ++v) {
        const int idx = Lw + (v << PF);
        uint64_t ar = xr[v], ai = xi[v];
        gi_mul_const3(ar, ai, tab + L.off_untwist + 3 * idx, p);
        xc[idx] = make_ulonglong2(ar, ai);
      }
    }
  }
}

template <int LOGN>
__device__ __forceinline__ void tile_polymul(const TileGroup& G, int row0, int count, ulonglong2* smem,
                                             ulonglong2* slot) {
  constexpr int N = 1 << LOGN, R = 1 << kTileLogR, T = N >> kTileLogR;
  using C = PassCfg<LOGN, kTileLogR>;
  static_assert(C::field(C::NP - 1) == 0, "the last pass covers the lowest index bits");
  static_assert(C::NP >= 3, "at least one middle pass");
  const int u = threadIdx.x / T, c = threadIdx.x % T;
  const bool live = u < count;
  const int gb = 1 + u;  // this residue's named barrier
  if (!live) {  // a residue slot the tile does not fill: nothing to wait for but the tile's end
    __syncthreads();
    return;
  }
  const int row = row0 + u;
  const int rid = G.rid[row];
  const uint64_t p = G.A.mc[rid].p;
  const ulonglong2* tab = G.A.tab + (size_t)rid * G.A.stride;
  const DgtTableLayout& L = G.A.L;
  ulonglong2* sdat = smem + u * (N + (N >> 4));
  ulonglong2* srad = smem + kTileElems + (kTileElems >> 4) + u * R;
  if (c < R) srad[c] = tab[L.off_rad + c];
  group_sync(gb, T);
  const size_t off = (size_t)row * N;
  // element v of thread c (position c R + v of the last pass) at my[v T]
  ulonglong2* my = slot + (size_t)u * N + c;

  // 1. a: forward transform; its last pass's registers to the slot
  tile_fwd_first<LOGN>(sdat, G.a + off, srad, tab, L, p, c, true, gb);
  tile_fwd_mid<LOGN, 1>(sdat, srad, tab, L, p, c, gb);
  tile_last_a<LOGN>(sdat, srad, p, c, my);
  group_sync(gb, T);  // the residue's shared memory is reused for b
  // 2. b: forward transform, product, the inverse's first pass
  tile_fwd_first<LOGN>(sdat, G.b + off, srad, tab, L, p, c, true, gb);
  tile_fwd_mid<LOGN, 1>(sdat, srad, tab, L, p, c, gb);
  tile_last_b<LOGN>(sdat, srad, G.A.mc + rid, c, my);
  __syncwarp();  // the next inverse pass (field 3) reads what the 8 threads sharing c >> 3 wrote
  // 3. the remaining inverse passes, untwist, c to HBM
  tile_inv_mid<LOGN, C::NP - 2>(sdat, srad, tab, L, p, c, gb);
  tile_inv_last<LOGN>(sdat, srad, tab, L, p, c, true, G.c + off);
  __syncthreads();  // shared memory is rewritten by the next tile
}

__global__ void __launch_bounds__(kTileThreads, 1)
    k_polymul_tiles(const __grid_constant__ TileArgs args, const Tile* __restrict__ tiles, int ntiles,
                    ulonglong2* __restrict__ ws) {
  extern __shared__ ulonglong2 smem[];
  ulonglong2* slot = ws + (size_t)blockIdx.x * kTileElems;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    // a tile naming an absent group, rows outside it, or more rows than fit is skipped
    const bool ok = tl.lg >= 0 && tl.lg < 4 && args.g[tl.lg].rid != nullptr && tl.count >= 1 &&
                    tl.count <= (8 >> tl.lg) && tl.row0 >= 0 && tl.row0 + tl.count <= args.g[tl.lg].rows;
    if (!ok) {
      if (threadIdx.x == 0) atomicExch(args.err, 1);
      continue;
    }
    switch (tl.lg) {
      case 0: tile_polymul<10>(args.g[0], tl.row0, tl.count, smem, slot); break;
      case 1: tile_polymul<11>(args.g[1], tl.row0, tl.count, smem, slot); break;
      case 2: tile_polymul<12>(args.g[2], tl.row0, tl.count, smem, slot); break;
      default: tile_polymul<13>(args.g[3], tl.row0, tl.count, smem, slot); break;
    }
  }
}

constexpr int tile_smem_bytes() { return (kTileElems + (kTileElems >> 4) + 8 * 8) * 16; }

}  // namespace

}  // namespace cpoly

using namespace cpoly;

extern "C" size_t cp_polymul_tiles_workspace_bytes(void) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                cudaSuccess)
    return 0;
  return (size_t)sms * kTileElems * 16;
}

extern "C" int cp_polymul_tiles(const cp_engine* const* engines, void* const* c, const void* const* a,
                                const void* const* b, const int* const* rid, const int* rows, const void* tiles,
                                int ntiles, void* workspace, size_t workspace_bytes, void* stream) {
  if (!engines || !c || !a || !b || !rid || !rows || (ntiles > 0 && (!tiles || !workspace))) {
    set_error("cp_polymul_tiles: NULL argument");
    return CP_ERR_INVALID;
  }
  TileArgs args{};
  for (int lg = 0; lg < 4; ++lg) {
    const cp_engine* h = engines[lg];
    TileGroup& g = args.g[lg];
    if (!h) continue;
    const Engine& e = h->e;
    if (e.logN != 10 + lg || e.plan.logR != kTileLogR || e.plan.logNc != e.logN || e.plan.S != 0) {
      set_error("cp_polymul_tiles: engine " + std::to_string(lg) +
                " must have N = 2^" + std::to_string(10 + lg) + " and the whole-CTA radix-8 plan "
                "(cp_engine_set_plan(e, 3, log2 N))");
      return CP_ERR_INVALID;
    }
    if (rows[lg] > 0 && (!a[lg] || !b[lg] || !c[lg] || !rid[lg])) {
      set_error("cp_polymul_tiles: NULL buffer of a size group with rows");
      return CP_ERR_INVALID;
    }
    g.a = reinterpret_cast<const ulonglong2*>(a[lg]);
    g.b = reinterpret_cast<const ulonglong2*>(b[lg]);
    g.c = reinterpret_cast<ulonglong2*>(c[lg]);
    g.rid = rows[lg] > 0 ? rid[lg] : nullptr;
    g.rows = rows[lg];
    g.A = DgtArgs{e.d_tab, e.layout.stride, e.layout, e.d_mc, nullptr};
    if (!args.err) args.err = e.d_err;
  }
  if (ntiles > 0 && !args.err) {
    set_error("cp_polymul_tiles: no engine given");
    return CP_ERR_INVALID;
  }
  if (ntiles <= 0) return CP_OK;
  int dev = 0, sms = 0;
  if (cudaError_t err = cudaGetDevice(&dev)) return cuda_fail("cp_polymul_tiles: cudaGetDevice", err);
  if (cudaError_t err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
    return cuda_fail("cp_polymul_tiles: cudaDeviceGetAttribute", err);
  const int grid = ntiles < sms ? ntiles : sms;
  if (workspace_bytes < (size_t)grid * kTileElems * 16) {
    set_error("cp_polymul_tiles: workspace smaller than cp_polymul_tiles_workspace_bytes()");
    return CP_ERR_INVALID;
  }
  static bool attr_done[64] = {};
  if (dev < 64 && !attr_done[dev]) {
    if (cudaError_t err = cudaFuncSetAttribute(k_polymul_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               tile_smem_bytes()))
      return cuda_fail("cp_polymul_tiles: cudaFuncSetAttribute", err);
    attr_done[dev] = true;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  k_polymul_tiles<<<grid, kTileThreads, tile_smem_bytes(), st>>>(
      args, reinterpret_cast<const Tile*>(tiles), ntiles, reinterpret_cast<ulonglong2*>(workspace));
  return check_launch("cp_polymul_tiles");
}
