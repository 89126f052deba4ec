// Host launchers of the DGT kernels (replaces cuPoly's
// DGTEngine::execute_dgt and its runDGT dispatch, src/cuda/dgt.cu:107-205,
// 1069-1094).
#include "dgt_kernels.cuh"
#include "launch.cuh"

namespace cpoly {

namespace {

// Grid of a DGT launch.  When only one CTA fits per SM (N = 8192 in one CTA)
// the grid is persistent -- one CTA per SM striding over the units, each
// prefetching its next unit into L2 -- which measured 3-8 % faster on B200;
// with two or more resident CTAs per SM one CTA per unit is faster (the
// hardware balances the tail), so the grid is the unit count.
template <typename K>
unsigned persistent_grid(K kernel, int threads, int smem, std::atomic<int>& resident, long long units) {
  int per_device = resident.load();
  if (per_device == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    per_device = per_sm == 1 ? (sms > 0 ? sms : 1) : -1;
    resident.store(per_device);
  }
  if (per_device < 0) return (unsigned)units;
  return (unsigned)(units < per_device ? units : per_device);
}

template <int LOGNC, int LOGR>
int run_cta(const Engine& e, const DgtPlan& P, const DgtTableLayout& L, ulonglong2* data, const ulonglong2* fsrc,
            const InvSrc& isrc, int nres, int rid_off, int npolys, long long poly_stride, bool inverse, bool twist,
            cudaStream_t st, const int* rid_list) {
  constexpr int T = (1 << LOGNC) >> LOGR;
  constexpr int smem = dgt_smem_bytes<LOGNC, LOGR>();
  DgtArgs A{e.d_tab, L.stride, L, e.d_mc, rid_list};
  const int S = P.S;
  const long long blocks = (long long)npolys * nres << S;
  if (blocks <= 0) return 0;
  if (blocks > 0x7fffffffLL) {
    set_error("dgt: grid too large");
    return 1;
  }
  if (!inverse) {
    static std::atomic<unsigned long long> done{0};
    static std::atomic<int> resident{0};
    if (int rc = ensure_smem(k_dgt_fwd<LOGNC, LOGR>, smem, done)) return rc;
    const unsigned grid = persistent_grid(k_dgt_fwd<LOGNC, LOGR>, T, smem, resident, blocks);
    k_dgt_fwd<LOGNC, LOGR><<<grid, T, smem, st>>>(data, fsrc, A, nres, rid_off, poly_stride, S, twist ? 1 : 0,
                                                  (unsigned)blocks);
  } else {
    static std::atomic<unsigned long long> done{0};
    static std::atomic<int> resident{0};
    if (int rc = ensure_smem(k_dgt_inv<LOGNC, LOGR>, smem, done)) return rc;
    const unsigned grid = persistent_grid(k_dgt_inv<LOGNC, LOGR>, T, smem, resident, blocks);
    k_dgt_inv<LOGNC, LOGR><<<grid, T, smem, st>>>(data, isrc, A, nres, rid_off, poly_stride, S, twist ? 1 : 0,
                                                  (unsigned)blocks);
  }
  return check_launch("dgt");
}

using RunFn = int (*)(const Engine&, const DgtPlan&, const DgtTableLayout&, ulonglong2*, const ulonglong2*,
                      const InvSrc&, int, int, int, long long, bool, bool, cudaStream_t, const int*);

constexpr int kNoCluster = -1;  // the cluster form cannot be scheduled on this device: use the split kernel

// Transform with the split stage inside a thread-block cluster of 2^CL CTAs (one CTA
// per unit: the cluster's CTAs are the chunks of one residue).  Returns kNoCluster,
// having launched nothing, when the device cannot co-schedule such a cluster.
template <int LOGNC, int LOGR, int CL>
int run_cluster(const Engine& e, const DgtPlan&, const DgtTableLayout& L, ulonglong2* data, const ulonglong2* fsrc,
                const InvSrc& isrc, int nres, int rid_off, int npolys, long long poly_stride, bool inverse, bool,
                cudaStream_t st, const int* rid_list) {
  constexpr int T = (1 << LOGNC) >> LOGR;
  constexpr int smem = dgt_smem_bytes<LOGNC, LOGR>();
  DgtArgs A{e.d_tab, L.stride, L, e.d_mc, rid_list};
  const long long blocks = (long long)npolys * nres << CL;
  if (blocks <= 0) return 0;
  if (blocks > 0x7fffffffLL) {
    set_error("dgt: grid too large");
    return 1;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 1u << CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  static std::atomic<unsigned long long> done_f{0}, done_i{0};
  static std::atomic<int> ok_f{0}, ok_i{0};  // 0 unknown, 1 schedulable, -1 not
  auto schedulable = [&](auto kernel, std::atomic<int>& ok) {
    int v = ok.load();
    if (v == 0) {
      int n = 0;
      const cudaError_t err = cudaOccupancyMaxActiveClusters(&n, kernel, &cfg);
      v = (err == cudaSuccess && n > 0) ? 1 : -1;
      if (err != cudaSuccess) cudaGetLastError();  // clear the sticky-free error of the query
      ok.store(v);
    }
    return v > 0;
  };
  cudaError_t err;
  if (!inverse) {
    if (int rc = ensure_smem(k_dgt_fwd<LOGNC, LOGR, CL>, smem, done_f)) return rc;
    if (!schedulable(k_dgt_fwd<LOGNC, LOGR, CL>, ok_f)) return kNoCluster;
    err = cudaLaunchKernelEx(&cfg, k_dgt_fwd<LOGNC, LOGR, CL>, data, fsrc, A, nres, rid_off, poly_stride, CL, 1,
                             (unsigned)blocks);
  } else {
    if (int rc = ensure_smem(k_dgt_inv<LOGNC, LOGR, CL>, smem, done_i)) return rc;
    if (!schedulable(k_dgt_inv<LOGNC, LOGR, CL>, ok_i)) return kNoCluster;
    err = cudaLaunchKernelEx(&cfg, k_dgt_inv<LOGNC, LOGR, CL>, data, isrc, A, nres, rid_off, poly_stride, CL, 0,
                             (unsigned)blocks);
  }
  if (err != cudaSuccess) return cuda_fail("dgt (cluster)", err);
  return check_launch("dgt (cluster)");
}

// (logNc, logR, split bits) -> cluster instantiation, or nullptr.
RunFn pick_cluster(int logNc, int logR, int S) {
#define CP_CASE(A, B, C) \
  if (logNc == A && logR == B && S == C) return &run_cluster<A, B, C>;
  CP_CASE(11, 3, 1) CP_CASE(11, 3, 2) CP_CASE(12, 3, 1) CP_CASE(12, 3, 2) CP_CASE(13, 3, 1) CP_CASE(13, 3, 2)
#undef CP_CASE
  return nullptr;
}

// The plan's split stage inside a cluster, when the plan asks for it and a kernel exists;
// returns kNoCluster otherwise (nothing launched).
int try_cluster(const Engine& e, const DgtPlan& P, const DgtTableLayout& L, ulonglong2* data, const ulonglong2* fsrc,
                const InvSrc& isrc, int nres, int rid_off, int npolys, long long poly_stride, bool inverse,
                cudaStream_t st, const int* rid_list) {
  if (!P.cluster || P.S == 0) return kNoCluster;
  RunFn fc = pick_cluster(P.logNc, P.logR, P.S);
  if (!fc) return kNoCluster;
  return fc(e, P, L, data, fsrc, isrc, nres, rid_off, npolys, poly_stride, inverse, false, st, rid_list);
}

// (logNc, effective logR) -> instantiation.
RunFn pick(int logNc, int logR) {
#define CP_CASE(A, B) \
  if (logNc == A && logR == B) return &run_cta<A, B>;
  CP_CASE(1, 1) CP_CASE(2, 2) CP_CASE(3, 3) CP_CASE(4, 4) CP_CASE(4, 3)
  CP_CASE(5, 4) CP_CASE(5, 3) CP_CASE(6, 4) CP_CASE(6, 3) CP_CASE(7, 4) CP_CASE(7, 3)
  CP_CASE(8, 4) CP_CASE(8, 3) CP_CASE(9, 4) CP_CASE(9, 3) CP_CASE(10, 4) CP_CASE(10, 3)
  CP_CASE(11, 4) CP_CASE(11, 3) CP_CASE(12, 4) CP_CASE(12, 3) CP_CASE(13, 4) CP_CASE(13, 3)
  CP_CASE(5, 2) CP_CASE(6, 2) CP_CASE(7, 2) CP_CASE(8, 2) CP_CASE(9, 2) CP_CASE(10, 2)
  CP_CASE(11, 2) CP_CASE(12, 2)
#undef CP_CASE
  return nullptr;
}

int launch_split(const Engine& e, const DgtPlan& P, const DgtTableLayout& L, ulonglong2* data, const ulonglong2* src,
                 int nres, int rid_off, int npolys, long long poly_stride, bool inverse, cudaStream_t st,
                 const int* rid_list = nullptr) {
  DgtArgs A{e.d_tab, L.stride, L, e.d_mc, rid_list};
  const int Nc = 1 << P.logNc;
  const long long blocks = (long long)npolys * nres * (Nc / 256);
  if (blocks > 0x7fffffffLL) {
    set_error("dgt: grid too large");
    return 1;
  }
  const int S = P.S, lc = P.logNc, lr = P.logR;
  if (!inverse) {
    if (S == 1)
      k_dgt_split<1, false><<<(unsigned)blocks, 256, 0, st>>>(data, src, A, nres, rid_off, poly_stride, lc, lr);
    else
      k_dgt_split<2, false><<<(unsigned)blocks, 256, 0, st>>>(data, src, A, nres, rid_off, poly_stride, lc, lr);
  } else {
    if (S == 1)
      k_dgt_split<1, true><<<(unsigned)blocks, 256, 0, st>>>(data, nullptr, A, nres, rid_off, poly_stride, lc, lr);
    else
      k_dgt_split<2, true><<<(unsigned)blocks, 256, 0, st>>>(data, nullptr, A, nres, rid_off, poly_stride, lc, lr);
  }
  return check_launch("dgt split");
}

// The plan of a launch of `units` residue transforms: the small-launch plan when the
// engine has one and the launch is at most its size, else the main plan.
struct PlanSel {
  const DgtPlan& P;
  const DgtTableLayout& L;
};
PlanSel select_plan(const Engine& e, long long units) {
  if (e.narrow_units > 0 && units <= e.narrow_units) return {e.plan_narrow, e.layout_narrow};
  return {e.plan, e.layout};
}

}  // namespace

namespace {

// One transform of npolys x nres residues with the plan selected for that many units:
// forward = split stage (when any) then the in-CTA kernel, which also twists when there is
// no split stage; inverse = the in-CTA kernel (untwisting when there is no split stage)
// then the split stage.  With the cluster form the split stage runs inside the kernel.
int run_transform(const Engine& e, ulonglong2* data, const ulonglong2* fsrc, const InvSrc& isrc, int nres,
                  int rid_off, int npolys, long long poly_stride, bool inverse, cudaStream_t st, const int* rid_list) {
  const PlanSel ps = select_plan(e, (long long)npolys * nres);
  const DgtPlan& P = ps.P;
  DgtTableLayout Lsel = ps.L;
  if (inverse && isrc.untwist > 0) {  // a prescaled untwist table (off_untwist_pre)
    if (isrc.untwist > 2) {
      set_error("dgt: unknown untwist table");
      return 1;
    }
    Lsel.off_untwist = Lsel.off_untwist_pre[isrc.untwist - 1];
  }
  const DgtTableLayout& L = Lsel;
  RunFn fn = pick(P.logNc, P.logR);
  if (!fn) {
    set_error("dgt: no kernel for this size");
    return 3;
  }
  {
    const int rc = try_cluster(e, P, L, data, fsrc, isrc, nres, rid_off, npolys, poly_stride, inverse, st, rid_list);
    if (rc != kNoCluster) return rc;
  }
  const int S = P.S;
  if (!inverse) {
    if (S > 0) {
      int rc = launch_split(e, P, L, data, fsrc, nres, rid_off, npolys, poly_stride, false, st, rid_list);
      if (rc) return rc;
      return fn(e, P, L, data, nullptr, isrc, nres, rid_off, npolys, poly_stride, false, false, st, rid_list);
    }
    return fn(e, P, L, data, fsrc, isrc, nres, rid_off, npolys, poly_stride, false, true, st, rid_list);
  }
  int rc = fn(e, P, L, data, nullptr, isrc, nres, rid_off, npolys, poly_stride, true, S == 0, st, rid_list);
  if (rc || S == 0) return rc;
  return launch_split(e, P, L, data, nullptr, nres, rid_off, npolys, poly_stride, true, st, rid_list);
}

}  // namespace

int launch_dgt_ex(const Engine& e, void* dst_v, const void* fsrc_v, const InvSrc* isrc_p, int base, int npolys,
                  long long poly_stride, bool inverse, cudaStream_t st) {
  if (base == 3) return 0;  // TBase: no transform (cuPoly dgt.cu:1087-1088)
  const int nres = e.n_residues(base);
  if (nres < 0) {
    set_error("dgt: unknown base");
    return 1;
  }
  const int rid_off = e.rid_offset(base);
  ulonglong2* data = reinterpret_cast<ulonglong2*>(dst_v);
  const ulonglong2* fsrc = reinterpret_cast<const ulonglong2*>(fsrc_v);
  if (poly_stride == 0) poly_stride = (long long)nres * e.N;
  InvSrc isrc{};
  if (isrc_p) {
    isrc = *isrc_p;
  } else {
    isrc.p[0] = data;
    isrc.mode = 0;
    isrc.npairs = 1;
  }
  return run_transform(e, data, fsrc, isrc, nres, rid_off, npolys, poly_stride, inverse, st, nullptr);
}

// Residues rid_off .. rid_off + nres - 1 of npolys polynomials (stride poly_stride
// elements), from src (nullptr: in place) into dst.
int launch_dgt_part(const Engine& e, void* dst_v, const void* src_v, int rid_off, int nres, int npolys,
                    long long poly_stride, bool inverse, cudaStream_t st) {
  if (nres <= 0 || npolys <= 0) return 0;
  ulonglong2* data = reinterpret_cast<ulonglong2*>(dst_v);
  const ulonglong2* src = reinterpret_cast<const ulonglong2*>(src_v);
  InvSrc isrc{};
  isrc.p[0] = src ? src : data;
  isrc.mode = 0;
  isrc.npairs = 1;
  return run_transform(e, data, src, isrc, nres, rid_off, npolys, poly_stride, inverse, st, nullptr);
}

int launch_dgt(const Engine& e, void* data, int base, int npolys, long long poly_stride, bool inverse,
               cudaStream_t st) {
  return launch_dgt_ex(e, data, nullptr, nullptr, base, npolys, poly_stride, inverse, st);
}

// Work-list form: `nlist` residues of N elements back to back, residue i
// transformed with engine prime rid_list[i] (a device array).  Residues of
// different polynomials and widths share one launch.
int launch_dgt_list(const Engine& e, void* data_v, const int* rid_list, int nlist, bool inverse, cudaStream_t st) {
  return launch_dgt_list_ex(e, data_v, nullptr, nullptr, rid_list, nlist, inverse, st);
}

// Work-list form with sources: forward from `fsrc` (nullptr: in place); inverse
// reading per `isrc_p` (nullptr: in place; mode 3 forms products on load).
int launch_dgt_list_ex(const Engine& e, void* data_v, const void* fsrc_v, const InvSrc* isrc_p, const int* rid_list,
                       int nlist, bool inverse, cudaStream_t st) {
  if (nlist <= 0) return 0;
  ulonglong2* data = reinterpret_cast<ulonglong2*>(data_v);
  const ulonglong2* fsrc = reinterpret_cast<const ulonglong2*>(fsrc_v);
  InvSrc isrc{};
  if (isrc_p) {
    isrc = *isrc_p;
  } else {
    isrc.p[0] = data;
    isrc.mode = 0;
    isrc.npairs = 1;
  }
  return run_transform(e, data, fsrc, isrc, 1, 0, nlist, (long long)e.N, inverse, st, rid_list);
}

}  // namespace cpoly
