// Launcher of the power-of-two operator passes (cm_op_p2.cuh).  The first
// pass of a sequence (k_op_row_fwd of the operator) launches plainly; every
// later one with programmatic stream serialization (launch_pdl).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "cm_ccg_p2.cuh"
#include "cm_launch.h"
#include "cm_op_p2.cuh"

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("CM_PDL");
    return !(e && std::strcmp(e, "0") == 0);
  }();
  return on;
}

namespace {

// Whether the passes of length code L (cm_fft_p2.cuh) run here: every
// power-of-two length; 3 * 2^m when both transform buffers of every pass fit
// a block's shared memory.
template <typename R, int L>
constexpr bool len_fits() {
  return LenCode<L>::F == 1 ||
         (!OpShape<R, L>::ONEBUF && !InvShape<R, MODE_T, L>::ONEBUF &&
          !InvShape<R, MODE_F, L>::ONEBUF && !ColShape<R, L>::ONEBUF &&
          OpShape<R, L>::SMEM <= CM_SMEM_DYN_MAX && ColShape<R, L>::SMEM <= CM_SMEM_DYN_MAX);
}

struct KernelInfo {
  bool ready = false;
  int grid_per_sm = 0;
};

template <typename R, int LOGN, typename K, typename Sh = OpShape<R, LOGN>>
int prepare(K kernel, KernelInfo& info) {
  if (info.ready) return info.grid_per_sm > 0 ? 0 : -1;
  const size_t smem = Sh::smem();
  if (cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return 1;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, Sh::THREADS, smem) != cudaSuccess)
    return 1;
  info.grid_per_sm = per_sm;
  info.ready = true;
  return per_sm > 0 ? 0 : -1;
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  }
  return n;
}

std::mutex g_op_mu;

template <typename R, int LOGN>
int row_fwd(const OpArgs<R>& a, cudaStream_t s, bool launch = true) {
  if constexpr (!len_fits<R, LOGN>()) {
    return -1;
  } else {
    typedef OpShape<R, LOGN> Sh;
    static KernelInfo info;
    int rc;
    {
      std::lock_guard<std::mutex> g(g_op_mu);
      rc = prepare<R, LOGN>(k_op_row_fwd<R, LOGN>, info);
    }
    if (rc || !launch) return rc;
    const int tiles = (a.in_rows + 2 * Sh::NP - 1) / (2 * Sh::NP);
    const int grid = std::max(1, std::min(tiles, info.grid_per_sm * sm_count()));
    k_op_row_fwd<R, LOGN><<<grid, Sh::THREADS, Sh::smem(), s>>>(a);
    return 0;
  }
}

template <typename R, int LOGX, typename K>
int prepare_col(K kernel, KernelInfo& info) {
  typedef ColShape<R, LOGX> Sh;
  if (info.ready) return info.grid_per_sm > 0 ? 0 : -1;
  const size_t smem = Sh::smem();
  if (smem > CM_SMEM_DYN_MAX) return -1;
  if (cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return 1;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, Sh::THREADS, smem) != cudaSuccess)
    return 1;
  info.grid_per_sm = per_sm;
  info.ready = true;
  return per_sm > 0 ? 0 : -1;
}

// column pass on the pair-major spectrum (k_op_col); LOGX: log2 of the
// column length (domain rows)
template <typename R, int LOGX>
int col(const OpArgs<R>& a, cudaStream_t s, bool launch = true) {
  if constexpr (!len_fits<R, LOGX>()) {
    return -1;
  } else {
    typedef ColShape<R, LOGX> Sh;
    static KernelInfo info;
    int rc;
    {
      std::lock_guard<std::mutex> g(g_op_mu);
      rc = prepare_col<R, LOGX>(k_op_col<R, LOGX>, info);
    }
    if (rc || !launch) return rc;
    const int units = a.ny / 2 + 1;
    const int groups = (units + Sh::W - 1) / Sh::W;
    const int blocks = (groups + Sh::NG - 1) / Sh::NG;
    const int grid = std::max(1, std::min(blocks, info.grid_per_sm * sm_count()));
    launch_pdl(k_op_col<R, LOGX>, grid, Sh::THREADS, Sh::smem(), s, a);
    return 0;
  }
}

template <typename R, int LOGN>
int row_inv(const OpArgs<R>& a, cudaStream_t s, bool launch = true) {
  if constexpr (!len_fits<R, LOGN>()) {
    return -1;
  } else {
    typedef OpShape<R, LOGN> Sh;
    static KernelInfo info;
    int rc;
    {
      std::lock_guard<std::mutex> g(g_op_mu);
      rc = prepare<R, LOGN>(k_op_row_inv<R, LOGN>, info);
    }
    if (rc || !launch) return rc;
    const int tiles = (a.out_rows + 2 * Sh::NP - 1) / (2 * Sh::NP);
    const int grid = std::max(1, std::min(tiles, info.grid_per_sm * sm_count()));
    launch_pdl(k_op_row_inv<R, LOGN>, grid, Sh::THREADS, Sh::smem(), s, a);
    return 0;
  }
}

template <typename R>
int dispatch_row_fwd(int logn, const OpArgs<R>& a, cudaStream_t s) {
  switch (logn) {
#define CM_CASE(L) case L: return row_fwd<R, L>(a, s);
    CM_OP_LEN_CASES(CM_CASE)
#undef CM_CASE
    default: return -1;
  }
}
template <typename R>
int dispatch_col(int logn, const OpArgs<R>& a, cudaStream_t s) {
  switch (logn) {
#define CM_CASE(L) case L: return col<R, L>(a, s);
    CM_OP_LEN_CASES(CM_CASE)
#undef CM_CASE
    default: return -1;
  }
}
template <typename R>
int dispatch_row_inv(int logn, const OpArgs<R>& a, cudaStream_t s) {
  switch (logn) {
#define CM_CASE(L) case L: return row_inv<R, L>(a, s);
    CM_OP_LEN_CASES(CM_CASE)
#undef CM_CASE
    default: return -1;
  }
}

template <typename R, int MODE, int LOGN>
int ccg_row_fwd(const CcgArgs<R>& a, cudaStream_t s, bool launch = true) {
  if constexpr (!len_fits<R, LOGN>()) {
    return -1;
  } else {
    typedef OpShape<R, LOGN> Sh;
    static KernelInfo info;
    int rc;
    {
      std::lock_guard<std::mutex> g(g_op_mu);
      rc = prepare<R, LOGN>(k_ccg_row_fwd<R, MODE, LOGN>, info);
    }
    if (rc || !launch) return rc;
    const int tiles = (a.tx + 2 * Sh::NP - 1) / (2 * Sh::NP);
    const int grid = std::max(1, std::min(tiles, info.grid_per_sm * sm_count()));
    launch_pdl(k_ccg_row_fwd<R, MODE, LOGN>, grid, Sh::THREADS, Sh::smem(), s, a);
    return 0;
  }
}

template <typename R, int MODE, int LOGN>
int ccg_row_inv(const CcgArgs<R>& a, cudaStream_t s, bool launch = true) {
  if constexpr (!len_fits<R, LOGN>()) {
    return -1;
  } else {
    typedef InvShape<R, MODE, LOGN> Sh;
    static KernelInfo info;
    int rc;
    {
      std::lock_guard<std::mutex> g(g_op_mu);
      rc = prepare<R, LOGN, decltype(&k_ccg_row_inv<R, MODE, LOGN>), Sh>(k_ccg_row_inv<R, MODE, LOGN>,
                                                                         info);
    }
    if (rc || !launch) return rc;
    const int rows = MODE == MODE_T ? a.tx : a.u_rows;
    const int tiles = (rows + 2 * Sh::NP - 1) / (2 * Sh::NP);
    const int grid = std::max(1, std::min(tiles, info.grid_per_sm * sm_count()));
    launch_pdl(k_ccg_row_inv<R, MODE, LOGN>, grid, Sh::THREADS, Sh::smem(), s, a);
    return 0;
  }
}

}  // namespace

template <typename R, int MODE>
int ccg_p2_row_fwd(const CcgArgs<R>& a, int logy, cudaStream_t s) {
  switch (logy) {
#define CM_CASE(L) case L: return ccg_row_fwd<R, MODE, L>(a, s);
    CM_OP_LEN_CASES(CM_CASE)
#undef CM_CASE
    default: return -1;
  }
}

template <typename R>
int ccg_p2_col(const OpArgs<R>& a, int logx, cudaStream_t s) {
  return dispatch_col<R>(logx, a, s);
}

template <typename R, int MODE>
int ccg_p2_row_inv(const CcgArgs<R>& a, int logy, cudaStream_t s) {
  switch (logy) {
#define CM_CASE(L) case L: return ccg_row_inv<R, MODE, L>(a, s);
    CM_OP_LEN_CASES(CM_CASE)
#undef CM_CASE
    default: return -1;
  }
}

template <typename R>
int ccg_p2_prepare(const CcgArgs<R>& a, int logx, int logy) {
  int rc = 0;
  switch (logy) {
#define CM_CASE(L)                                                       \
  case L:                                                                \
    rc = ccg_row_fwd<R, MODE_T, L>(a, nullptr, false);                   \
    if (!rc) rc = ccg_row_fwd<R, MODE_F, L>(a, nullptr, false);          \
    if (!rc) rc = ccg_row_inv<R, MODE_T, L>(a, nullptr, false);          \
    if (!rc) rc = ccg_row_inv<R, MODE_F, L>(a, nullptr, false);          \
    break;
    CM_OP_LEN_CASES(CM_CASE)
#undef CM_CASE
    default: return -1;
  }
  if (rc) return rc;
  switch (logx) {
#define CM_CASE(L) case L: return col<R, L>(a.op, nullptr, false);
    CM_OP_LEN_CASES(CM_CASE)
#undef CM_CASE
    default: return -1;
  }
}

// loads of each field in flight per thread in the element-wise passes
#define CM_EW_UNROLL 2

template <typename R>
int ccg_p2_gsum(const CcgArgs<R>& a, cudaStream_t s, bool chained) {
  const cudaError_t e =
      ew_pow2(a) ? launch_chained(chained, k_ew_gsum<R, CM_EW_UNROLL, true>, a.ew_grid, CM_EW_THREADS, 0, s, a)
                 : launch_chained(chained, k_ew_gsum<R, CM_EW_UNROLL, false>, a.ew_grid, CM_EW_THREADS, 0, s, a);
  return e == cudaSuccess ? 0 : 1;
}

template <typename R>
int ccg_p2_update(const CcgArgs<R>& a, cudaStream_t s, bool chained) {
  const cudaError_t e =
      ew_pow2(a)
          ? launch_chained(chained, k_ew_update<R, CM_EW_UNROLL, true>, a.ew_grid, CM_EW_THREADS, 0, s, a)
          : launch_chained(chained, k_ew_update<R, CM_EW_UNROLL, false>, a.ew_grid, CM_EW_THREADS, 0, s, a);
  return e == cudaSuccess ? 0 : 1;
}

template <typename R>
int ccg_p2_ew_blocks_per_sm(const CcgArgs<R>& a) {
  const bool p2 = ew_pow2(a);
  const void* ks[2] = {p2 ? (const void*)k_ew_gsum<R, CM_EW_UNROLL, true>
                          : (const void*)k_ew_gsum<R, CM_EW_UNROLL, false>,
                       p2 ? (const void*)k_ew_update<R, CM_EW_UNROLL, true>
                          : (const void*)k_ew_update<R, CM_EW_UNROLL, false>};
  int n = 1 << 30;
  for (const void* k : ks) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, CM_EW_THREADS, 0) != cudaSuccess) return -1;
    n = std::min(n, b);
  }
  return n;
}

template <typename R>
static bool len_ok(int code) {
  switch (code) {
#define CM_CASE(L) case L: return len_fits<R, L>();
    CM_OP_LEN_CASES(CM_CASE)
#undef CM_CASE
    default: return false;
  }
}

template <typename R>
int op_p2_supported(int logx, int logy, int lw) {
  (void)lw;  // the column pass reads the tables in any column tiling
  return len_ok<R>(logx) && len_ok<R>(logy);
}

template <typename R>
int op_p2_apply(const OpArgs<R>& a, int logx, int logy, cudaStream_t s) {
  if (!op_p2_supported<R>(logx, logy, a.lw)) return -1;
  int rc = dispatch_row_fwd<R>(logy, a, s);
  if (!rc) rc = dispatch_col<R>(logx, a, s);
  if (!rc) rc = dispatch_row_inv<R>(logy, a, s);
  if (!rc && cudaGetLastError() != cudaSuccess) rc = 1;
  return rc;
}

template <typename R>
int op_p2_fwd_real(const OpArgs<R>& a, int logx, int logy, cudaStream_t s) {
  if (!op_p2_supported<R>(logx, logy, a.lw) || !a.fwd_real) return -1;
  int rc = dispatch_row_fwd<R>(logy, a, s);
  if (!rc) rc = dispatch_col<R>(logx, a, s);
  if (!rc && cudaGetLastError() != cudaSuccess) rc = 1;
  return rc;
}

template int op_p2_fwd_real<double>(const OpArgs<double>&, int, int, cudaStream_t);
template int op_p2_supported<float>(int, int, int);
template int op_p2_supported<double>(int, int, int);
template int op_p2_apply<float>(const OpArgs<float>&, int, int, cudaStream_t);
template int op_p2_apply<double>(const OpArgs<double>&, int, int, cudaStream_t);
template int ccg_p2_row_fwd<float, MODE_T>(const CcgArgs<float>&, int, cudaStream_t);
template int ccg_p2_row_fwd<float, MODE_F>(const CcgArgs<float>&, int, cudaStream_t);
template int ccg_p2_row_fwd<double, MODE_T>(const CcgArgs<double>&, int, cudaStream_t);
template int ccg_p2_row_fwd<double, MODE_F>(const CcgArgs<double>&, int, cudaStream_t);
template int ccg_p2_col<float>(const OpArgs<float>&, int, cudaStream_t);
template int ccg_p2_col<double>(const OpArgs<double>&, int, cudaStream_t);
template int ccg_p2_row_inv<float, MODE_T>(const CcgArgs<float>&, int, cudaStream_t);
template int ccg_p2_row_inv<float, MODE_F>(const CcgArgs<float>&, int, cudaStream_t);
template int ccg_p2_row_inv<double, MODE_T>(const CcgArgs<double>&, int, cudaStream_t);
template int ccg_p2_row_inv<double, MODE_F>(const CcgArgs<double>&, int, cudaStream_t);
template int ccg_p2_prepare<float>(const CcgArgs<float>&, int, int);
template int ccg_p2_prepare<double>(const CcgArgs<double>&, int, int);
template int ccg_p2_gsum<float>(const CcgArgs<float>&, cudaStream_t, bool);
template int ccg_p2_gsum<double>(const CcgArgs<double>&, cudaStream_t, bool);
template int ccg_p2_update<float>(const CcgArgs<float>&, cudaStream_t, bool);
template int ccg_p2_update<double>(const CcgArgs<double>&, cudaStream_t, bool);
template int ccg_p2_ew_blocks_per_sm<float>(const CcgArgs<float>&);
template int ccg_p2_ew_blocks_per_sm<double>(const CcgArgs<double>&);
