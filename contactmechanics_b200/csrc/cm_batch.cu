// Persistent batch solver: every elastic solve of a batch runs, from the
// heights to the result fields, inside one launch.
//
// The grid is a set of thread-block clusters (CM_BATCH_CLUSTER blocks each,
// as many clusters as fit the GPU at once).  A cluster takes the next solve
// from a device queue (the host orders it by decreasing grid size), runs
// its FP32 phase, the FP64 refinement and the result fields, and takes the
// next one, so solves of uneven sizes and iteration counts never wait for
// each other and no launch is spent per pass or per iteration.
//
// Inside a cluster the blocks split the tiles of every pass (tile = rank,
// rank + CM_BATCH_CLUSTER, ...) of the same per-tile bodies the per-pass
// kernels run (cm_kernels.cuh).  A pass that feeds the next one through the
// spectrum ends at a cluster barrier (release / acquire at cluster scope, so
// the spectrum written by one block is seen by the others; those loads
// bypass L1).  A pass that reduces writes each block's partials to its
// shared memory; after the barrier every block reads all partials through
// distributed shared memory in rank order, so every block computes the same
// values bit for bit and applies the same scalar step (fin_*) to its own
// copy of the solve's state.  The state is therefore replicated, never
// exchanged, and every branch the blocks take (continue, converge, next
// phase) is the same in all blocks of the cluster: each block meets exactly
// the barriers the others meet.  A solve ends by the reference's tests or at
// its iteration budget, so every loop is bounded.
//
// Scope: solves without a hardness cap (the plastic projection's bisection
// runs on the per-pass path) and without a wall-clock timeout.
//
// Measured on a B200 against the lockstep graph of per-pass launches (the
// default batch path): 331 ms against 294 ms for 512 mixed-precision solves
// of sides 64..512, 31 ms against 25 ms for 36.  With every body of the
// solve in one kernel the registers cap residency at two 256-thread blocks
// per SM and some values spill; the blocks of a cluster then wait at the
// barriers of a pass whose tiles they do not share evenly, while the
// lockstep launches keep several tiles of different solves in flight on
// every SM.  The kernel is therefore opt-in (cm_tuning_set_batch_persistent).
#include <algorithm>
#include <mutex>

#include "cm_b200.h"
#include "cm_kernels.cuh"
#include "cm_launch.h"

#ifndef CM_BATCH_CLUSTER
#define CM_BATCH_CLUSTER 8     // blocks per cluster (the portable maximum)
#endif
#ifndef CM_BATCH_THREADS
#define CM_BATCH_THREADS 256
#endif
#ifndef CM_BATCH_MINB
#define CM_BATCH_MINB 2        // resident blocks per SM the registers are sized for
#endif

CM_DEVINL unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// every thread of every block of the cluster; orders memory at cluster scope
CM_DEVINL void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}

// the shared-memory variable at p in block `rank` of the cluster
CM_DEVINL unsigned dsmem_addr(const void* p, unsigned rank) {
  unsigned a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_addr(p)), "r"(rank));
  return a;
}
CM_DEVINL double ld_dsmem_f64(const double* p, unsigned rank) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(dsmem_addr(p, rank)) : "memory");
  return v;
}
CM_DEVINL int ld_dsmem_s32(const int* p, unsigned rank) {
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(dsmem_addr(p, rank)) : "memory");
  return v;
}

// per-block shared state of the persistent kernel
struct BatchShared {
  Slot<float> s32;
  Slot<double> s64;
  CcgState st32, st64;
  FftDesc fd;
  double part[2][CM_RED_MAX];  // this block's partials (double-buffered)
  double red_sm[32 * CM_RED_MAX];
  int job, job_read;
};

// Reduce v over the block, then over the cluster in rank order; thread 0 of
// every block applies fin to the reduced values; all threads return after
// it.  rb alternates the partial buffers: a block writes buffer b again only
// two reductions later, after a barrier that every block passes only once
// it has read buffer b.
template <int NV, typename Fin>
CM_DEVINL void cluster_reduce(BatchShared& sh, int& rb, double (&v)[NV], const int (&kinds)[NV],
                              Fin fin) {
  block_reduce<NV>(v, kinds, sh.red_sm);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) sh.part[rb][i] = v[i];
  }
  cluster_sync();
  if (threadIdx.x < 32) {
    // lane r reads block r's partials (the reads overlap), lane 0 combines
    // them in rank order
    const unsigned lane = threadIdx.x;
    double mine[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i)
      mine[i] = lane < CM_BATCH_CLUSTER ? ld_dsmem_f64(&sh.part[rb][i], lane) : 0.0;
    double acc[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] = red_neutral(kinds[i]);
#pragma unroll
    for (int r = 0; r < CM_BATCH_CLUSTER; ++r) {
#pragma unroll
      for (int i = 0; i < NV; ++i)
        acc[i] = red_apply(kinds[i], acc[i], __shfl_sync(0xffffffffu, mine[i], r));
    }
    if (lane == 0) fin(acc);
  }
  rb ^= 1;
  __syncthreads();
}

template <typename R> CM_DEVINL Slot<R>& slot_of(BatchShared& sh);
template <> CM_DEVINL Slot<float>& slot_of<float>(BatchShared& sh) { return sh.s32; }
template <> CM_DEVINL Slot<double>& slot_of<double>(BatchShared& sh) { return sh.s64; }
template <typename R> CM_DEVINL CcgState& state_of(BatchShared& sh);
template <> CM_DEVINL CcgState& state_of<float>(BatchShared& sh) { return sh.st32; }
template <> CM_DEVINL CcgState& state_of<double>(BatchShared& sh) { return sh.st64; }

// Run `body(tile)` for this block's tiles of a pass of nt tiles.
template <typename Body>
CM_DEVINL void for_tiles(int nt, unsigned rank, Body body) {
  for (int tile = (int)rank; tile < nt; tile += CM_BATCH_CLUSTER) {
    body(tile);
    __syncthreads();  // the tile's shared buffers are reused by the next one
  }
}

// The plain operator in -> out (rows, columns, leading dimension each) with
// Green's table `sel` (0 displacement, 1 force); ends at a cluster barrier.
template <typename R>
CM_DEVINL void batch_plain_op(BatchShared& sh, unsigned rank, unsigned char* smem, int sel,
                              const R* in, int in_rows, int in_cols, int in_ld, R* out, int out_rows,
                              int out_cols, int out_ld) {
  typedef typename CT<R>::C C;
  Slot<R>& S = slot_of<R>(sh);
  if (threadIdx.x == 0) {
    S.in = in;
    S.in_rows = in_rows;
    S.in_cols = in_cols;
    S.in_ld = in_ld;
    S.out = out;
    S.out_rows = out_rows;
    S.out_cols = out_cols;
    S.out_ld = out_ld;
    S.table_sel = sel;
  }
  __syncthreads();
  const CcgView cv{};
  C* tws = reinterpret_cast<C*>(smem);
  double d0 = 0, d1 = 0;
  {
    C* buf = tws + S.ny;
    C* scratch = buf + (S.row_tile >> 1) * S.ny;
    stage_fft(sh.fd, S.fy, tws, S.twy, S.ny);
    for_tiles((in_rows + S.row_tile - 1) / S.row_tile, rank, [&](int tile) {
      row_fwd_tile<R, MODE_PLAIN>(&S, cv, tile, sh.fd, tws, buf, scratch, d0, d1);
    });
  }
  cluster_sync();
  {
    C* buf = tws + S.nx;
    C* scratch = buf + S.nx * (1 << S.lw);
    stage_fft(sh.fd, S.fx, tws, S.twx, S.nx);
    for_tiles(S.nt_col, rank, [&](int tile) {
      col_tile<R, MODE_PLAIN>(&S, tile, sh.fd, tws, buf, scratch);
    });
  }
  cluster_sync();
  {
    C* buf = tws + S.ny;
    C* scratch = buf + (S.row_tile >> 1) * S.ny;
    stage_fft(sh.fd, S.fy, tws, S.twy, S.ny);
    for_tiles((out_rows + S.row_tile - 1) / S.row_tile, rank, [&](int tile) {
      row_inv_tile<R, MODE_PLAIN>(&S, cv, tile, sh.fd, tws, buf, scratch, d0, d1);
    });
  }
  cluster_sync();
}

// One phase of a solve in precision R: the heights, the initial field (from
// u0, or from the previous phase's forces f_prev), then CCG iterations until
// the phase's state is done.  The phase's slot and initial state are in sh.
template <typename R>
CM_DEVINL void batch_phase(BatchShared& sh, int& rb, unsigned rank, unsigned char* smem,
                           const BatchJob& J, double rel_pentol, const float* f_prev) {
  typedef typename CT<R>::C C;
  Slot<R>& S = slot_of<R>(sh);
  CcgState& st = state_of<R>(sh);
  const int nt_comp = S.nt_comp;
  // heights: working copy and statistics, then rms and pentol
  {
    double v[3] = {-INFINITY, INFINITY, 0.0};
    for (int tile = (int)rank; tile < nt_comp; tile += CM_BATCH_CLUSTER)
      h_prep_tile<R>(&S, tile, J.h64, v[0], v[1], v[2]);
    const int kinds[3] = {RED_MAX, RED_MIN, RED_SUM};
    cluster_reduce<3>(sh, rb, v, kinds, [&](double (&a)[3]) { fin_h_prep(st, a); });
  }
  {
    double v[1] = {0.0};
    const double mean = st.sum_cg / st.p.n_surface;
    for (int tile = (int)rank; tile < nt_comp; tile += CM_BATCH_CLUSTER)
      h_var_tile<R>(&S, tile, J.h64, mean, v[0]);
    const int kinds[1] = {RED_SUM};
    const int tx = S.tx, ty = S.ty, pa = J.pentol_auto;
    cluster_reduce<1>(sh, rb, v, kinds,
                      [&](double (&a)[1]) { fin_h_var(st, a, pa, rel_pentol, tx, ty); });
  }
  const long step = (long)CM_BATCH_CLUSTER * blockDim.x;
  const long me = (long)rank * blockDim.x + threadIdx.x;
  if (f_prev == nullptr) {
    // u = max(u0, h + offset) on the surface, then f = K u
    const long n = (long)S.nx * S.ny;
    for (long i = me; i < n; i += step) init_u_at<R>(S, J.u0, st.p.offset0, i);
    cluster_sync();
    batch_plain_op<R>(sh, rank, smem, 1, S.u, S.nx, S.ny, S.ny, S.f[0], S.tx, S.ty, S.ty);
  } else {
    // warm start from the previous phase's forces: f, then u = G f
    const long n = (long)S.tx * S.ty;
    for (long i = me; i < n; i += step) S.f[0][i] = (R)ldf(f_prev + i);
    cluster_sync();
    batch_plain_op<R>(sh, rank, smem, 0, S.f[0], S.tx, S.ty, S.ty, S.u, S.nx, S.ny, S.ny);
  }
  C* tws = reinterpret_cast<C*>(smem);
  C* rbuf = tws + S.ny;
  C* rscr = rbuf + (S.row_tile >> 1) * S.ny;
  C* cbuf = tws + S.nx;
  C* cscr = cbuf + S.nx * (1 << S.lw);
  while (!st.done) {
    const R hdn = neg_down<R>(st.p.H);
    const int has_h = st.p.has_h;
    // start of the iteration: areas, gap sums, offset
    {
      const R* f = (st.parity & 1) ? S.f[1] : S.f[0];
      int a_c = 0, a_cg = 0;
      double s_cg = 0;
      R gmax = -INFINITY, gmin = INFINITY;
      for (int tile = (int)rank; tile < nt_comp; tile += CM_BATCH_CLUSTER)
        begin_tile<R>(&S, tile, f, has_h, hdn, a_c, a_cg, s_cg, gmax, gmin);
      double v[5] = {(double)a_c, (double)a_cg, s_cg, (double)gmax, (double)gmin};
      const int kinds[5] = {RED_SUM, RED_SUM, RED_SUM, RED_MAX, RED_MIN};
      cluster_reduce<5>(sh, rb, v, kinds, [&](double (&a)[5]) { fin_begin(st, a); });
    }
    // G and the conjugation factor
    {
      const R* f = (st.parity & 1) ? S.f[1] : S.f[0];
      double v[1] = {0.0};
      const R off = (R)st.offset;
      for (int tile = (int)rank; tile < nt_comp; tile += CM_BATCH_CLUSTER)
        gsum_tile<R>(&S, tile, f, has_h, hdn, off, v[0]);
      const int kinds[1] = {RED_SUM};
      cluster_reduce<1>(sh, rb, v, kinds, [&](double (&a)[1]) { fin_gsum(st, a); });
    }
    // r = G t (the search direction is built by the forward prologue)
    double s_gt = 0, unused = 0;
    {
      CcgView cv;
      load_view(&st, cv);
      stage_fft(sh.fd, S.fy, tws, S.twy, S.ny);
      for_tiles(S.nt_rowt, rank, [&](int tile) {
        row_fwd_tile<R, MODE_T>(&S, cv, tile, sh.fd, tws, rbuf, rscr, s_gt, unused);
      });
      cluster_sync();
      stage_fft(sh.fd, S.fx, tws, S.twx, S.nx);
      for_tiles(S.nt_col, rank, [&](int tile) { col_tile<R, MODE_T>(&S, tile, sh.fd, tws, cbuf, cscr); });
      cluster_sync();
      double s_rt = 0, u1 = -INFINITY;
      stage_fft(sh.fd, S.fy, tws, S.twy, S.ny);
      for_tiles(S.nt_rowt, rank, [&](int tile) {
        row_inv_tile<R, MODE_T>(&S, cv, tile, sh.fd, tws, rbuf, rscr, s_rt, u1);
      });
      double v[2] = {s_gt, s_rt};
      const int kinds[2] = {RED_SUM, RED_SUM};
      cluster_reduce<2>(sh, rb, v, kinds, [&](double (&a)[2]) {
        st.sum_cgt = a[0];
        double b[1] = {a[1]};
        fin_tau(st, b);
      });
    }
    // force update and projection
    {
      const int par = st.parity & 1;
      const R* f = par ? S.f[1] : S.f[0];
      R* fo = par ? S.f[0] : S.f[1];
      UpdateAcc<R> A;
      const double H = st.p.H;
      const R off = (R)st.offset, tau = (R)st.tau;
      const double mix = st.cur_mixfac;
      const int branch = st.branch;
      for (int tile = (int)rank; tile < nt_comp; tile += CM_BATCH_CLUSTER)
        update_tile<R>(&S, tile, f, fo, has_h, branch, H, hdn, off, tau, mix, A);
      double v[5] = {(double)A.a_fl, (double)A.min_fn + H, (double)A.max_t, A.s_fp, (double)A.n_nc};
      const int kinds[5] = {RED_SUM, RED_MIN, RED_MAX, RED_SUM, RED_SUM};
      cluster_reduce<5>(sh, rb, v, kinds, [&](double (&a)[5]) { fin_update(st, a); });
    }
    // u = G f (the final force is built by the forward prologue), then the
    // displacement update and the convergence test
    {
      CcgView cv;
      load_view(&st, cv);
      double s_f = 0, m_f = 0;
      stage_fft(sh.fd, S.fy, tws, S.twy, S.ny);
      for_tiles(S.nt_rowt, rank, [&](int tile) {
        row_fwd_tile<R, MODE_F>(&S, cv, tile, sh.fd, tws, rbuf, rscr, s_f, m_f);
      });
      cluster_sync();
      stage_fft(sh.fd, S.fx, tws, S.twx, S.nx);
      for_tiles(S.nt_col, rank, [&](int tile) { col_tile<R, MODE_F>(&S, tile, sh.fd, tws, cbuf, cscr); });
      cluster_sync();
      double du = 0, pen = -INFINITY;
      stage_fft(sh.fd, S.fy, tws, S.twy, S.ny);
      for_tiles(S.nt_rowd, rank, [&](int tile) {
        row_inv_tile<R, MODE_F>(&S, cv, tile, sh.fd, tws, rbuf, rscr, du, pen);
      });
      double v[4] = {s_f, m_f, du, pen};
      const int kinds[4] = {RED_SUM, RED_MAX, RED_MAX, RED_MAX};
      cluster_reduce<4>(sh, rb, v, kinds, [&](double (&a)[4]) {
        double b[2] = {a[0], a[1]};
        fin_force(st, b);
        ccg_converge(st, a[2], a[3]);
      });
    }
  }
}

// result fields of the final phase, and its state to global memory
template <typename R>
CM_DEVINL void batch_result(BatchShared& sh, int& rb, unsigned rank, const BatchJob& J) {
  Slot<R>& S = slot_of<R>(sh);
  CcgState& st = state_of<R>(sh);
  double v[4] = {0, 0, 0, 0};
  for (int tile = (int)rank; tile < S.nt_comp; tile += CM_BATCH_CLUSTER)
    result_tile<R>(&S, tile, st.parity, st.p.has_h, st.branch == 1, st.p.H, J.jac, J.active,
                   J.plastic, v);
  const int kinds[4] = {RED_SUM, RED_SUM, RED_SUM, RED_SUM};
  cluster_reduce<4>(sh, rb, v, kinds, [&](double (&a)[4]) { fin_result(st, a); });
  if (J.x) {
    const long n = (long)S.nx * S.ny;
    for (long i = (long)rank * blockDim.x + threadIdx.x; i < n; i += (long)CM_BATCH_CLUSTER * blockDim.x)
      J.x[i] = (double)ldf(S.u + i);
  }
}

// copy a state to global memory (thread 0 of rank 0)
CM_DEVINL void put_state(CcgState* dst, const CcgState& src) {
  const int n = (int)(sizeof(CcgState) / sizeof(int));
  for (int i = 0; i < n; ++i) reinterpret_cast<int*>(dst)[i] = reinterpret_cast<const int*>(&src)[i];
}

template <typename R>
CM_DEVINL void load_slot(Slot<R>& dst, const Slot<R>& src) {
  const int n = (int)(sizeof(Slot<R>) / sizeof(int));
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    reinterpret_cast<int*>(&dst)[i] = reinterpret_cast<const int*>(&src)[i];
}

__global__ void __launch_bounds__(CM_BATCH_THREADS, CM_BATCH_MINB)
k_batch_solve(const BatchJob* __restrict__ jobs, const int* __restrict__ order, int n, int* next) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BatchShared sh;
  const unsigned rank = cluster_rank();
  int rb = 0;
  while (true) {
    // rank 0 takes the next solve; the others read its choice
    if (rank == 0 && threadIdx.x == 0) sh.job = atomicAdd(next, 1);
    cluster_sync();
    if (threadIdx.x == 0) sh.job_read = ld_dsmem_s32(&sh.job, 0);
    // every block has read rank 0's choice before rank 0 writes it again or
    // exits (a block's shared memory must outlive the other blocks' reads)
    cluster_sync();
    const int q = sh.job_read;
    if (q >= n) break;
    const BatchJob& J = jobs[order[q]];
    const int prec = J.prec;
    if (prec != CM_FP64) {
      load_slot(sh.s32, J.s32);
      if (threadIdx.x == 0) sh.st32 = J.init32;
      __syncthreads();
      batch_phase<float>(sh, rb, rank, smem, J, prec == CM_MIXED ? J.rel_pentol32 : 0.0, nullptr);
    }
    // the FP32 phase's error states end the solve (the host reports them)
    const bool refine = prec == CM_FP64 ||
                        (prec == CM_MIXED && (sh.st32.status == CMS_CONVERGED || sh.st32.status == CMS_MAXITER));
    if (refine) {
      load_slot(sh.s64, J.s64);
      if (threadIdx.x == 0) {
        sh.st64 = J.init64;
        if (prec == CM_MIXED) sh.st64.p.maxiter = max(1, J.maxiter - sh.st32.it);
      }
      __syncthreads();
      const float* fp = nullptr;
      if (prec == CM_MIXED) fp = (sh.st32.parity & 1) ? sh.s32.f[1] : sh.s32.f[0];
      batch_phase<double>(sh, rb, rank, smem, J, 0.0, fp);
      batch_result<double>(sh, rb, rank, J);
    } else if (prec == CM_FP32) {
      batch_result<float>(sh, rb, rank, J);
    }
    if (rank == 0 && threadIdx.x == 0) {
      if (prec != CM_FP64) put_state(J.s32.st, sh.st32);
      if (refine) put_state(J.s64.st, sh.st64);
    }
    // every block has finished with sh before the next solve overwrites it
    cluster_sync();
  }
}

int batch_solve_launch(const BatchJob* jobs, const int* order, int n, int* next, size_t smem,
                       cudaStream_t s, int* clusters) {
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [] {
    attr_err = cudaFuncSetAttribute(k_batch_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)CM_SMEM_DYN_MAX);
  });
  if (attr_err != cudaSuccess) return 1;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CM_BATCH_CLUSTER;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(CM_BATCH_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(CM_BATCH_CLUSTER);
  int nc = 0;
  if (cudaOccupancyMaxActiveClusters(&nc, k_batch_solve, &cfg) != cudaSuccess || nc < 1) {
    cudaGetLastError();
    return 1;
  }
  nc = std::min(nc, n);
  cfg.gridDim = dim3(nc * CM_BATCH_CLUSTER);
  if (clusters) *clusters = nc;
  if (cudaLaunchKernelEx(&cfg, k_batch_solve, jobs, order, n, next) != cudaSuccess) return 1;
  return 0;
}
