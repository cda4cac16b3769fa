// Host side of libcm_b200: plans, Green's tables, operator application and
// the constrained-conjugate-gradient driver behind the C ABI of cm_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "cm_b200.h"
#include "cm_kernels.cuh"
#include "cm_launch.h"

// Named range of a timeline (NVTX): the library's entry points and solve
// phases show up in profilers that record NVTX (no cost without one).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

#define CM_SMEM_ROW (64 * 1024)   // ping-pong buffers of a row tile
#define CM_COMP_ELEMS 2048
#define CM_MAX_PARTIAL_VALS 32
#define CM_FP32_ITER_CAP 2000
#define CM_FP32_ITER_CAP_PLASTIC 256
// iterations the FP64 refinement of a mixed single solve may take before it
// restarts cold: at least CM_REFINE_MIN_ITERS, else CM_REFINE_PER_FP32_ITER
// per FP32-phase iteration (refinements seen: 10-170 iterations)
#define CM_REFINE_MIN_ITERS 1000
#define CM_REFINE_PER_FP32_ITER 4
#ifndef CM_BY_VALUE_PASSES
#define CM_BY_VALUE_PASSES 1  // single solves on power-of-two domains use cm_ccg_p2.cuh
#endif

#define CK(...)                               \
  do {                                        \
    cudaError_t e_ = (__VA_ARGS__);           \
    if (e_ != cudaSuccess) {                  \
      last_cuda_error() = e_;                 \
      return CM_ERR_CUDA;                     \
    }                                         \
  } while (0)

#define CKS(...)                     \
  do {                               \
    int s_ = (__VA_ARGS__);          \
    if (s_ != CM_OK) return s_;      \
  } while (0)

// kernels launched by this library (serving worker threads launch concurrently)
static std::atomic<unsigned long long> g_launches{0};
static thread_local int g_polls = 0;        // convergence polls of the current call

// Iterations the FP32 phase of a mixed solve may take: at most
// CM_FP32_ITER_CAP (CM_FP32_ITER_CAP_PLASTIC with a hardness) and half of the
// solve's maxiter, so that a phase that stalls at FP32 resolution leaves the
// FP64 refinement at least half.  Plastic phases get the lower cap: on
// plastic requests whose FP64 solve converges in 40-214 iterations, FP32
// phases were seen to run to 2000 without meeting the load test.
static int fp32_cap(int maxiter, bool plastic) {
  return std::min(plastic ? CM_FP32_ITER_CAP_PLASTIC : CM_FP32_ITER_CAP, std::max(1, maxiter / 2));
}

static cudaError_t& last_cuda_error() {
  static thread_local cudaError_t e = cudaSuccess;
  return e;
}

// ---------------------------------------------------------------------------
// FFT descriptors and twiddles
// ---------------------------------------------------------------------------
static bool make_fft_desc(int n, FftDesc* d) {
  memset(d, 0, sizeof(*d));
  d->n = n;
  int m = n, k = 0;
  auto push = [&](int r) {
    if (k >= CM_MAX_STAGES) return false;
    d->rad[k++] = r;
    return true;
  };
  while (m % 8 == 0 && m >= 8) { if (!push(8)) return false; m /= 8; }
  while (m % 4 == 0) { if (!push(4)) return false; m /= 4; }
  while (m % 2 == 0) { if (!push(2)) return false; m /= 2; }
  const int small[3] = {3, 5, 7};
  for (int p : small)
    while (m % p == 0) { if (!push(p)) return false; m /= p; }
  for (int p = 11; m > 1; p += 2) {
    while (m % p == 0) {
      if (!push(p)) return false;
      d->generic = 1;
      m /= p;
    }
  }
  d->nst = k;
  return true;
}

template <typename C>
static std::vector<C> make_twiddles(int n) {
  std::vector<C> tw(n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < n; ++m) {
    const long double a = -two_pi * (long double)m / (long double)n;
    tw[m].x = (decltype(tw[m].x))cosl(a);
    tw[m].y = (decltype(tw[m].y))sinl(a);
  }
  return tw;
}

struct Tiles {
  bool generic_ok;                  // the per-pass kernels fit (else only the by-value passes)
  int row_tile, col_tile, lw, comp_rows;
  int threads_row, threads_col;
  size_t smem_row, smem_col;
  int ntile_cols;  // number of spectrum column tiles
};

static int pow2_threads(size_t work) {
  // about sixteen transform elements per thread, 128..256 threads
  size_t t = 128;
  while (t < 256 && t * 16 < work) t *= 2;
  return (int)t;
}

// ---------------------------------------------------------------------------
// tuning of the per-pass kernels (batched solves, stepping interface, sizes
// without power-of-two passes): transform elements per row or column tile
// by sequence length and precision, and the threads of a batched transform
// launch; set through cm_tuning_* (the package's autotuner measures them)
// ---------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::vector<std::pair<int, int>> g_tune_elems[2];  // [FP64, FP32]: (length, elements)
static int g_batch_threads[2] = {CM_THREADS, CM_THREADS};
// batches of elastic solves run in the persistent cluster kernel (cm_batch.cu)
// when set; by default they take the lockstep per-pass graph, measured faster
static std::atomic<int> g_batch_persistent{0};

static int tuned_elems(size_t csize, int length, int dflt) {
  const int pi = csize == 16 ? 0 : 1;
  std::lock_guard<std::mutex> g(g_tune_mu);
  for (const auto& e : g_tune_elems[pi])
    if (e.first == length) return e.second;
  return dflt;
}

// Tile shapes: a row tile holds `row_tile` real rows (packed in pairs), a
// column tile `col_tile` = 2^lw half-spectrum columns.  Shared memory holds
// the twiddles of the transform plus two ping-pong buffers; when a sequence
// and its buffers do not fit (FP64 sides of 8192), generic_ok is false and
// only the power-of-two by-value passes can serve the plan.
static int choose_tiles(int nx, int ny, int nyh, int tx, int ty, size_t csize, Tiles* t) {
  // 2048 transform elements per tile by default (the autotuner's table sets
  // others per sequence length): several blocks share an SM and overlap
  // memory with compute
  const size_t elems_max = CM_SMEM_ROW / (2 * csize);
  const size_t elems = std::min<size_t>(elems_max, 2048);
  const size_t relems = std::min<size_t>(std::max(tuned_elems(csize, ny, (int)elems), 1), elems_max);
  const size_t celems = std::min<size_t>(std::max(tuned_elems(csize, nx, (int)elems), 1), elems_max);
  int np = (int)std::max<size_t>(1, relems / (size_t)ny);
  np = std::min(np, (nx + 1) / 2);
  const size_t srow = (2 * (size_t)np * ny + ny) * csize;
  t->generic_ok = srow <= CM_SMEM_DYN_MAX;
  t->row_tile = 2 * np;
  t->smem_row = srow;
  t->threads_row = pow2_threads((size_t)np * ny);
  int lw = 0;
  while ((2ul << lw) * (size_t)nx <= celems && (1 << (lw + 1)) <= nyh) ++lw;
  const size_t scol = (2 * ((size_t)1 << lw) * nx + nx) * csize;
  t->generic_ok = t->generic_ok && scol <= CM_SMEM_DYN_MAX;
  t->lw = lw;
  t->col_tile = 1 << lw;
  t->smem_col = scol;
  t->threads_col = pow2_threads(((size_t)1 << lw) * nx);
  t->ntile_cols = (nyh + t->col_tile - 1) / t->col_tile;
  t->comp_rows = std::max(1, std::min(tx, CM_COMP_ELEMS / std::max(1, ty)));
  return CM_OK;
}

// ---------------------------------------------------------------------------
// Green's-function tables (FP64 on the device)
// ---------------------------------------------------------------------------
__global__ void k_table_periodic(double* G, int nx, int ny, int nyh, double sx, double sy,
                                 double Es, double young, double poisson, int q0_mode,
                                 double q0_val, double thick, int dim) {
  const double pi = 3.14159265358979323846;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)nx * nyh;
       idx += (long)gridDim.x * blockDim.x) {
    const int x = (int)(idx / nyh), k = (int)(idx % nyh);
    const double qx = ((x <= nx / 2) ? (double)x : (double)(nx - x)) / sx;
    const double qy = (double)k / sy;
    const double q = sqrt(qx * qx + qy * qy);
    double K = (pi * Es) * q;
    if (thick > 0 && dim == 2) {
      const double qq = q * (2 * pi * thick);
      const double fac = 3 - 4 * poisson;
      const double off = 4 * poisson * (2 * poisson - 3) + 5;
      double corr = (fac * cosh(2 * qq) + 2 * (qq * qq) + off) / (fac * sinh(2 * qq) - 2 * qq);
      if (isnan(corr)) corr = 1.0;
      K *= corr;
    }
    if (x == 0 && k == 0) {
      if (thick > 0 && dim == 2) {
        K = young / thick * (1 - poisson) / ((1 - 2 * poisson) * (1 + poisson));
      } else if (q0_mode == CM_Q0_DEFAULT) {
        K = (dim == 1) ? (pi * Es) * (1.0 / sx) : ((pi * Es) * (1.0 / sx) + (pi * Es) * (1.0 / sy)) / 2;
      } else if (q0_mode == CM_Q0_ZERO) {
        K = 1.0;
      } else {
        K = q0_val;
      }
    }
    double g = 1.0 / K;
    if (x == 0 && k == 0 && q0_mode == CM_Q0_ZERO) g = 0.0;
    G[idx] = g;
  }
}

// Love's kernel: displacement of a uniformly loaded dx x dy pixel
// (FFTElasticHalfSpace.py:1033-1137, Johnson 1985 p.54).  The formula sums
// four corner terms that cancel: at a distance of r pixels they exceed the
// result by about r^2, so evaluated in FP64 it carries relative errors of
// about r^2 * 1e-16 (1e-9 of the displacement at a 1024^2 topography, more
// for the far periodic images of a semi-periodic kernel).  It is therefore
// evaluated on the host in extended precision and rounded once to FP64, on
// the quadrant of non-negative offsets only (the kernel, and its sum over a
// symmetric range of periodic images, is even in x and y):
//   q[a][b] = sum over images (mx, my) of love(a dx + mx Lx, b dy + my Ly),
// a < qx, b < qy; images -nimx..nimx along x (Lx the period), likewise y.
struct LoveKey {
  int qx, qy, nimx, nimy;
  double dx, dy, young, Lx, Ly;
  bool operator==(const LoveKey& o) const {
    return qx == o.qx && qy == o.qy && nimx == o.nimx && nimy == o.nimy && dx == o.dx &&
           dy == o.dy && young == o.young && Lx == o.Lx && Ly == o.Ly;
  }
};

static void love_quadrant_compute(std::vector<double>& q, const LoveKey& k) {
  typedef long double L;
  const L pi = 3.141592653589793238462643383279502884L;
  const L dx = k.dx, dy = k.dy, a = dx / 2, b = dy / 2, c = 1 / (pi * (L)k.young);
  const L Lx = k.Lx, Ly = k.Ly;
  const int qx = k.qx, qy = k.qy;
  q.assign((size_t)qx * qy, 0.0);
  auto rows = [&](int i0, int i1) {
    for (int i = i0; i < i1; ++i) {
      for (int j = 0; j < qy; ++j) {
        L v = 0;
        for (int mx = -k.nimx; mx <= k.nimx; ++mx) {
          const L x = (L)i * dx + (L)mx * Lx, xp = x + a, xm = x - a;
          for (int my = -k.nimy; my <= k.nimy; ++my) {
            const L y = (L)j * dy + (L)my * Ly, yp = y + b, ym = y - b;
            const L r_pp = sqrtl(yp * yp + xp * xp), r_mp = sqrtl(ym * ym + xp * xp);
            const L r_pm = sqrtl(yp * yp + xm * xm), r_mm = sqrtl(ym * ym + xm * xm);
            v += xp * logl((yp + r_pp) / (ym + r_mp)) + yp * logl((xp + r_pp) / (xm + r_pm)) +
                 xm * logl((ym + r_mm) / (yp + r_pm)) + ym * logl((xm + r_mm) / (xp + r_mp));
          }
        }
        q[(size_t)i * qy + j] = (double)(c * v);
      }
    }
  };
  const int nt = std::max(1, std::min(32, (int)std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  const int per = (qx + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const int i0 = t * per, i1 = std::min(qx, i0 + per);
    if (i0 < i1) pool.emplace_back(rows, i0, i1);
  }
  for (auto& th : pool) th.join();
}

// The quadrant of the last few geometries, so that plans of a geometry seen
// before (a pool of solvers of one size) skip the extended-precision pass.
#define CM_LOVE_CACHE 16
static std::mutex g_love_mu;
static std::vector<std::pair<LoveKey, std::shared_ptr<const std::vector<double>>>> g_love_cache;

static std::shared_ptr<const std::vector<double>> love_quadrant(const LoveKey& key) {
  {
    std::lock_guard<std::mutex> g(g_love_mu);
    for (size_t i = 0; i < g_love_cache.size(); ++i)
      if (g_love_cache[i].first == key) {
        auto hit = g_love_cache[i];
        g_love_cache.erase(g_love_cache.begin() + i);
        g_love_cache.push_back(hit);  // most recently used last
        return hit.second;
      }
  }
  auto q = std::make_shared<std::vector<double>>();
  love_quadrant_compute(*q, key);
  std::lock_guard<std::mutex> g(g_love_mu);
  g_love_cache.emplace_back(key, q);
  if (g_love_cache.size() > CM_LOVE_CACHE) g_love_cache.erase(g_love_cache.begin());
  return q;
}

// out[i][j] of the (nxd, nyd) domain = quadrant value at the absolute
// signed offset (|x|, |y|) = (min(i, nxd - i), min(j, nyd - j)) pixels; the
// quadrant has rows of qy values
__global__ void k_love_expand(double* out, const double* q, int qy, int nxd, int nyd) {
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < (long)nxd * nyd;
       idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / nyd), j = (int)(idx % nyd);
    const int ai = min(i, nxd - i), aj = min(j, nyd - j);
    out[idx] = q[(size_t)ai * qy + aj];
  }
}

// real part of a spectrum stored in column tiles of width 2^lw -> natural (nx, nyh)
__global__ void k_real_part(const double2* spec, double* G, int nx, int nyh, int lw) {
  const long n = (long)nx * nyh;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i / nyh), k = (int)(i % nyh);
    G[i] = spec[spec_at(x, k, nx, lw)].x;
  }
}

// Scaled operator tables in the tiled spectrum layout of each precision:
// disp = -G/(a N), force = -K a / N with K = 1/G (G != 0).
__global__ void k_tables_scale(const double* G, int nx, int nyh, double aN_inv, double a_over_N,
                               double* td, double* tf, int lw64, float* td32, float* tf32, int lw32) {
  const long n = (long)nx * nyh;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i / nyh), k = (int)(i % nyh);
    const double g = G[i];
    const double kk = (g != 0.0) ? 1.0 / g : 0.0;
    const double d = -g * aN_inv, f = -kk * a_over_N;
    const size_t j64 = spec_at(x, k, nx, lw64), j32 = spec_at(x, k, nx, lw32);
    td[j64] = d;
    tf[j64] = f;
    td32[j32] = (float)d;
    tf32[j32] = (float)f;
  }
}

// ---------------------------------------------------------------------------
// CCG preparation and result kernels
// ---------------------------------------------------------------------------
// heights -> working precision; max, min and sum of the heights.
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_h_prep(const Slot<R>* __restrict__ slots, const int2* __restrict__ items, const double* h64) {
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  double v[3] = {-INFINITY, INFINITY, 0.0};
  h_prep_tile<R>(Sp, item.y, h64 ? h64 : Sp->h64, v[0], v[1], v[2]);
  const int kinds[3] = {RED_MAX, RED_MIN, RED_SUM};
  CcgState* st = Sp->st;
  tile_finish<3>(Sp->partials, Sp->counter, item.y, Sp->nt_comp, v, kinds,
                 [&](double (&a)[3]) { fin_h_prep(*st, a); });
}

// rms height and the default penetration tolerance; pentol_auto < 0: from
// the solve's own parameters (pentol <= 0), batches of mixed callers
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_h_var(const Slot<R>* __restrict__ slots, const int2* __restrict__ items, const double* h64,
        int pentol_auto, double rel_pentol) {
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  double v[1] = {0.0};
  h_var_tile<R>(Sp, item.y, h64 ? h64 : Sp->h64, st->sum_cg / st->p.n_surface, v[0]);
  const int kinds[1] = {RED_SUM};
  const int tx = Sp->tx, ty = Sp->ty;
  tile_finish<1>(Sp->partials, Sp->counter, item.y, Sp->nt_comp, v, kinds, [&](double (&a)[1]) {
    const int automatic = pentol_auto >= 0 ? pentol_auto : (st->p.pentol <= 0);
    fin_h_var(*st, a, automatic, rel_pentol, tx, ty);
  });
}

// Lockstep batches: every solve's initial state (staged in `init`) to its
// slot, reduction ticket cleared.
template <typename R>
__global__ void k_put_states(const Slot<R>* __restrict__ slots, const CcgState* __restrict__ init,
                             int n) {
  const int words = (int)(sizeof(CcgState) / sizeof(int));
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int* src = reinterpret_cast<const int*>(init + i);
    int* dst = reinterpret_cast<int*>(slots[i].st);
    for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
    if (threadIdx.x == 0) *slots[i].counter = 0;
  }
}

// Lockstep batches: initial displacement of the domain rows of a row tile
template <typename R>
__global__ void k_init_u_rows(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  const int x0 = item.y * S.row_tile;
  const int rows = min(S.row_tile, S.nx - x0);
  const double off = S.st->p.offset0;
  const long base = (long)x0 * S.ny, n = (long)rows * S.ny;
  for (long e = threadIdx.x; e < n; e += blockDim.x) init_u_at<R>(S, S.u0, off, base + e);
}

// Lockstep batches, FP64 phase of mixed solves: f = the FP32 phase's forces
// over a comp tile
template <typename R>
__global__ void k_init_f_prev(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  const CompTile<R> T(Sp, item.y);
  const float* __restrict__ fp = Sp->prev_f[Sp->prev_st->parity & 1];
  R* __restrict__ f = Sp->f[0];
  const size_t base = (size_t)T.cx0 * T.ty;
  for (int e = threadIdx.x; e < T.cn; e += blockDim.x) f[base + e] = (R)fp[base + e];
}

// Lockstep batches: result fields of every solve (outputs from the slots)
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_result_slots(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  double v[4] = {0, 0, 0, 0};
  result_tile<R>(Sp, item.y, st->parity, st->p.has_h, st->branch == 1, st->p.H, Sp->jac_out,
                 Sp->act_out, Sp->pl_out, v);
  const int kinds[4] = {RED_SUM, RED_SUM, RED_SUM, RED_SUM};
  tile_finish<4>(Sp->partials, Sp->counter, item.y, Sp->nt_comp, v, kinds,
                 [&](double (&a)[4]) { fin_result(*st, a); });
}

// Lockstep batches: the displacement of a row tile's domain rows to FP64
template <typename R>
__global__ void k_x_rows(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  if (!S.x_out) return;
  const int x0 = item.y * S.row_tile;
  const int rows = min(S.row_tile, S.nx - x0);
  const long base = (long)x0 * S.ny, n = (long)rows * S.ny;
  for (long e = threadIdx.x; e < n; e += blockDim.x) S.x_out[base + e] = (double)ldf(S.u + base + e);
}

template <typename R>
__global__ void k_init_u(Slot<R> S, const double* u0, double offset) {
  const long n = (long)S.nx * S.ny;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    init_u_at<R>(S, u0, offset, i);
}

// copy the topography part of a domain-sized FP64 force field
template <typename R>
__global__ void k_init_f(Slot<R> S, const double* f0, int ld) {
  const long n = (long)S.tx * S.ty;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i / S.ty), y = (int)(i % S.ty);
    S.f[0][i] = (R)f0[(size_t)x * ld + y];
  }
}

// result.jac, active_set, plastic and the elastic energy
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_result(const Slot<R>* __restrict__ slots, const int2* __restrict__ items, double* jac,
             unsigned char* active, unsigned char* plastic) {
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  double v[4] = {0, 0, 0, 0};
  result_tile<R>(Sp, item.y, st->parity, st->p.has_h, st->branch == 1, st->p.H, jac, active,
                 plastic, v);
  const int kinds[4] = {RED_SUM, RED_SUM, RED_SUM, RED_SUM};
  tile_finish<4>(Sp->partials, Sp->counter, item.y, Sp->nt_comp, v, kinds,
                 [&](double (&a)[4]) { fin_result(*st, a); });
}

template <typename R>
__global__ void k_to_f64(const R* src, double* dst, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

// force field of one precision -> FP64 domain-sized field (zero padding)
template <typename R>
__global__ void k_force_to_domain(const CcgState* st, const R* f0, const R* f1, int tx, int ty,
                                  double* out, int nx, int ny) {
  const R* f = st->parity ? f1 : f0;  // the buffer holding the solver's current forces
  // a force the phase set to the hardness cap (-H rounded to R) goes on
  // exactly at -H, where the FP64 iteration would have put it
  const bool cap = st->p.has_h != 0;
  const double H = st->p.H;
  const R fcap = (R)(-H);
  const long n = (long)nx * ny;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i / ny), y = (int)(i % ny);
    double v = 0.0;
    if (x < tx && y < ty) {
      const R fv = f[(size_t)x * ty + y];
      v = (cap && fv == fcap) ? -H : (double)fv;
    }
    out[i] = v;
  }
}

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
template <typename R>
struct Work {
  typedef typename CT<R>::C C;
  Tiles tiles{};
  C* twx = nullptr;
  C* twy = nullptr;
  C* spec = nullptr;
  R* tab[2] = {nullptr, nullptr};
  Slot<R>* d_plain = nullptr;  // slot used by cm_apply
  Slot<R>* d_ccg = nullptr;    // slot used by the solver
  // solver fields
  R* h = nullptr;
  R* u = nullptr;
  R* f[2] = {nullptr, nullptr};
  R* t = nullptr;
  unsigned char* gneg = nullptr;
  CcgState* st = nullptr;
  double* partials = nullptr;
  unsigned int* counter = nullptr;
  bool ccg_ready = false;
  GridBarrier* bar = nullptr;   // one-launch bisection: grid barrier
  bool by_value = false;    // single solves: the by-value power-of-two passes (cm_ccg_p2.cuh)
  int ew_grid[5] = {0, 0, 0, 0, 0};  // by-value path: grids of begin, gsum, update, bisect,
                                     // and of the one-launch bisection (0: not used)
  CcgArgs<R> ccg_args{};    // their arguments
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // [bisect passes]
  int graph_iters[2] = {0, 0};
  int graph_variant[2] = {0, 0};  // ccg_args.u_rows and fuse_gsum the graph was captured with
  int nt_comp = 0, nt_rowt = 0, nt_rowd = 0, nt_col = 0;
  int partial_blocks = 0;   // blocks whose reduction partials fit the partials buffer
};

struct cm_plan {
  cm_plan_desc d;
  int nx, ny, nyh, tx, ty;
  FftDesc fx, fy;
  cudaStream_t stream;
  bool own_stream;
  double* G = nullptr;
  double* tab64[2] = {nullptr, nullptr};
  float* tab32[2] = {nullptr, nullptr};
  int2* items = nullptr;
  int max_items = 0;
  Work<float> w32;
  Work<double> w64;
  // pinned host states: [0] readback, [1] and [2] staging of the FP32 and FP64
  // initial states (a pageable source would make each copy wait for the stream)
  CcgState* h_state = nullptr;
  std::vector<void*> allocs;
  // stepping interface: phase of the solve this plan holds
  int phase = 0;          // 0 none, 1 FP32, 2 FP64
  int phase_prec = 0;     // CM_FP32 / CM_FP64 / CM_MIXED of the solve
  int nit32 = 0, nfev32 = 0;
  cm_ccg_params params{};
  int obs_it_offset = 0;  // observer: iterations of earlier phases of the solve
};

template <typename R> static Work<R>& work_of(cm_plan* p);
template <> Work<float>& work_of<float>(cm_plan* p) { return p->w32; }
template <> Work<double>& work_of<double>(cm_plan* p) { return p->w64; }

static int dev_alloc(cm_plan* p, void** ptr, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    last_cuda_error() = e;
    cudaGetLastError();
    return CM_ERR_OOM;
  }
  p->allocs.push_back(*ptr);
  return CM_OK;
}

template <typename T>
static int dalloc(cm_plan* p, T** ptr, size_t count) {
  return dev_alloc(p, reinterpret_cast<void**>(ptr), count * sizeof(T));
}

static int log2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return (1 << l) == n ? l : -1;
}

// Length code of the register-resident passes for a domain side
// (cm_fft_p2.cuh): log2 n for n = 2^k, 32 + m for n = 3 * 2^m, -1 otherwise.
static int len_code(int n) {
  const int l = log2_exact(n);
  if (l >= 0) return l;
  if (n % 3 == 0) {
    const int m = log2_exact(n / 3);
    if (m >= 0) return 32 + m;
  }
  return -1;
}

static int grid_for(long n) {
  long g = (n + 255) / 256;
  if (g > 148L * 16) g = 148L * 16;
  if (g < 1) g = 1;
  return (int)g;
}

template <typename R>
static void set_smem_attrs_once();

// Shared-memory attributes of the per-pass kernels, set once per process
// before any thread's first launch (callers from several threads wait for
// the first to finish).
template <typename R>
static void set_smem_attrs() {
  static std::once_flag once;
  std::call_once(once, set_smem_attrs_once<R>);
}

template <typename R>
static void set_smem_attrs_once() {
  const int mx = CM_SMEM_DYN_MAX;
  const int carve = cudaSharedmemCarveoutMaxShared;
  cudaFuncSetAttribute(k_row_fwd<R, MODE_T>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
  cudaFuncSetAttribute(k_row_fwd<R, MODE_F>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
  cudaFuncSetAttribute(k_col<R, MODE_T>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
  cudaFuncSetAttribute(k_col<R, MODE_F>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
  cudaFuncSetAttribute(k_row_inv<R, MODE_T>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
  cudaFuncSetAttribute(k_row_inv<R, MODE_F>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
  cudaFuncSetAttribute(k_row_fwd<R, MODE_PLAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_row_fwd<R, MODE_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_row_fwd<R, MODE_T>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_row_fwd<R, MODE_F>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_col<R, MODE_PLAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_col<R, MODE_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_col<R, MODE_T>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_col<R, MODE_F>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_row_inv<R, MODE_PLAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_row_inv<R, MODE_T>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_row_inv<R, MODE_F>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
}

template <typename R>
static Slot<R> base_slot(cm_plan* p, Work<R>& w) {
  Slot<R> s;
  memset(&s, 0, sizeof(s));
  s.nx = p->nx;
  s.ny = p->ny;
  s.nyh = p->nyh;
  s.tx = p->tx;
  s.ty = p->ty;
  s.row_tile = w.tiles.row_tile;
  s.col_tile = w.tiles.col_tile;
  s.lw = w.tiles.lw;
  s.comp_rows = w.tiles.comp_rows;
  s.nt_comp = (p->tx + s.comp_rows - 1) / s.comp_rows;
  s.nt_rowt = (p->tx + s.row_tile - 1) / s.row_tile;
  s.nt_rowd = (p->nx + s.row_tile - 1) / s.row_tile;
  s.nt_col = w.tiles.ntile_cols;
  s.dv_ny = make_fastdiv(p->ny);
  s.dv_nyh = make_fastdiv(p->nyh);
  s.dv_ty = make_fastdiv(p->ty);
  s.fx = p->fx;
  s.fy = p->fy;
  s.twx = w.twx;
  s.twy = w.twy;
  s.spec = w.spec;
  s.tab[0] = w.tab[0];
  s.tab[1] = w.tab[1];
  s.h = w.h;
  s.u = w.u;
  s.f[0] = w.f[0];
  s.f[1] = w.f[1];
  s.t = w.t;
  s.gneg = w.gneg;
  s.st = w.st;
  s.partials = w.partials;
  s.counter = w.counter;
  return s;
}

template <typename R>
static int init_work(cm_plan* p, Work<R>& w) {
  typedef typename CT<R>::C C;
  CKS(choose_tiles(p->nx, p->ny, p->nyh, p->tx, p->ty, sizeof(C), &w.tiles));
  std::vector<C> twx = make_twiddles<C>(p->nx), twy = make_twiddles<C>(p->ny);
  CKS(dalloc(p, &w.twx, p->nx));
  CKS(dalloc(p, &w.twy, p->ny));
  CK(cudaMemcpyAsync(w.twx, twx.data(), sizeof(C) * p->nx, cudaMemcpyHostToDevice, p->stream));
  CK(cudaMemcpyAsync(w.twy, twy.data(), sizeof(C) * p->ny, cudaMemcpyHostToDevice, p->stream));
  CKS(dalloc(p, &w.spec, (size_t)p->nx * w.tiles.ntile_cols * w.tiles.col_tile));
  CKS(dalloc(p, &w.d_plain, 1));
  CKS(dalloc(p, &w.d_ccg, 1));
  // reduction scratch is shared by the plain-operator slot and the solver
  const int nt_max = std::max({(p->tx + w.tiles.comp_rows - 1) / w.tiles.comp_rows,
                               (p->nx + w.tiles.row_tile - 1) / w.tiles.row_tile,
                               w.tiles.ntile_cols, 1});
  // (the by-value row passes use tiles of at least two rows: at most nx tiles)
  CKS(dalloc(p, &w.partials, (size_t)std::max(nt_max, p->nx) * CM_MAX_PARTIAL_VALS));
  w.partial_blocks = std::max(nt_max, p->nx);
  CKS(dalloc(p, &w.counter, 1));
  CK(cudaMemsetAsync(w.counter, 0, sizeof(unsigned int), p->stream));
  CKS(dalloc(p, &w.st, 1));
  if (nt_max > p->max_items) p->max_items = nt_max;
  return CM_OK;
}

template <typename R>
static int ensure_ccg(cm_plan* p, Work<R>& w) {
  if (w.ccg_ready) return CM_OK;
  const size_t nt = (size_t)p->tx * p->ty, nd = (size_t)p->nx * p->ny;
  CKS(dalloc(p, &w.h, nt));
  CKS(dalloc(p, &w.u, nd));
  CKS(dalloc(p, &w.f[0], nt));
  CKS(dalloc(p, &w.f[1], nt));
  CKS(dalloc(p, &w.t, nt));
  CKS(dalloc(p, &w.gneg, nt));
  CK(cudaMemsetAsync(w.t, 0, nt * sizeof(R), p->stream));
  CK(cudaMemsetAsync(w.gneg, 0, nt, p->stream));
  Slot<R> s = base_slot(p, w);
  w.nt_comp = s.nt_comp;
  w.nt_rowt = s.nt_rowt;
  w.nt_rowd = s.nt_rowd;
  w.nt_col = s.nt_col;
  CK(cudaMemcpyAsync(w.d_ccg, &s, sizeof(s), cudaMemcpyHostToDevice, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  {
    // by-value passes for domain sides 2^k and 3 * 2^m (single solves)
    const int lx = len_code(p->nx), ly = len_code(p->ny);
    CcgArgs<R>& a = w.ccg_args;
    a.op.in = nullptr;
    a.op.out = nullptr;
    a.op.in_rows = p->tx;
    a.op.in_cols = p->ty;
    a.op.in_ld = p->ty;
    a.op.out_rows = p->nx;
    a.op.out_cols = p->ny;
    a.op.out_ld = p->ny;
    a.op.nx = p->nx;
    a.op.nyh = p->nyh;
    a.op.lw = w.tiles.lw;
    a.op.ny = p->ny;
    a.op.ntile_cols = w.tiles.ntile_cols;
    a.op.spec = w.spec;
    a.op.tab = w.tab[0];
    a.op.twx = s.twx;
    a.op.twy = s.twy;
    a.op.st = s.st;
    a.op.cg_only = 0;
    a.u = w.u;
    a.h = w.h;
    a.f[0] = w.f[0];
    a.f[1] = w.f[1];
    a.t = w.t;
    a.gneg = w.gneg;
    a.st = s.st;
    a.partials = w.partials;
    a.counter = w.counter;
    a.tx = p->tx;
    a.ty = p->ty;
    a.ny = p->ny;
    a.ew_grid = 0;
    a.u_rows = p->nx;
    a.fuse_gsum = 0;
    a.ew_vpr = make_fastdiv((unsigned)(p->ty / (16 / (int)sizeof(R))));
    w.by_value = CM_BY_VALUE_PASSES && lx > 0 && ly > 0 && op_p2_supported<R>(lx, ly, w.tiles.lw);
    if (w.by_value) {
      const int rc = ccg_p2_prepare<R>(a, lx, ly);
      if (rc > 0) return CM_ERR_CUDA;
      w.by_value = rc == 0;
    }
    if (!w.by_value && !w.tiles.generic_ok) return CM_ERR_SIZE;
    if (w.by_value) {
      // the element-wise passes walk the solve's tiles with at most one
      // resident wave of blocks (one reduction partial per block)
      int dev = 0, nsm = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
      const void* ks[4] = {(const void*)k_ccg_begin<R>, (const void*)k_ccg_gsum<R>,
                           (const void*)k_ccg_update<R>, (const void*)k_ccg_bisect<R>};
      for (int k = 0; k < 4; ++k) {
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ks[k], CM_THREADS, 0));
        w.ew_grid[k] = std::max(1, std::min(w.nt_comp, per_sm * nsm));
      }
      // all bisection passes of an iteration in one cooperative launch
      int coop = 0, per_sm = 0;
      CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ccg_bisect_passes<R>, CM_THREADS, 0));
      const char* e = std::getenv("CM_BISECT_ONE_LAUNCH");
      w.ew_grid[4] = (coop && per_sm > 0 && !(e && e[0] == '0'))
                         ? std::max(1, std::min(w.nt_comp, per_sm * nsm)) : 0;
      if (w.ew_grid[4] && !w.bar) CKS(dalloc(p, &w.bar, 1));
      // the vectorised element-wise passes (gsum, force update): one resident
      // wave, no more blocks than vectors to walk or reduction partials
      const int ew_per_sm = ccg_p2_ew_blocks_per_sm<R>(a);
      if (ew_per_sm < 1) return CM_ERR_CUDA;
      const long nvec = (long)p->tx * p->ty / (16 / (long)sizeof(R));
      const long need = (nvec + 2L * 256 - 1) / (2L * 256);
      a.ew_grid = (int)std::max(1L, std::min({(long)ew_per_sm * nsm, need, (long)w.partial_blocks}));
    }
  }
  w.ccg_ready = true;
  return CM_OK;
}

template <typename R>
static int launch_plain(cm_plan* p, Work<R>& w, int mode, int table_sel, const R* in, int in_rows,
                        int in_cols, int in_ld, R* out, int out_rows, int out_cols, int out_ld,
                        cudaStream_t s) {
  set_smem_attrs<R>();
  Slot<R> hs = base_slot(p, w);
  hs.in = in;
  hs.out = out;
  hs.in_rows = in_rows;
  hs.in_cols = in_cols;
  hs.in_ld = in_ld;
  hs.out_rows = out_rows;
  hs.out_cols = out_cols;
  hs.out_ld = out_ld;
  hs.table_sel = table_sel;
  if (mode == MODE_PLAIN) {
    // domain sides 2^k and 3 * 2^m: the by-value operator passes (cm_op_p2.cuh)
    const int lx = len_code(p->nx), ly = len_code(p->ny);
    if (lx > 0 && ly > 0 && op_p2_supported<R>(lx, ly, w.tiles.lw)) {
      OpArgs<R> a;
      a.in = in;
      a.out = out;
      a.in_rows = in_rows;
      a.in_cols = in_cols;
      a.in_ld = in_ld;
      a.out_rows = out_rows;
      a.out_cols = out_cols;
      a.out_ld = out_ld;
      a.nx = p->nx;
      a.nyh = p->nyh;
      a.lw = w.tiles.lw;
      a.ny = p->ny;
      a.ntile_cols = w.tiles.ntile_cols;
      a.spec = w.spec;
      a.tab = w.tab[table_sel];
      a.twx = hs.twx;
      a.twy = hs.twy;
      a.st = nullptr;
      a.cg_only = 0;
      a.fwd_real = nullptr;
      const int rc = op_p2_apply<R>(a, lx, ly, s);
      if (rc == 0) {
        g_launches += 3;
        return CM_OK;
      }
      if (rc > 0) return CM_ERR_CUDA;
    }
  }
  if (!w.tiles.generic_ok) return CM_ERR_SIZE;  // only the by-value passes fit this domain
  CK(cudaMemcpyAsync(w.d_plain, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
  const int nt_in = (in_rows + hs.row_tile - 1) / hs.row_tile;
  const int nt_out = (out_rows + hs.row_tile - 1) / hs.row_tile;
  g_launches += (mode == MODE_FWD) ? 2 : 3;
  if (mode == MODE_FWD) {
    k_row_fwd<R, MODE_FWD><<<nt_in, w.tiles.threads_row, w.tiles.smem_row, s>>>(w.d_plain, p->items);
    k_col<R, MODE_FWD><<<hs.nt_col, w.tiles.threads_col, w.tiles.smem_col, s>>>(w.d_plain, p->items);
  } else {
    k_row_fwd<R, MODE_PLAIN><<<nt_in, w.tiles.threads_row, w.tiles.smem_row, s>>>(w.d_plain, p->items);
    k_col<R, MODE_PLAIN><<<hs.nt_col, w.tiles.threads_col, w.tiles.smem_col, s>>>(w.d_plain, p->items);
    k_row_inv<R, MODE_PLAIN><<<nt_out, w.tiles.threads_row, w.tiles.smem_row, s>>>(w.d_plain, p->items);
  }
  CK(cudaGetLastError());
  return CM_OK;
}

// G = Re FFT2(in) of a real FP64 domain field in the natural (nx, nyh) layout,
// by the register-resident row pass and a forward-only column pass; -1 when
// the domain has no such passes
static int forward_real_p2(cm_plan* p, const double* in, double* out, cudaStream_t s) {
  const int lx = len_code(p->nx), ly = len_code(p->ny);
  if (!(lx > 0 && ly > 0 && op_p2_supported<double>(lx, ly, p->w64.tiles.lw))) return -1;
  set_smem_attrs<double>();
  OpArgs<double> a;
  memset(&a, 0, sizeof(a));
  a.in = in;
  a.in_rows = p->nx;
  a.in_cols = p->ny;
  a.in_ld = p->ny;
  a.out_rows = p->nx;
  a.out_cols = p->ny;
  a.out_ld = p->ny;
  a.nx = p->nx;
  a.nyh = p->nyh;
  a.lw = p->w64.tiles.lw;
  a.ny = p->ny;
  a.ntile_cols = p->w64.tiles.ntile_cols;
  a.spec = p->w64.spec;
  a.tab = p->w64.tab[0];
  a.twx = p->w64.twx;
  a.twy = p->w64.twy;
  a.fwd_real = out;
  const int rc = op_p2_fwd_real<double>(a, lx, ly, s);
  if (rc == 0) g_launches += 2;
  return rc > 0 ? CM_ERR_CUDA : rc;
}

static int apply_dispatch(cm_plan* p, int op, int precision, const void* in, int in_rows, int in_cols,
                          int in_ld, void* out, int out_rows, int out_cols, int out_ld, cudaStream_t s) {
  if (precision == CM_FP64)
    return launch_plain<double>(p, p->w64, MODE_PLAIN, op, (const double*)in, in_rows, in_cols,
                                           in_ld, (double*)out, out_rows, out_cols, out_ld, s);
  return launch_plain<float>(p, p->w32, MODE_PLAIN, op, (const float*)in, in_rows, in_cols,
                                        in_ld, (float*)out, out_rows, out_cols, out_ld, s);
}

// ---------------------------------------------------------------------------
// solver driver
// ---------------------------------------------------------------------------
// ---- power-of-two specialisations -------------------------------------------

// kernels of one iteration, in launch order (bisection passes excluded).  The
// by-value passes launch no k_ccg_begin after the first iteration: the
// previous iteration's k_ccg_row_inv<MODE_F> computes its statistics.
#define CM_ITER_KERNELS 10
static const char* const k_iter_names[CM_ITER_KERNELS] = {
    "k_ccg_begin", "k_ccg_gsum", "k_row_fwd<T>", "k_col<T>", "k_row_inv<T>",
    "k_ccg_update", "k_row_fwd<F>", "k_col<F>", "k_row_inv<F>", "k_ccg_bisect"};

static int iteration_launches(bool bisect, bool by_value, bool one_bisect_launch = false) {
  return CM_ITER_KERNELS - (by_value ? 2 : 1) + (bisect ? (one_bisect_launch ? 1 : CM_BISECT_PASSES) : 0);
}

// One CCG iteration.  With `ev` (CM_ITER_KERNELS + 1 events) an event is
// recorded before the first and after every kernel, for the profiler.
// The by-value passes launch with programmatic stream serialization, all but
// the first kernel of a sequence (`first`: nothing of ours precedes it).
template <typename R>
static void launch_iteration(cm_plan* p, Work<R>& w, bool bisect, cudaStream_t s,
                             cudaEvent_t* ev = nullptr, bool first = true) {
  const Slot<R>* S = w.d_ccg;
  const int2* it = p->items;
  const Tiles& T = w.tiles;
  int k = 0;
  auto mark = [&]() { if (ev) cudaEventRecord(ev[k++], s); };
  // element-wise kernel k (0 begin, 1 gsum, 2 update, 3 bisect): chained
  // behind the previous pass and walking the tiles in the by-value path
  bool chain = w.by_value && !first;
  auto elementwise = [&](void (*kern)(const Slot<R>*, const int2*, int), int k) {
    const int grid = w.by_value ? w.ew_grid[k] : w.nt_comp;
    const int strided = w.by_value ? w.nt_comp : 0;
    if (chain) launch_pdl(kern, grid, CM_THREADS, 0, s, S, it, strided);
    else kern<<<grid, CM_THREADS, 0, s>>>(S, it, strided);
    chain = w.by_value;
  };
  mark();
  if (!w.by_value) elementwise(k_ccg_begin<R>, 0);
  if (bisect && w.by_value && w.ew_grid[4]) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(w.ew_grid[4]);
    cfg.blockDim = dim3(CM_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_ccg_bisect_passes<R>, S, it, w.nt_comp, w.bar) == cudaSuccess) {
      chain = true;
    } else {
      // the cooperative launch was refused (for example fewer SMs available
      // than the occupancy query counted): clear the error and run the
      // passes as separate launches from now on
      cudaGetLastError();
      w.ew_grid[4] = 0;
      for (int i = 0; i < CM_BISECT_PASSES; ++i) elementwise(k_ccg_bisect<R>, 3);
    }
  } else if (bisect) {
    for (int i = 0; i < CM_BISECT_PASSES; ++i) elementwise(k_ccg_bisect<R>, 3);
  }
  mark();
  if (w.by_value) {
    // with fuse_gsum the previous iteration's displacement pass formed G
    if (!w.ccg_args.fuse_gsum) ccg_p2_gsum<R>(w.ccg_args, s, chain);
    chain = true;
  } else {
    elementwise(k_ccg_gsum<R>, 1);
  }
  mark();
  const int ly = p->fy.n, lx = p->fx.n;
  const int ry = len_code(ly), rx = len_code(lx);
  if (w.by_value) {
    // by-value passes: one launch each; a launch error surfaces at the next check
    const CcgArgs<R>& a = w.ccg_args;
    OpArgs<R> col_t = a.op, col_f = a.op;
    col_t.out_rows = p->tx;
    col_t.cg_only = 1;
    col_f.out_rows = a.u_rows;
    ccg_p2_row_fwd<R, MODE_T>(a, ry, s);
    mark();
    ccg_p2_col<R>(col_t, rx, s);
    mark();
    ccg_p2_row_inv<R, MODE_T>(a, ry, s);
    mark();
    ccg_p2_update<R>(a, s, true);
    mark();
    ccg_p2_row_fwd<R, MODE_F>(a, ry, s);
    mark();
    ccg_p2_col<R>(col_f, rx, s);
    mark();
    ccg_p2_row_inv<R, MODE_F>(a, ry, s);
    mark();
    return;
  }
  k_row_fwd<R, MODE_T><<<w.nt_rowt, T.threads_row, T.smem_row, s>>>(S, it);
  mark();
  k_col<R, MODE_T><<<w.nt_col, T.threads_col, T.smem_col, s>>>(S, it);
  mark();
  k_row_inv<R, MODE_T><<<w.nt_rowt, T.threads_row, T.smem_row, s>>>(S, it);
  mark();
  k_ccg_update<R><<<w.nt_comp, CM_THREADS, 0, s>>>(S, it, 0);
  mark();
  k_row_fwd<R, MODE_F><<<w.nt_rowt, T.threads_row, T.smem_row, s>>>(S, it);
  mark();
  k_col<R, MODE_F><<<w.nt_col, T.threads_col, T.smem_col, s>>>(S, it);
  mark();
  k_row_inv<R, MODE_F><<<w.nt_rowd, T.threads_row, T.smem_row, s>>>(S, it);
  mark();
}

template <typename R>
static int get_graph(cm_plan* p, Work<R>& w, bool bisect, int iters, cudaGraphExec_t* out) {
  const int gi = bisect ? 1 : 0;
  const int variant = 2 * w.ccg_args.u_rows + w.ccg_args.fuse_gsum;
  if (w.graph[gi] && w.graph_iters[gi] == iters && w.graph_variant[gi] == variant) {
    *out = w.graph[gi];
    return CM_OK;
  }
  if (w.graph[gi]) {
    cudaGraphExecDestroy(w.graph[gi]);
    w.graph[gi] = nullptr;
  }
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaSuccess;
  for (int attempt = 0; attempt < 2; ++attempt) {
    const bool coop = bisect && w.ew_grid[4] > 0;
    CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeRelaxed));
    for (int i = 0; i < iters; ++i) launch_iteration<R>(p, w, bisect, p->stream, nullptr, i == 0);
    e = cudaStreamEndCapture(p->stream, &g);
    if (e == cudaSuccess) {
      e = cudaGraphInstantiate(&w.graph[gi], g, 0);
      cudaGraphDestroy(g);
    }
    if (e == cudaSuccess || !coop) break;
    // a graph with the cooperative bisection launch could not be built:
    // capture again with the bisection passes as separate launches
    cudaGetLastError();
    w.graph[gi] = nullptr;
    w.ew_grid[4] = 0;
  }
  CK(e);
  w.graph_iters[gi] = iters;
  w.graph_variant[gi] = variant;
  *out = w.graph[gi];
  return CM_OK;
}

struct SolveInput {
  const double* h64;
  const double* u0;
  const double* f0;
  int f0_ld;
};

// State, heights and initial fields of one solve (ConstrainedConjugateGradients.py
// :132-219), enqueued on stream s.
// The solver state at the start of a solve phase (ConstrainedConjugateGradients.py:132-215).
static void initial_state(const cm_plan* p, const cm_ccg_params* prm, double rel_forcetol,
                          int maxiter, CcgState& st) {
  memset(&st, 0, sizeof(st));
  CcgParams& P = st.p;
  P.F = prm->external_force;
  P.offset0 = prm->load_control ? 0.0 : prm->offset;
  P.H = prm->hardness;
  P.has_h = prm->has_hardness;
  P.pentol = prm->pentol;
  P.forcetol = prm->forcetol;
  P.thermotol = prm->thermotol;
  P.mixfac = prm->mixfac;
  P.mixdecfac = prm->mixdecfac;
  P.rel_forcetol = rel_forcetol;
  P.minmixsteps = prm->minmixsteps;
  P.maxiter = maxiter;
  P.load_control = prm->load_control;
  P.n_surface = (double)p->tx * (double)p->ty;
  st.it = 1;
  st.mode = CMM_RESET;
  st.G_old = 1.0;
  st.offset = P.offset0;
  st.cur_mixfac = P.mixfac;
  st.nfev = 1;
  st.scale = 1.0;
}

template <typename R>
static int ccg_init(cm_plan* p, Work<R>& w, const cm_ccg_params* prm, const SolveInput& in,
                    double rel_pentol, double rel_forcetol, int maxiter, cudaStream_t s) {
  set_smem_attrs<R>();
  CKS(ensure_ccg(p, w));
  CcgState st;
  initial_state(p, prm, rel_forcetol, maxiter, st);
  // Staged through pinned memory so that the copy does not wait for the
  // stream.  Every path reads a solve's results (a synchronisation) before
  // it initialises the same Work again, so the staging slot is free here.
  CcgState* stage = p->h_state + (sizeof(R) == 8 ? 2 : 1);
  *stage = st;
  CK(cudaMemcpyAsync(w.st, stage, sizeof(st), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(w.counter, 0, sizeof(unsigned int), s));  // a solve that gave up may leave it set
  if (w.bar) CK(cudaMemsetAsync(w.bar, 0, sizeof(GridBarrier), s));
  g_launches += 3;  // heights statistics (2) and the initial field
  k_h_prep<R><<<w.nt_comp, CM_THREADS, 0, s>>>(w.d_ccg, p->items, in.h64);
  k_h_var<R><<<w.nt_comp, CM_THREADS, 0, s>>>(w.d_ccg, p->items, in.h64, prm->pentol <= 0, rel_pentol);
  Slot<R> hs = base_slot(p, w);
  const int gd = grid_for((long)p->nx * p->ny);
  if (in.f0) {
    k_init_f<R><<<gd, 256, 0, s>>>(hs, in.f0, in.f0_ld);
    CKS(launch_plain<R>(p, w, MODE_PLAIN, CM_OP_DISP, w.f[0], p->tx, p->ty, p->ty, w.u, p->nx,
                              p->ny, p->ny, s));
  } else {
    k_init_u<R><<<gd, 256, 0, s>>>(hs, in.u0, st.p.offset0);
    CKS(launch_plain<R>(p, w, MODE_PLAIN, CM_OP_FORCE, w.u, p->nx, p->ny, p->ny, w.f[0], p->tx,
                              p->ty, p->ty, s));
  }
  CK(cudaGetLastError());
  return CM_OK;
}

template <typename R>
static int run_ccg(cm_plan* p, Work<R>& w, const cm_ccg_params* prm, const SolveInput& in,
                   double rel_pentol, double rel_forcetol, int maxiter, CcgState* fin,
                   int prof_iters = 0, float* prof_ms = nullptr, bool topo_u = false) {
  NvtxRange range(sizeof(R) == 8 ? "ccg phase fp64" : "ccg phase fp32");
  cudaStream_t s = p->stream;
  CKS(ccg_init(p, w, prm, in, rel_pentol, rel_forcetol, maxiter, s));
  // topo_u (FP32 phase of a mixed solve): the displacement pass updates
  // the topography's rows only and forms the next iteration's G as well
  // (set after ccg_init, whose first call on a plan initialises the arguments)
  w.ccg_args.u_rows = topo_u ? p->tx : p->nx;
  w.ccg_args.fuse_gsum = topo_u ? 1 : 0;
  if (w.by_value) {
    // start of the first iteration; later ones come from k_ccg_row_inv<MODE_F>
    k_ccg_begin<R><<<w.ew_grid[0], CM_THREADS, 0, s>>>(w.d_ccg, p->items, w.nt_comp);
    g_launches += 1;
    if (w.ccg_args.fuse_gsum) {
      CKS(ccg_p2_gsum<R>(w.ccg_args, s, true) == 0 ? CM_OK : CM_ERR_CUDA);
      g_launches += 1;
    }
  }
  const bool bisect = prm->has_hardness && prm->load_control;
  if (prof_iters > 0) {
    // profiler: eager launches with an event between kernels
    std::vector<cudaEvent_t> ev(CM_ITER_KERNELS + 1);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int k = 0; k < CM_ITER_KERNELS; ++k) prof_ms[k] = 0;
    for (int i = 0; i < prof_iters; ++i) {
      launch_iteration<R>(p, w, bisect, s, ev.data());
      CK(cudaEventSynchronize(ev[CM_ITER_KERNELS - 1]));
      for (int k = 0; k < CM_ITER_KERNELS - 1; ++k) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
        prof_ms[k] += ms / prof_iters;
      }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    CK(cudaMemcpyAsync(p->h_state, w.st, sizeof(CcgState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *fin = *p->h_state;
    return CM_OK;
  }
  int every = prm->check_every;
  if (every <= 0) {
    const long work = (long)p->nx * p->ny;
    every = work >= (1L << 20) ? (w.by_value ? 8 : 4) : (work >= (1L << 16) ? 8 : 16);
  }
  const bool observe = prm->on_iteration != nullptr && prm->iteration_forces != nullptr;
  if (observe) every = 1;
  auto t0 = std::chrono::steady_clock::now();
  cudaGraphExec_t g;
  CKS(get_graph<R>(p, w, bisect, every, &g));
  for (int done_iters = 0;; done_iters += every) {
    CK(cudaGraphLaunch(g, s));
    g_launches += (unsigned long long)every *
                   (iteration_launches(bisect, w.by_value, w.by_value && w.ew_grid[4] > 0) -
                    (w.by_value && w.ccg_args.fuse_gsum ? 1 : 0));
    CK(cudaMemcpyAsync(p->h_state, w.st, sizeof(CcgState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    ++g_polls;
    if (observe) {
      const CcgState st = *p->h_state;
      if (!(st.done && st.status == CMS_CONVERGED)) {
        // the reference reports every iteration that did not converge
        k_force_to_domain<R><<<grid_for((long)p->nx * p->ny), 256, 0, s>>>(
            w.st, w.f[0], w.f[1], p->tx, p->ty, prm->iteration_forces, p->nx, p->ny);
        g_launches += 1;
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        cm_iteration info;
        memset(&info, 0, sizeof(info));
        info.it = p->obs_it_offset + (st.done ? st.it : st.it - 1);
        info.precision = sizeof(R) == 8 ? CM_FP64 : CM_FP32;
        info.mode = st.rep_mode;
        info.done = st.done;
        info.area = st.rep_area;
        info.cg_area = st.rep_cg_area;
        info.plastic_area = st.A_fl;
        info.nc_count = st.n_nc;
        info.rms_pen = st.rms_pen;
        info.max_pen = st.max_pen;
        info.max_pres = st.max_pres;
        info.pad_pres = st.pad_pres;
        info.maxdu = st.maxdu;
        info.total_force = st.total_force;
        info.offset = st.rep_offset;
        info.tau = st.tau;
        info.mixfac = st.cur_mixfac;
        info.pentol = st.p.pentol;
        info.forcetol = std::max(st.p.forcetol, st.p.rel_forcetol * st.fmax);
        info.forces = prm->iteration_forces;
        if (prm->on_iteration(prm->user, &info) != 0) return CM_ERR_STOPPED;
      }
    }
    if (p->h_state->done) break;
    if (prm->timeout_s > 0) {
      const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (el > prm->timeout_s) return CM_ERR_TIMEOUT;
    }
    if (done_iters > maxiter + 2 * every) return CM_ERR_CUDA;  // state machine failed to stop
  }
  *fin = *p->h_state;
  if (fin->status == CMS_TIMEOUT) return CM_ERR_TIMEOUT;
  if (fin->status == CMS_NAN) return CM_ERR_NAN;
  if (fin->status == CMS_BISECT_SIGN) return CM_ERR_BISECT;
  if (fin->status == CMS_BISECT_SIGN + 1) return CM_ERR_BISECT_CONV;
  return CM_OK;
}

// Result fields of a finished solve (launches only).
template <typename R>
static int launch_result(cm_plan* p, Work<R>& w, double* x, double* jac, unsigned char* active,
                         unsigned char* plastic, cudaStream_t s) {
  k_ccg_result<R><<<w.nt_comp, CM_THREADS, 0, s>>>(w.d_ccg, p->items, jac, active, plastic);
  g_launches += 1;
  if (x) {
    k_to_f64<R><<<grid_for((long)p->nx * p->ny), 256, 0, s>>>(w.u, x, (long)p->nx * p->ny);
    g_launches += 1;
  }
  CK(cudaGetLastError());
  return CM_OK;
}

// Solver states of n plans to the host with one synchronisation.
template <typename R>
static int read_states(int n, cm_plan* const* plans, std::vector<CcgState>& out, cudaStream_t s) {
  CcgState* hb = nullptr;
  if (cudaMallocHost(&hb, sizeof(CcgState) * n) != cudaSuccess) {
    cudaGetLastError();
    return CM_ERR_OOM;
  }
  int rc = CM_OK;
  for (int i = 0; i < n && rc == CM_OK; ++i)
    if (cudaMemcpyAsync(hb + i, work_of<R>(plans[i]).st, sizeof(CcgState), cudaMemcpyDeviceToHost,
                        s) != cudaSuccess)
      rc = CM_ERR_CUDA;
  if (rc == CM_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = CM_ERR_CUDA;
  if (rc == CM_OK) out.assign(hb, hb + n);
  cudaFreeHost(hb);
  return rc;
}

template <typename R>
static int finish_ccg(cm_plan* p, Work<R>& w, double* x, double* jac, unsigned char* active,
                      unsigned char* plastic, CcgState* fin, cudaStream_t s = nullptr) {
  if (!s) s = p->stream;
  CKS(launch_result<R>(p, w, x, jac, active, plastic, s));
  CK(cudaMemcpyAsync(p->h_state, w.st, sizeof(CcgState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *fin = *p->h_state;
  return CM_OK;
}

static void fill_result(const CcgState& st, cm_ccg_result* r) {
  r->status = st.status == CMS_CONVERGED ? CM_SOLVE_CONVERGED : CM_SOLVE_MAXITER;
  r->nit = st.it;
  r->nfev = st.nfev;
  r->last_step_mix = st.branch == 1;
  r->offset = st.offset;
  r->fun = st.sum_cgt;
  r->rms_pen = st.rms_pen;
  r->max_pen = st.max_pen;
  r->max_pres = st.max_pres;
  r->pad_pres = st.pad_pres;
  r->maxdu = st.maxdu;
  r->total_force = st.total_force;
  r->pentol_used = st.p.pentol;
  r->area = st.A_contact;
  r->cg_area = st.A_cg;
  r->plastic_area = st.A_fl;
}

// ---------------------------------------------------------------------------
// batches of independent solves
// ---------------------------------------------------------------------------
// Device arrays of one batch: slot descriptors and the (slot, tile) work
// lists of the four tile spaces.
template <typename R>
struct BatchDev {
  Slot<R>* slots = nullptr;
  int2* items[4] = {nullptr, nullptr, nullptr, nullptr};  // comp, rows<tx, rows<nx, columns
  int n_items[4] = {0, 0, 0, 0};
  int* running = nullptr;  // count of running solves, then one done flag per solve
  size_t smem_row = 0, smem_col = 0;
  std::vector<void*> allocs;
  ~BatchDev() {
    for (void* a : allocs) cudaFree(a);
  }
};

// Work lists of the solves `which` (indices into the batch's slot array).
template <typename R>
static int batch_items(cm_plan* const* plans, const std::vector<int>& which, BatchDev<R>& b,
                       cudaStream_t s) {
  std::vector<int2> it[4];
  for (int i : which) {
    const Work<R>& w = work_of<R>(plans[i]);
    for (int t = 0; t < w.nt_comp; ++t) it[0].push_back(make_int2(i, t));
    for (int t = 0; t < w.nt_rowt; ++t) it[1].push_back(make_int2(i, t));
    for (int t = 0; t < w.nt_rowd; ++t) it[2].push_back(make_int2(i, t));
    for (int t = 0; t < w.nt_col; ++t) it[3].push_back(make_int2(i, t));
  }
  for (int k = 0; k < 4; ++k) {
    b.n_items[k] = (int)it[k].size();
    CK(cudaMemcpyAsync(b.items[k], it[k].data(), sizeof(int2) * it[k].size(),
                       cudaMemcpyHostToDevice, s));
  }
  CK(cudaStreamSynchronize(s));  // the host vectors go out of scope
  return CM_OK;
}

template <typename R, typename Fill>
static int batch_build(int n, cm_plan* const* plans, BatchDev<R>& b, cudaStream_t s, Fill fill) {
  std::vector<Slot<R>> hs(n);
  size_t cap[4] = {0, 0, 0, 0};
  for (int i = 0; i < n; ++i)
    if (!work_of<R>(plans[i]).tiles.generic_ok) return CM_ERR_SIZE;  // single-solve passes only
  for (int i = 0; i < n; ++i) {
    Work<R>& w = work_of<R>(plans[i]);
    hs[i] = base_slot(plans[i], w);
    fill(i, hs[i]);
    cap[0] += hs[i].nt_comp;
    cap[1] += hs[i].nt_rowt;
    cap[2] += hs[i].nt_rowd;
    cap[3] += hs[i].nt_col;
    b.smem_row = std::max(b.smem_row, w.tiles.smem_row);
    b.smem_col = std::max(b.smem_col, w.tiles.smem_col);
  }
  auto al = [&](void** ptr, size_t bytes) -> int {
    if (cudaMalloc(ptr, bytes) != cudaSuccess) { cudaGetLastError(); return CM_ERR_OOM; }
    b.allocs.push_back(*ptr);
    return CM_OK;
  };
  CKS(al((void**)&b.slots, sizeof(Slot<R>) * n));
  CK(cudaMemcpyAsync(b.slots, hs.data(), sizeof(Slot<R>) * n, cudaMemcpyHostToDevice, s));
  for (int k = 0; k < 4; ++k) CKS(al((void**)&b.items[k], sizeof(int2) * std::max<size_t>(1, cap[k])));
  CKS(al((void**)&b.running, sizeof(int) * (1 + n)));  // count, then the done flags
  std::vector<int> all(n);
  for (int i = 0; i < n; ++i) all[i] = i;
  return batch_items<R>(plans, all, b, s);
}

// One iteration of every solve of the batch (generic transforms: the solves
// may all have different sizes).
template <typename R>
static void launch_iteration_batch(const BatchDev<R>& b, bool bisect, cudaStream_t s) {
  const Slot<R>* S = b.slots;
  const int TT = g_batch_threads[sizeof(R) == 8 ? 0 : 1];  // threads of the transform launches
  k_ccg_begin<R><<<b.n_items[0], CM_THREADS, 0, s>>>(S, b.items[0], 0);
  if (bisect)
    for (int i = 0; i < CM_BISECT_PASSES; ++i)
      k_ccg_bisect<R><<<b.n_items[0], CM_THREADS, 0, s>>>(S, b.items[0], 0);
  k_ccg_gsum<R><<<b.n_items[0], CM_THREADS, 0, s>>>(S, b.items[0], 0);
  k_row_fwd<R, MODE_T><<<b.n_items[1], TT, b.smem_row, s>>>(S, b.items[1]);
  k_col<R, MODE_T><<<b.n_items[3], TT, b.smem_col, s>>>(S, b.items[3]);
  k_row_inv<R, MODE_T><<<b.n_items[1], TT, b.smem_row, s>>>(S, b.items[1]);
  k_ccg_update<R><<<b.n_items[0], CM_THREADS, 0, s>>>(S, b.items[0], 0);
  k_row_fwd<R, MODE_F><<<b.n_items[1], TT, b.smem_row, s>>>(S, b.items[1]);
  k_col<R, MODE_F><<<b.n_items[3], TT, b.smem_col, s>>>(S, b.items[3]);
  k_row_inv<R, MODE_F><<<b.n_items[2], TT, b.smem_row, s>>>(S, b.items[2]);
}

// Count the solves of a batch that have not finished; done flags after it.
template <typename R>
__global__ void k_batch_running(const Slot<R>* __restrict__ slots, int n, int* out) {
  int c = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int d = slots[i].st->done;
    out[1 + i] = d;
    c += d ? 0 : 1;
  }
  c = __reduce_add_sync(0xffffffffu, c);
  __shared__ int sm[32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < (int)(blockDim.x + 31) / 32; ++i) t += sm[i];
    out[0] = t;
  }
}

// Run the CCG loop of every solve of the batch to completion.  The work
// lists (and the graph of `every` iterations over them) are rebuilt for the
// running solves whenever their number has halved since the last build, so
// the launches of a batch's tail cover only the solves still iterating.
template <typename R>
static int batch_loop(int n, cm_plan* const* plans, BatchDev<R>& b, bool bisect, int maxiter,
                      double timeout_s, cudaStream_t s, int* polls) {
  long work = 0;
  for (int i = 0; i < n; ++i) work += (long)plans[i]->nx * plans[i]->ny;
  const int every = work >= (1L << 22) ? 4 : 16;
  cudaGraphExec_t ge = nullptr;
  auto capture = [&]() -> int {
    if (ge) cudaGraphExecDestroy(ge);
    ge = nullptr;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    for (int i = 0; i < every; ++i) launch_iteration_batch<R>(b, bisect, s);
    k_batch_running<R><<<1, 256, 0, s>>>(b.slots, n, b.running);
    CK(cudaStreamEndCapture(s, &g));
    const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    return CM_OK;
  };
  CKS(capture());
  std::vector<int> flags(1 + n);
  int running = n, built = n;
  int rc = CM_OK;
  auto t0 = std::chrono::steady_clock::now();
  for (int done_iters = 0; running > 0; done_iters += every) {
    if (cudaGraphLaunch(ge, s) != cudaSuccess) { rc = CM_ERR_CUDA; break; }
    g_launches += (unsigned long long)every * (iteration_launches(bisect, false)) + 1;
    if (cudaMemcpyAsync(flags.data(), b.running, sizeof(int) * (1 + n), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) { rc = CM_ERR_CUDA; break; }
    running = flags[0];
    if (polls) ++*polls;
    if (timeout_s > 0 &&
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_s) {
      rc = CM_ERR_TIMEOUT;
      break;
    }
    if (done_iters > maxiter + 2 * every) { rc = CM_ERR_CUDA; break; }
    if (running > 0 && 2 * running <= built) {
      std::vector<int> which;
      for (int i = 0; i < n; ++i)
        if (!flags[1 + i]) which.push_back(i);
      if ((rc = batch_items<R>(plans, which, b, s)) != CM_OK) break;
      if ((rc = capture()) != CM_OK) break;
      built = running;
    }
  }
  if (ge) cudaGraphExecDestroy(ge);
  return rc;
}

// One phase of a lockstep batch in precision R: every solve's initial
// state, working heights (with the default pentol), initial field and
// operator are set up by a few launches over the batch's work lists (not a
// sequence per solve), then the loop runs, then (final) the result fields;
// `out` receives the solves' states.  from_fp32: warm start from the FP32
// phase's forces (the FP64 phase of mixed solves), else from u0.
template <typename R>
static int lockstep_phase(int n, cm_plan* const* plans, const cm_ccg_params* params,
                          const double* const* h, const double* const* u0, double* const* x,
                          double* const* jac, unsigned char* const* active,
                          unsigned char* const* plastic, bool from_fp32, double rel_pentol,
                          double rel_forcetol, const std::vector<int>& maxiters, bool final,
                          bool bisect, int maxiter_all, double timeout, cudaStream_t s, int* polls,
                          std::vector<CcgState>& out) {
  NvtxRange range(sizeof(R) == 8 ? "batch phase fp64" : "batch phase fp32");
  set_smem_attrs<R>();
  for (int i = 0; i < n; ++i) CKS(ensure_ccg(plans[i], work_of<R>(plans[i])));
  BatchDev<R> b;
  CKS(batch_build<R>(n, plans, b, s, [&](int i, Slot<R>& sl) {
    cm_plan* p = plans[i];
    sl.h64 = h[i];
    sl.u0 = (!from_fp32 && u0) ? u0[i] : nullptr;
    sl.prev_f[0] = p->w32.f[0];
    sl.prev_f[1] = p->w32.f[1];
    sl.prev_st = p->w32.st;
    sl.x_out = x ? x[i] : nullptr;
    sl.jac_out = jac ? jac[i] : nullptr;
    sl.act_out = active ? active[i] : nullptr;
    sl.pl_out = plastic ? plastic[i] : nullptr;
    // the set-up's operator: f = K u from u0, or u = G f from the FP32 forces
    if (!from_fp32) {
      sl.in = sl.u; sl.in_rows = p->nx; sl.in_cols = p->ny; sl.in_ld = p->ny;
      sl.out = sl.f[0]; sl.out_rows = p->tx; sl.out_cols = p->ty; sl.out_ld = p->ty;
      sl.table_sel = 1;
    } else {
      sl.in = sl.f[0]; sl.in_rows = p->tx; sl.in_cols = p->ty; sl.in_ld = p->ty;
      sl.out = sl.u; sl.out_rows = p->nx; sl.out_cols = p->ny; sl.out_ld = p->ny;
      sl.table_sel = 0;
    }
  }));
  // initial states through one pinned staging copy
  CcgState* hst = nullptr;
  if (cudaMallocHost(&hst, sizeof(CcgState) * n) != cudaSuccess) {
    cudaGetLastError();
    return CM_ERR_OOM;
  }
  for (int i = 0; i < n; ++i) initial_state(plans[i], &params[i], rel_forcetol, maxiters[i], hst[i]);
  CcgState* dst = nullptr;
  int rc = CM_OK;
  if (cudaMalloc(&dst, sizeof(CcgState) * n) != cudaSuccess) { cudaGetLastError(); rc = CM_ERR_OOM; }
  else b.allocs.push_back(dst);
  if (rc == CM_OK && cudaMemcpyAsync(dst, hst, sizeof(CcgState) * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
    rc = CM_ERR_CUDA;
  if (rc == CM_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = CM_ERR_CUDA;
  cudaFreeHost(hst);
  CKS(rc);
  const int TT = g_batch_threads[sizeof(R) == 8 ? 0 : 1];
  const Slot<R>* S = b.slots;
  k_put_states<R><<<std::min(n, 1024), 128, 0, s>>>(S, dst, n);
  k_h_prep<R><<<b.n_items[0], CM_THREADS, 0, s>>>(S, b.items[0], nullptr);
  k_h_var<R><<<b.n_items[0], CM_THREADS, 0, s>>>(S, b.items[0], nullptr, -1, rel_pentol);
  if (!from_fp32) {
    k_init_u_rows<R><<<b.n_items[2], 256, 0, s>>>(S, b.items[2]);
    k_row_fwd<R, MODE_PLAIN><<<b.n_items[2], TT, b.smem_row, s>>>(S, b.items[2]);
    k_col<R, MODE_PLAIN><<<b.n_items[3], TT, b.smem_col, s>>>(S, b.items[3]);
    k_row_inv<R, MODE_PLAIN><<<b.n_items[1], TT, b.smem_row, s>>>(S, b.items[1]);
  } else {
    k_init_f_prev<R><<<b.n_items[0], 256, 0, s>>>(S, b.items[0]);
    k_row_fwd<R, MODE_PLAIN><<<b.n_items[1], TT, b.smem_row, s>>>(S, b.items[1]);
    k_col<R, MODE_PLAIN><<<b.n_items[3], TT, b.smem_col, s>>>(S, b.items[3]);
    k_row_inv<R, MODE_PLAIN><<<b.n_items[2], TT, b.smem_row, s>>>(S, b.items[2]);
  }
  g_launches += 7;
  CK(cudaGetLastError());
  CKS(batch_loop<R>(n, plans, b, bisect, maxiter_all, timeout, s, polls));
  if (final) {
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    CKS(batch_items<R>(plans, all, b, s));  // the loop kept only the last running solves
    k_ccg_result_slots<R><<<b.n_items[0], CM_THREADS, 0, s>>>(S, b.items[0]);
    k_x_rows<R><<<b.n_items[2], 256, 0, s>>>(S, b.items[2]);
    g_launches += 2;
    CK(cudaGetLastError());
  }
  return read_states<R>(n, plans, out, s);
}

static int status_error(const CcgState& st) {
  if (st.status == CMS_NAN) return CM_ERR_NAN;
  if (st.status == CMS_BISECT_SIGN) return CM_ERR_BISECT;
  if (st.status == CMS_BISECT_SIGN + 1) return CM_ERR_BISECT_CONV;
  if (st.status == CMS_TIMEOUT) return CM_ERR_TIMEOUT;
  return CM_OK;
}

// ---------------------------------------------------------------------------
// stepping interface (continuous batching)
// ---------------------------------------------------------------------------
// Reusable device and pinned host buffers of a stepper: slot descriptors and
// work lists of the solves advanced together in one step.
struct cm_stepper {
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  size_t cap_slots = 0, cap_items = 0;
  void* d_slots = nullptr;       // Slot<float> or Slot<double> array
  int2* d_items[4] = {nullptr, nullptr, nullptr, nullptr};
  int* d_done = nullptr;
  void* h_slots = nullptr;       // pinned staging
  int2* h_items = nullptr;
  int* h_done = nullptr;
  size_t cap_h_items = 0;
};

static void stepper_free(cm_stepper* st) {
  cudaFree(st->d_slots);
  for (int k = 0; k < 4; ++k) cudaFree(st->d_items[k]);
  cudaFree(st->d_done);
  cudaFreeHost(st->h_slots);
  cudaFreeHost(st->h_items);
  cudaFreeHost(st->h_done);
  st->d_slots = nullptr;
  for (int k = 0; k < 4; ++k) st->d_items[k] = nullptr;
  st->d_done = nullptr;
  st->h_slots = nullptr;
  st->h_items = nullptr;
  st->h_done = nullptr;
  st->cap_slots = st->cap_items = st->cap_h_items = 0;
}

// grow the buffers to n slots (of the larger slot type) and `items` entries per list
static int stepper_reserve(cm_stepper* st, size_t n, size_t items) {
  if (n <= st->cap_slots && items <= st->cap_items) return CM_OK;
  CK(cudaStreamSynchronize(st->stream));
  const size_t ns = std::max(n, st->cap_slots * 2), ni = std::max(items, st->cap_items * 2);
  stepper_free(st);
  const size_t slot_bytes = std::max(sizeof(Slot<float>), sizeof(Slot<double>));
  if (cudaMalloc(&st->d_slots, slot_bytes * ns) != cudaSuccess) { cudaGetLastError(); return CM_ERR_OOM; }
  for (int k = 0; k < 4; ++k)
    if (cudaMalloc(&st->d_items[k], sizeof(int2) * ni) != cudaSuccess) { cudaGetLastError(); return CM_ERR_OOM; }
  if (cudaMalloc(&st->d_done, sizeof(int) * ns) != cudaSuccess) { cudaGetLastError(); return CM_ERR_OOM; }
  if (cudaMallocHost(&st->h_slots, slot_bytes * ns) != cudaSuccess) { cudaGetLastError(); return CM_ERR_OOM; }
  if (cudaMallocHost(&st->h_items, sizeof(int2) * ni * 4) != cudaSuccess) { cudaGetLastError(); return CM_ERR_OOM; }
  if (cudaMallocHost(&st->h_done, sizeof(int) * ns) != cudaSuccess) { cudaGetLastError(); return CM_ERR_OOM; }
  st->cap_slots = ns;
  st->cap_items = ni;
  return CM_OK;
}

template <typename R>
__global__ void k_collect_done(const Slot<R>* __restrict__ slots, int n, int* done) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    done[i] = slots[i].st->done;
}

// Advance the solves of one precision by `iters` iterations; done flags to h_done[off..].
template <typename R>
static int stepper_run(cm_stepper* stp, const std::vector<cm_plan*>& plans, int iters, int* done_out) {
  const int n = (int)plans.size();
  if (n == 0) return CM_OK;
  cudaStream_t s = stp->stream;
  set_smem_attrs<R>();
  size_t ni[4] = {0, 0, 0, 0};
  bool bisect = false;
  for (cm_plan* p : plans) {
    Work<R>& w = work_of<R>(p);
    ni[0] += w.nt_comp; ni[1] += w.nt_rowt; ni[2] += w.nt_rowd; ni[3] += w.nt_col;
    bisect = bisect || (p->params.has_hardness && p->params.load_control);
  }
  CKS(stepper_reserve(stp, n, std::max({ni[0], ni[1], ni[2], ni[3], (size_t)1})));
  Slot<R>* hs = (Slot<R>*)stp->h_slots;
  int2* hi[4];
  for (int k = 0; k < 4; ++k) hi[k] = stp->h_items + k * stp->cap_items;
  size_t c[4] = {0, 0, 0, 0};
  BatchDev<R> b;  // views into the stepper's buffers (owns nothing)
  for (int i = 0; i < n; ++i) {
    Work<R>& w = work_of<R>(plans[i]);
    hs[i] = base_slot(plans[i], w);
    for (int t = 0; t < hs[i].nt_comp; ++t) hi[0][c[0]++] = make_int2(i, t);
    for (int t = 0; t < hs[i].nt_rowt; ++t) hi[1][c[1]++] = make_int2(i, t);
    for (int t = 0; t < hs[i].nt_rowd; ++t) hi[2][c[2]++] = make_int2(i, t);
    for (int t = 0; t < hs[i].nt_col; ++t) hi[3][c[3]++] = make_int2(i, t);
    b.smem_row = std::max(b.smem_row, w.tiles.smem_row);
    b.smem_col = std::max(b.smem_col, w.tiles.smem_col);
  }
  CK(cudaMemcpyAsync(stp->d_slots, hs, sizeof(Slot<R>) * n, cudaMemcpyHostToDevice, s));
  for (int k = 0; k < 4; ++k) {
    CK(cudaMemcpyAsync(stp->d_items[k], hi[k], sizeof(int2) * c[k], cudaMemcpyHostToDevice, s));
    b.items[k] = stp->d_items[k];
    b.n_items[k] = (int)c[k];
  }
  b.slots = (Slot<R>*)stp->d_slots;
  for (int it = 0; it < iters; ++it) launch_iteration_batch<R>(b, bisect, s);
  g_launches += (unsigned long long)iters * iteration_launches(bisect, false) + 1;
  k_collect_done<R><<<grid_for(n), 256, 0, s>>>(b.slots, n, stp->d_done);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(stp->h_done, stp->d_done, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int i = 0; i < n; ++i) done_out[i] = stp->h_done[i];
  b.slots = nullptr;
  for (int k = 0; k < 4; ++k) b.items[k] = nullptr;
  return CM_OK;
}

// ---------------------------------------------------------------------------
// k-space operators on half spectra of the reference's layout
// ---------------------------------------------------------------------------
// out[kx][ky] (kx <= nx/2, ky < ny) of the reference's half spectrum, halved
// along x, from the library's spectrum halved along y (column tiles of
// width 2^lw): the mirror (-kx, -ky) holds the conjugate of a real field's
// transform for ky > ny/2.
__global__ void k_spec_to_ref(const double2* __restrict__ spec, double2* __restrict__ out, int nx,
                              int ny, int lw) {
  const int nxh = nx / 2 + 1, nyh = ny / 2 + 1;
  const long n = (long)nxh * ny;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int kx = (int)(i / ny), ky = (int)(i % ny);
    double2 v;
    if (ky < nyh) {
      v = spec[spec_at(kx, ky, nx, lw)];
    } else {
      v = spec[spec_at((nx - kx) % nx, ny - ky, nx, lw)];
      v.y = -v.y;
    }
    out[i] = v;
  }
}

// k_out = scale T k_in, T = G (op 0) or 1/G (op 1, 0 where G = 0); G is the
// natural (nx, nyh) table, even in kx and ky
__global__ void k_kspace_apply(const double* __restrict__ G, const double2* k_in, double2* k_out,
                               int nx, int ny, int op, double scale) {
  const int nxh = nx / 2 + 1, nyh = ny / 2 + 1;
  const long n = (long)nxh * ny;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int kx = (int)(i / ny), ky = (int)(i % ny);
    const double g = G[(size_t)kx * nyh + min(ky, ny - ky)];
    const double t = op == CM_OP_DISP ? g : (g != 0.0 ? 1.0 / g : 0.0);
    double2 v = k_in[i];
    v.x *= scale * t;
    v.y *= scale * t;
    k_out[i] = v;
  }
}

// per-block partial sums of w_kx Re(conj(a) b) over the reference half spectrum
__global__ void __launch_bounds__(256) k_kspace_dot(const double2* __restrict__ a,
                                                    const double2* __restrict__ b, int nx, int ny,
                                                    double* partial) {
  const int nxh = nx / 2 + 1;
  const long n = (long)nxh * ny;
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int kx = (int)(i / ny);
    const double w = (kx == 0 || (nx % 2 == 0 && 2 * kx == nx)) ? 1.0 : 2.0;
    const double2 u = a[i], v = b[i];
    acc += w * (u.x * v.x + u.y * v.y);
  }
  __shared__ double sm[256];
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) sm[threadIdx.x] += sm[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

// ---------------------------------------------------------------------------
// self-test of the bounded grid barrier
// ---------------------------------------------------------------------------
// Every block meets at one grid barrier (cm_kernels.cuh: grid_barrier) with a
// wait limit of `limit` SM clock cycles; blocks whose wait gave up are counted.
__global__ void __launch_bounds__(128) k_selftest_barrier(GridBarrier* bar, long long limit,
                                                          int* gave_up) {
  __shared__ int ok_sm;
  unsigned gen = 0;
  if (threadIdx.x == 0) gen = ld_acquire_gpu(&bar->gen);
  const bool ok = grid_barrier(bar, gen, &ok_sm, limit);
  if (threadIdx.x == 0 && !ok) atomicAdd(gave_up, 1);
}

// ---------------------------------------------------------------------------
// periodic operator that allocates nothing
// ---------------------------------------------------------------------------
// Scratch of cm_apply_periodic_noalloc: a fixed 4 MiB array in the library's
// own device memory (every GPU that loads the library holds it until exit).
// It fits a periodic grid of up to 512 x 512 points.  Layout, in order:
// slot descriptor, work list, twiddles (x then y), tiled Green's table,
// spectrum.  Every call rewrites each part it reads, so nothing has to start
// at zero; calls that overlap on the GPU (two streams, or two host threads)
// share the array and race.
#define CM_NOALLOC_MAX_SIDE 512
#define CM_NOALLOC_BYTES (4u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[CM_NOALLOC_BYTES];

// Device address of the scratch on the current device.  Looked up on every
// call (cudaGetSymbolAddress allocates nothing and is cheap), so an address
// never outlives the context it was taken in (cudaDeviceReset, a primary
// context released and created again).  The first lookup on a device may
// load the library's module there, which is why the first call should come
// before any stream capture.
static int noalloc_scratch(unsigned char** out) {
  void* ptr = nullptr;
  CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
  *out = (unsigned char*)ptr;
  return CM_OK;
}

__global__ void k_noalloc_setup(Slot<double>* slot, Slot<double> sv, int2* items, int nitems,
                                double2* twx, int nx, double2* twy, int ny) {
  const long stride = (long)gridDim.x * blockDim.x;
  const long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i0 == 0) *slot = sv;
  for (long i = i0; i < nitems; i += stride) items[i] = make_int2(0, (int)i);
  for (long i = i0; i < nx; i += stride) {
    double sn, cs;
    sincospi(-2.0 * (double)i / (double)nx, &sn, &cs);
    twx[i] = make_double2(cs, sn);
  }
  for (long i = i0; i < ny; i += stride) {
    double sn, cs;
    sincospi(-2.0 * (double)i / (double)ny, &sn, &cs);
    twy[i] = make_double2(cs, sn);
  }
}

// one scaled operator table (-G/(aN) or -K a/N) in the tiled spectrum layout
__global__ void k_noalloc_table(const double* G, double* tab, int nx, int nyh, int lw, int op,
                                double aN_inv, double a_over_N) {
  const long n = (long)nx * nyh;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i / nyh), k = (int)(i % nyh);
    const double g = G[i];
    const double v = (op == CM_OP_DISP) ? -g * aN_inv : -((g != 0.0) ? 1.0 / g : 0.0) * a_over_N;
    tab[spec_at(x, k, nx, lw)] = v;
  }
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* cm_version(void) { return "cm_b200 0.1 (sm_100a)"; }

const char* cm_status_string(int status) {
  switch (status) {
    case CM_OK: return "ok";
    case CM_ERR_ARG: return "invalid argument";
    case CM_ERR_SHAPE: return "array shape mismatch";
    case CM_ERR_SIZE: return "grid too large for the single-pass transforms";
    case CM_ERR_CUDA: {
      static thread_local char buf[256];
      snprintf(buf, sizeof(buf), "CUDA error: %s", cudaGetErrorString(last_cuda_error()));
      return buf;
    }
    case CM_ERR_OOM: return "device allocation failed";
    case CM_ERR_NAN: return "nan encountered.";
    case CM_ERR_BISECT: return "f(a) and f(b) must have different signs";
    case CM_ERR_BISECT_CONV: return "Failed to converge after 100 iterations";
    case CM_ERR_TIMEOUT: return "solve exceeded its time budget";
    case CM_ERR_STOPPED: return "stopped by the per-iteration observer";
    default: return "unknown status";
  }
}

int cm_plan_create(const cm_plan_desc* desc, void* stream, cm_plan** out) {
  NvtxRange range("cm_plan_create");
  if (!desc || !out) return CM_ERR_ARG;
  *out = nullptr;
  if (desc->kind != CM_PERIODIC && desc->kind != CM_FREE && desc->kind != CM_SEMI) return CM_ERR_ARG;
  if (desc->dim != 1 && desc->dim != 2) return CM_ERR_ARG;
  if (desc->nx < 1 || desc->ny < 1 || (desc->dim == 1 && desc->ny != 1)) return CM_ERR_ARG;
  if (desc->kind != CM_PERIODIC && desc->dim != 2) return CM_ERR_ARG;
  if (desc->kind == CM_SEMI && (desc->n_images < 0 || desc->n_images > 10000)) return CM_ERR_ARG;
  if (!(desc->sx > 0) || !(desc->sy > 0)) return CM_ERR_ARG;
  cm_plan* p = new (std::nothrow) cm_plan();
  if (!p) return CM_ERR_OOM;
  p->d = *desc;
  p->tx = desc->nx;
  p->ty = desc->ny;
  if (desc->kind == CM_SEMI) {
    // a periodic axis keeps its points, a free one is padded to 2n - 1
    // (FFTElasticHalfSpace.py:1343-1353)
    p->nx = desc->periodic_x ? desc->nx : 2 * desc->nx - 1;
    p->ny = desc->periodic_y ? desc->ny : 2 * desc->ny - 1;
  } else {
    const int f = desc->kind == CM_FREE ? 2 : 1;
    p->nx = f * desc->nx;
    p->ny = f * desc->ny;
  }
  p->nyh = p->ny / 2 + 1;
  int rc = CM_OK;
  auto fail = [&](int code) {
    cm_plan_destroy(p);
    return code;
  };
  if (!make_fft_desc(p->nx, &p->fx) || !make_fft_desc(p->ny, &p->fy)) return fail(CM_ERR_SIZE);
  if (stream) {
    p->stream = (cudaStream_t)stream;
    p->own_stream = false;
  } else {
    // non-blocking: no implicit ordering with the legacy default stream, so
    // another thread's stream capture is never joined by this plan's work
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(CM_ERR_CUDA);
    p->own_stream = true;
  }
  if (cudaMallocHost(&p->h_state, 3 * sizeof(CcgState)) != cudaSuccess) {
    p->h_state = nullptr;
    return fail(CM_ERR_OOM);
  }
  if ((rc = init_work<double>(p, p->w64)) != CM_OK) return fail(rc);
  if ((rc = init_work<float>(p, p->w32)) != CM_OK) return fail(rc);
  // work items (0, i): every launch on this plan covers tiles 0..n-1 of slot 0
  {
    std::vector<int2> it(p->max_items);
    for (int i = 0; i < p->max_items; ++i) it[i] = make_int2(0, i);
    if ((rc = dalloc(p, &p->items, it.size())) != CM_OK) return fail(rc);
    if (cudaMemcpyAsync(p->items, it.data(), it.size() * sizeof(int2), cudaMemcpyHostToDevice,
                        p->stream) != cudaSuccess)
      return fail(CM_ERR_CUDA);
  }
  const long nh = (long)p->nx * p->nyh;
  const long nh64 = (long)p->nx * p->w64.tiles.ntile_cols * p->w64.tiles.col_tile;
  const long nh32 = (long)p->nx * p->w32.tiles.ntile_cols * p->w32.tiles.col_tile;
  if ((rc = dalloc(p, &p->G, nh)) != CM_OK) return fail(rc);
  for (int i = 0; i < 2; ++i) {
    if ((rc = dalloc(p, &p->tab64[i], nh64)) != CM_OK) return fail(rc);
    if ((rc = dalloc(p, &p->tab32[i], nh32)) != CM_OK) return fail(rc);
    cudaMemsetAsync(p->tab64[i], 0, nh64 * sizeof(double), p->stream);
    cudaMemsetAsync(p->tab32[i], 0, nh32 * sizeof(float), p->stream);
  }
  p->w64.tab[0] = p->tab64[0];
  p->w64.tab[1] = p->tab64[1];
  p->w32.tab[0] = p->tab32[0];
  p->w32.tab[1] = p->tab32[1];
  cudaStream_t s = p->stream;
  if (desc->kind == CM_PERIODIC) {
    const double Es = desc->young / (1 - desc->poisson * desc->poisson);
    k_table_periodic<<<grid_for(nh), 256, 0, s>>>(p->G, p->nx, p->ny, p->nyh, desc->sx, desc->sy, Es,
                                                   desc->young, desc->poisson, desc->q0_mode,
                                                   desc->stiffness_q0, desc->thickness, desc->dim);
  } else {
    double *love = nullptr, *quad = nullptr;
    if ((rc = dalloc(p, &love, (long)p->nx * p->ny)) != CM_OK) return fail(rc);
    // the kernel at every absolute offset the domain holds (the free
    // domain's offsets reach the topography's size, wrapped at i > nx), summed
    // over the periodic images of a semi-periodic substrate
    LoveKey key{};
    key.qx = p->nx / 2 + 1;
    key.qy = p->ny / 2 + 1;
    key.dx = desc->sx / p->tx;
    key.dy = desc->sy / p->ty;
    key.young = desc->young;
    key.Lx = desc->sx;
    key.Ly = desc->sy;
    const bool semi = desc->kind == CM_SEMI;
    key.nimx = semi && desc->periodic_x ? desc->n_images : 0;
    key.nimy = semi && desc->periodic_y ? desc->n_images : 0;
    const auto hq = love_quadrant(key);
    if ((rc = dalloc(p, &quad, (long)hq->size())) != CM_OK) return fail(rc);
    if (cudaMemcpyAsync(quad, hq->data(), hq->size() * sizeof(double), cudaMemcpyHostToDevice, s) !=
        cudaSuccess)
      return fail(CM_ERR_CUDA);
    k_love_expand<<<grid_for((long)p->nx * p->ny), 256, 0, s>>>(love, quad, key.qy, p->nx, p->ny);
    // its transform: the power-of-two passes where the domain has them, else
    // the per-pass kernels
    rc = forward_real_p2(p, love, p->G, s);
    if (rc < 0) {
      rc = launch_plain<double>(p, p->w64, MODE_FWD, 0, love, p->nx, p->ny, p->ny, nullptr, 0,
                                0, 0, s);
      if (rc != CM_OK) return fail(rc);
      k_real_part<<<grid_for(nh), 256, 0, s>>>(p->w64.spec, p->G, p->nx, p->nyh, p->w64.tiles.lw);
    } else if (rc != CM_OK) {
      return fail(rc);
    }
  }
  const double area = (desc->sx / p->tx) * (desc->sy / p->ty);
  const double N = (double)p->nx * (double)p->ny;
  k_tables_scale<<<grid_for(nh), 256, 0, s>>>(p->G, p->nx, p->nyh, 1.0 / (area * N), area / N,
                                               p->tab64[0], p->tab64[1], p->w64.tiles.lw, p->tab32[0],
                                               p->tab32[1], p->w32.tiles.lw);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
    return fail(CM_ERR_CUDA);
  *out = p;
  return CM_OK;
}

int cm_plan_destroy(cm_plan* p) {
  if (!p) return CM_OK;
  if (p->stream) cudaStreamSynchronize(p->stream);
  for (int i = 0; i < 2; ++i) {
    if (p->w32.graph[i]) cudaGraphExecDestroy(p->w32.graph[i]);
    if (p->w64.graph[i]) cudaGraphExecDestroy(p->w64.graph[i]);
  }
  for (void* a : p->allocs) cudaFree(a);
  if (p->h_state) cudaFreeHost(p->h_state);
  if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
  delete p;
  return CM_OK;
}

int cm_plan_shape(const cm_plan* p, int* nxd, int* nyd, int* nyh) {
  if (!p) return CM_ERR_ARG;
  if (nxd) *nxd = p->nx;
  if (nyd) *nyd = p->ny;
  if (nyh) *nyh = p->nyh;
  return CM_OK;
}

int cm_plan_engine(const cm_plan* p, int precision, int* engine) {
  if (!p || !engine || (precision != CM_FP64 && precision != CM_FP32)) return CM_ERR_ARG;
  const int lx = len_code(p->nx), ly = len_code(p->ny);
  const bool ok = lx > 0 && ly > 0 &&
                  (precision == CM_FP64 ? op_p2_supported<double>(lx, ly, p->w64.tiles.lw)
                                        : op_p2_supported<float>(lx, ly, p->w32.tiles.lw));
  *engine = ok ? 1 : 0;
  return CM_OK;
}

int cm_plan_greens_host(cm_plan* p, double* out) {
  if (!p || !out) return CM_ERR_ARG;
  CK(cudaMemcpyAsync(out, p->G, sizeof(double) * (size_t)p->nx * p->nyh, cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return CM_OK;
}

int cm_apply(cm_plan* p, int op, int precision, const void* in, int in_rows, int in_cols, int in_ld,
             void* out, int out_rows, int out_cols, int out_ld, void* stream) {
  NvtxRange range("cm_apply");
  if (!p || !in || !out) return CM_ERR_ARG;
  if (op != CM_OP_DISP && op != CM_OP_FORCE) return CM_ERR_ARG;
  if (precision != CM_FP64 && precision != CM_FP32) return CM_ERR_ARG;
  if (in_rows < 1 || in_rows > p->nx || in_cols < 1 || in_cols > p->ny || in_ld < in_cols) return CM_ERR_SHAPE;
  if (out_rows < 1 || out_rows > p->nx || out_cols < 1 || out_cols > p->ny || out_ld < out_cols)
    return CM_ERR_SHAPE;
  cudaStream_t s = stream ? (cudaStream_t)stream : p->stream;
  return apply_dispatch(p, op, precision, in, in_rows, in_cols, in_ld, out, out_rows, out_cols, out_ld, s);
}

int cm_ccg_solve(cm_plan* p, const cm_ccg_params* prm, const double* h, const double* u0,
                 const double* f0, double* x, double* jac, unsigned char* active,
                 unsigned char* plastic, cm_ccg_result* res) {
  NvtxRange range("cm_ccg_solve");
  if (!p || !prm || !h || !res) return CM_ERR_ARG;
  if (prm->precision != CM_FP64 && prm->precision != CM_FP32 && prm->precision != CM_MIXED) return CM_ERR_ARG;
  if (prm->maxiter < 1) return CM_ERR_ARG;
  if (prm->has_hardness && !(prm->hardness > 0)) return CM_ERR_ARG;
  memset(res, 0, sizeof(*res));
  SolveInput in{h, u0, f0, p->ny};
  CcgState fin;
  g_polls = 0;
  typedef std::chrono::steady_clock clk;
  const auto t0 = clk::now();
  auto ms_since = [](clk::time_point a) {
    return std::chrono::duration<double, std::milli>(clk::now() - a).count();
  };
  p->obs_it_offset = 0;
  if (prm->precision == CM_FP64) {
    CKS(run_ccg<double>(p, p->w64, prm, in, 0.0, 0.0, prm->maxiter, &fin));
    CKS(finish_ccg<double>(p, p->w64, x, jac, active, plastic, &fin));
    fill_result(fin, res);
    res->ms_fp64 = res->ms_total = ms_since(t0);
    res->polls = g_polls;
    return CM_OK;
  }
  const double rp = prm->precision == CM_MIXED ? (prm->fp32_pentol_rel > 0 ? prm->fp32_pentol_rel : 2e-6) : 0.0;
  const double rf = prm->precision == CM_MIXED ? 1e-5 : 0.0;
  // FP32 phase: tolerances widened to FP32 resolution; a phase that cannot
  // reach them within its iteration cap hands over to the FP64 refinement
  const int cap32 = prm->precision == CM_MIXED ? fp32_cap(prm->maxiter, prm->has_hardness) : prm->maxiter;
  // the FP32 phase of a mixed solve leaves the padding's displacement alone:
  // the refinement recomputes u = G f on the whole domain from its forces
  CKS(run_ccg<float>(p, p->w32, prm, in, rp, rf, cap32, &fin, 0, nullptr,
                     prm->precision == CM_MIXED));
  const double ms32 = ms_since(t0);
  if (prm->precision == CM_FP32) {
    CKS(finish_ccg<float>(p, p->w32, x, jac, active, plastic, &fin));
    fill_result(fin, res);
    res->nit_fp32 = fin.it;
    res->ms_fp32 = res->ms_total = ms_since(t0);
    res->polls = g_polls;
    return CM_OK;
  }
  const auto t1 = clk::now();
  // FP64 refinement warm-started from the FP32 forces (initial_forces semantics)
  const int nit32 = fin.it, nfev32 = fin.nfev;
  double* f64 = nullptr;
  {
    // the FP64 solver's f[1] buffer is free before the refinement starts
    CKS(ensure_ccg(p, p->w64));
    f64 = p->w64.u;  // borrow: overwritten by the refinement's own initialisation
  }
  k_force_to_domain<float><<<grid_for((long)p->nx * p->ny), 256, 0, p->stream>>>(
      p->w32.st, p->w32.f[0], p->w32.f[1], p->tx, p->ty, f64, p->nx, p->ny);
  CK(cudaGetLastError());
  // k_init_f reads f64 before the operator overwrites u, so the borrow is safe
  SolveInput in2{h, nullptr, f64, p->ny};
  const int rem = std::max(1, prm->maxiter - nit32);
  // A refinement that has not converged within its budget starts again
  // cold from the caller's own start, i.e. becomes the FP64 solve (seen on a
  // plastic request whose FP32 phase stopped at its cap: the refinement from
  // those forces ran to maxiter, the cold FP64 solve converged in 169).
  const int budget = std::min(rem, std::max(CM_REFINE_MIN_ITERS, CM_REFINE_PER_FP32_ITER * nit32));
  p->obs_it_offset = nit32;
  CKS(run_ccg<double>(p, p->w64, prm, in2, 0.0, 0.0, budget, &fin));
  int nit_refine = 0;
  if (fin.status != CMS_CONVERGED && budget < rem) {
    nit_refine = fin.it;
    p->obs_it_offset = nit32 + nit_refine;
    CKS(run_ccg<double>(p, p->w64, prm, in, 0.0, 0.0, rem - nit_refine, &fin));
  }
  CKS(finish_ccg<double>(p, p->w64, x, jac, active, plastic, &fin));
  fill_result(fin, res);
  res->nit += nit32 + nit_refine;
  res->nfev += nfev32;
  res->nit_fp32 = nit32;
  res->ms_fp32 = ms32;
  res->ms_fp64 = ms_since(t1);
  res->ms_total = ms_since(t0);
  res->polls = g_polls;
  return CM_OK;
}

// Shared memory of the per-pass bodies on a plan's tiles: twiddles plus two
// buffers of a row tile or of a column tile, whichever is larger.
static size_t pass_smem(const cm_plan* p, const Tiles& t, size_t csize) {
  const size_t r = (2 * (size_t)(t.row_tile / 2) * p->ny + p->ny) * csize;
  const size_t c = (2 * (size_t)t.col_tile * p->nx + p->nx) * csize;
  return std::max(r, c);
}

// Whether a batch runs in the persistent kernel: elastic solves (no
// plastic bisection) without a wall-clock timeout whose passes fit.
static bool batch_persistent_ok(int n, cm_plan* const* plans, const cm_ccg_params* params,
                                int prec) {
  if (!g_batch_persistent.load()) return false;
  for (int i = 0; i < n; ++i) {
    if (params[i].has_hardness || params[i].timeout_s > 0) return false;
    if (prec != CM_FP64 && !plans[i]->w32.tiles.generic_ok) return false;
    if (prec != CM_FP32 && !plans[i]->w64.tiles.generic_ok) return false;
  }
  return true;
}

// The whole batch in one launch of the persistent kernel: FP32 phase, FP64
// refinement and result fields of every solve.
static int batch_persistent(int n, cm_plan* const* plans, const cm_ccg_params* params,
                            const double* const* h, const double* const* u0, double* const* x,
                            double* const* jac, unsigned char* const* active,
                            unsigned char* const* plastic, cm_ccg_result* res, cudaStream_t s) {
  NvtxRange range("batch persistent kernel");
  typedef std::chrono::steady_clock clk;
  const auto t0 = clk::now();
  const int prec = params[0].precision;
  const bool use32 = prec != CM_FP64, use64 = prec != CM_FP32;
  size_t smem = 0;
  for (int i = 0; i < n; ++i) {
    cm_plan* p = plans[i];
    if (use32) {
      CKS(ensure_ccg(p, p->w32));
      smem = std::max(smem, pass_smem(p, p->w32.tiles, sizeof(float2)));
    }
    if (use64) {
      CKS(ensure_ccg(p, p->w64));
      smem = std::max(smem, pass_smem(p, p->w64.tiles, sizeof(double2)));
    }
  }
  if (smem > CM_SMEM_DYN_MAX) return CM_ERR_SIZE;
  const size_t jb = sizeof(BatchJob) * (size_t)n, ob = sizeof(int) * (size_t)(n + 1);
  unsigned char* hbuf = nullptr;
  if (cudaMallocHost(&hbuf, jb + ob) != cudaSuccess) {
    cudaGetLastError();
    return CM_ERR_OOM;
  }
  BatchJob* hj = reinterpret_cast<BatchJob*>(hbuf);
  int* ho = reinterpret_cast<int*>(hbuf + jb);
  for (int i = 0; i < n; ++i) {
    cm_plan* p = plans[i];
    const cm_ccg_params& P = params[i];
    BatchJob& J = hj[i];
    memset(&J, 0, sizeof(J));
    if (use32) {
      J.s32 = base_slot(p, p->w32);
      const int mi = prec == CM_MIXED ? fp32_cap(P.maxiter, false) : P.maxiter;
      initial_state(p, &P, prec == CM_MIXED ? 1e-5 : 0.0, mi, J.init32);
    }
    if (use64) {
      J.s64 = base_slot(p, p->w64);
      initial_state(p, &P, 0.0, P.maxiter, J.init64);
    }
    J.h64 = h[i];
    J.u0 = u0 ? u0[i] : nullptr;
    J.x = x ? x[i] : nullptr;
    J.jac = jac ? jac[i] : nullptr;
    J.active = active ? active[i] : nullptr;
    J.plastic = plastic ? plastic[i] : nullptr;
    J.prec = prec;
    J.pentol_auto = P.pentol <= 0;
    J.maxiter = P.maxiter;
    J.rel_pentol32 = prec == CM_MIXED ? (P.fp32_pentol_rel > 0 ? P.fp32_pentol_rel : 2e-6) : 0.0;
    ho[i] = i;
  }
  // largest grids first: the last solves to start are the shortest
  std::stable_sort(ho, ho + n, [&](int a, int b) {
    return (long)plans[a]->nx * plans[a]->ny > (long)plans[b]->nx * plans[b]->ny;
  });
  ho[n] = 0;  // the queue counter
  unsigned char* dbuf = nullptr;
  int rc = CM_OK;
  if (cudaMalloc(&dbuf, jb + ob) != cudaSuccess) {
    cudaGetLastError();
    rc = CM_ERR_OOM;
  }
  int clusters = 0;
  if (rc == CM_OK && cudaMemcpyAsync(dbuf, hbuf, jb + ob, cudaMemcpyHostToDevice, s) != cudaSuccess)
    rc = CM_ERR_CUDA;
  if (rc == CM_OK) {
    int* d_order = reinterpret_cast<int*>(dbuf + jb);
    if (batch_solve_launch(reinterpret_cast<const BatchJob*>(dbuf), d_order, n, d_order + n, smem,
                           s, &clusters) != 0)
      rc = CM_ERR_CUDA;
    else
      g_launches += 1;
  }
  std::vector<CcgState> st32, st64;
  if (rc == CM_OK && use32) rc = read_states<float>(n, plans, st32, s);
  if (rc == CM_OK && use64) rc = read_states<double>(n, plans, st64, s);
  if (rc != CM_OK) cudaStreamSynchronize(s);  // nothing may still read the buffers
  cudaFree(dbuf);
  cudaFreeHost(hbuf);
  CKS(rc);
  const double ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  for (int i = 0; i < n; ++i) {
    if (use32) CKS(status_error(st32[i]));
    const CcgState& fin = use64 ? st64[i] : st32[i];
    CKS(status_error(fin));
    fill_result(fin, &res[i]);
    if (prec == CM_MIXED) {
      res[i].nit += st32[i].it;
      res[i].nfev += st32[i].nfev;
      res[i].nit_fp32 = st32[i].it;
    } else if (prec == CM_FP32) {
      res[i].nit_fp32 = st32[i].it;
    }
    res[i].ms_total = ms;
    res[i].polls = 1;
  }
  return CM_OK;
}

int cm_ccg_solve_batch(int n, cm_plan* const* plans, const cm_ccg_params* params,
                       const double* const* h, const double* const* u0, double* const* x,
                       double* const* jac, unsigned char* const* active,
                       unsigned char* const* plastic, cm_ccg_result* res, void* stream) {
  NvtxRange range("cm_ccg_solve_batch");
  if (n < 1 || !plans || !params || !h || !res) return CM_ERR_ARG;
  const int prec = params[0].precision;
  bool bisect = false;
  for (int i = 0; i < n; ++i) {
    if (!plans[i] || !h[i]) return CM_ERR_ARG;
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) return CM_ERR_ARG;  // a plan's buffers serve one solve at a time
    if (params[i].precision != prec || params[i].maxiter < 1) return CM_ERR_ARG;
    if (params[i].has_hardness && !(params[i].hardness > 0)) return CM_ERR_ARG;
    bisect = bisect || (params[i].has_hardness && params[i].load_control);
    memset(&res[i], 0, sizeof(res[i]));
  }
  if (prec != CM_FP64 && prec != CM_FP32 && prec != CM_MIXED) return CM_ERR_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : plans[0]->stream;
  int maxiter = 0;
  double timeout = 0;
  for (int i = 0; i < n; ++i) {
    maxiter = std::max(maxiter, params[i].maxiter);
    timeout = std::max(timeout, params[i].timeout_s);
  }
  g_polls = 0;
  if (batch_persistent_ok(n, plans, params, prec))
    return batch_persistent(n, plans, params, h, u0, x, jac, active, plastic, res, s);
  typedef std::chrono::steady_clock clk;
  const auto t0 = clk::now();
  std::vector<int> nit32(n, 0), nfev32(n, 0);
  if (prec != CM_FP64) {
    const double rp = prec == CM_MIXED ? (params[0].fp32_pentol_rel > 0 ? params[0].fp32_pentol_rel : 2e-6) : 0.0;
    const double rf = prec == CM_MIXED ? 1e-5 : 0.0;
    std::vector<int> mi(n);
    for (int i = 0; i < n; ++i)
      mi[i] = prec == CM_MIXED ? fp32_cap(params[i].maxiter, params[i].has_hardness) : params[i].maxiter;
    std::vector<CcgState> st32;
    CKS(lockstep_phase<float>(n, plans, params, h, u0, x, jac, active, plastic, false, rp, rf, mi,
                              prec == CM_FP32, bisect, maxiter, timeout, s, &g_polls, st32));
    for (int i = 0; i < n; ++i) {
      CKS(status_error(st32[i]));
      nit32[i] = st32[i].it;
      nfev32[i] = st32[i].nfev;
      if (prec == CM_FP32) {
        fill_result(st32[i], &res[i]);
        res[i].nit_fp32 = nit32[i];
      }
    }
    if (prec == CM_FP32) {
      const double ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
      for (int i = 0; i < n; ++i) { res[i].ms_total = res[i].ms_fp32 = ms; res[i].polls = g_polls; }
      return CM_OK;
    }
  }
  const auto t1 = clk::now();
  std::vector<int> mi(n);
  for (int i = 0; i < n; ++i)
    mi[i] = prec == CM_MIXED ? std::max(1, params[i].maxiter - nit32[i]) : params[i].maxiter;
  std::vector<CcgState> st64;
  CKS(lockstep_phase<double>(n, plans, params, h, u0, x, jac, active, plastic, prec == CM_MIXED,
                             0.0, 0.0, mi, true, bisect, maxiter, timeout, s, &g_polls, st64));
  const double ms64 = std::chrono::duration<double, std::milli>(clk::now() - t1).count();
  const double ms32 = std::chrono::duration<double, std::milli>(t1 - t0).count();
  for (int i = 0; i < n; ++i) {
    const CcgState& st = st64[i];
    CKS(status_error(st));
    fill_result(st, &res[i]);
    res[i].nit += nit32[i];
    res[i].nfev += nfev32[i];
    res[i].nit_fp32 = nit32[i];
    res[i].ms_fp32 = ms32;
    res[i].ms_fp64 = ms64;
    res[i].ms_total = ms32 + ms64;
    res[i].polls = g_polls;
  }
  return CM_OK;
}

unsigned long long cm_launch_count(void) { return g_launches.load(); }

int cm_stepper_create(void* stream, cm_stepper** out) {
  if (!out) return CM_ERR_ARG;
  cm_stepper* st = new (std::nothrow) cm_stepper();
  if (!st) return CM_ERR_OOM;
  if (stream) {
    st->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete st;
      return CM_ERR_CUDA;
    }
    st->own_stream = true;
  }
  *out = st;
  return CM_OK;
}

int cm_stepper_destroy(cm_stepper* st) {
  if (!st) return CM_OK;
  if (st->stream) cudaStreamSynchronize(st->stream);
  stepper_free(st);
  if (st->own_stream) cudaStreamDestroy(st->stream);
  delete st;
  return CM_OK;
}

int cm_ccg_begin(cm_stepper* stp, cm_plan* p, const cm_ccg_params* prm, const double* h,
                 const double* u0, const double* f0) {
  if (!stp || !p || !prm || !h || prm->maxiter < 1) return CM_ERR_ARG;
  if (prm->precision != CM_FP64 && prm->precision != CM_FP32 && prm->precision != CM_MIXED) return CM_ERR_ARG;
  if (prm->has_hardness && !(prm->hardness > 0)) return CM_ERR_ARG;
  if (p->phase != 0) return CM_ERR_ARG;  // the plan already holds a solve
  // steps run the per-pass kernels, which must fit the domain
  if (!p->w64.tiles.generic_ok || (prm->precision != CM_FP64 && !p->w32.tiles.generic_ok))
    return CM_ERR_SIZE;
  p->params = *prm;
  p->phase_prec = prm->precision;
  p->nit32 = p->nfev32 = 0;
  SolveInput in{h, u0, f0, p->ny};
  if (prm->precision == CM_FP64) {
    CKS(ccg_init<double>(p, p->w64, prm, in, 0.0, 0.0, prm->maxiter, stp->stream));
    p->phase = 2;
  } else {
    const bool mixed = prm->precision == CM_MIXED;
    const double rp = mixed ? (prm->fp32_pentol_rel > 0 ? prm->fp32_pentol_rel : 2e-6) : 0.0;
    const int mi = mixed ? fp32_cap(prm->maxiter, prm->has_hardness) : prm->maxiter;
    CKS(ccg_init<float>(p, p->w32, prm, in, rp, mixed ? 1e-5 : 0.0, mi, stp->stream));
    p->phase = 1;
  }
  return CM_OK;
}

int cm_ccg_step(cm_stepper* stp, int n, cm_plan* const* plans, int iters, int* done) {
  NvtxRange range("cm_ccg_step");
  if (!stp || n < 0 || (n > 0 && (!plans || !done)) || iters < 1) return CM_ERR_ARG;
  std::vector<cm_plan*> g32, g64;
  std::vector<int> i32, i64;
  for (int i = 0; i < n; ++i) {
    if (!plans[i] || plans[i]->phase == 0) return CM_ERR_ARG;
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) return CM_ERR_ARG;
    if (plans[i]->phase == 1) { g32.push_back(plans[i]); i32.push_back(i); }
    else { g64.push_back(plans[i]); i64.push_back(i); }
  }
  std::vector<int> d32(g32.size()), d64(g64.size());
  CKS(stepper_run<float>(stp, g32, iters, d32.data()));
  CKS(stepper_run<double>(stp, g64, iters, d64.data()));
  for (size_t k = 0; k < g32.size(); ++k) done[i32[k]] = d32[k];
  for (size_t k = 0; k < g64.size(); ++k) done[i64[k]] = d64[k];
  return CM_OK;
}

int cm_ccg_handover(cm_stepper* stp, cm_plan* p, const double* h, int* finished) {
  if (!stp || !p || !h || !finished) return CM_ERR_ARG;
  cudaStream_t s = stp->stream;
  *finished = 0;
  if (p->phase == 1) {
    CK(cudaMemcpyAsync(p->h_state, p->w32.st, sizeof(CcgState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const CcgState st = *p->h_state;
    if (!st.done) return CM_ERR_ARG;
    const int err = status_error(st);
    if (err != CM_OK) { p->phase = 0; return err; }
    if (p->phase_prec == CM_FP32) { *finished = 1; return CM_OK; }
    p->nit32 = st.it;
    p->nfev32 = st.nfev;
    CKS(ensure_ccg(p, p->w64));
    k_force_to_domain<float><<<grid_for((long)p->nx * p->ny), 256, 0, s>>>(
        p->w32.st, p->w32.f[0], p->w32.f[1], p->tx, p->ty, p->w64.u, p->nx, p->ny);
    SolveInput in{h, nullptr, p->w64.u, p->ny};
    CKS(ccg_init<double>(p, p->w64, &p->params, in, 0.0, 0.0,
                         std::max(1, p->params.maxiter - st.it), s));
    p->phase = 2;
    return CM_OK;
  }
  if (p->phase == 2) {
    *finished = 1;
    return CM_OK;
  }
  return CM_ERR_ARG;
}

int cm_ccg_end(cm_stepper* stp, cm_plan* p, double* x, double* jac, unsigned char* active,
               unsigned char* plastic, cm_ccg_result* res) {
  if (!stp || !p || !res || p->phase == 0) return CM_ERR_ARG;
  memset(res, 0, sizeof(*res));
  CcgState st;
  int rc;
  if (p->phase == 1) rc = finish_ccg<float>(p, p->w32, x, jac, active, plastic, &st, stp->stream);
  else rc = finish_ccg<double>(p, p->w64, x, jac, active, plastic, &st, stp->stream);
  p->phase = 0;
  if (rc != CM_OK) return rc;
  CKS(status_error(st));
  fill_result(st, res);
  if (p->phase_prec == CM_MIXED) {
    res->nit += p->nit32;
    res->nfev += p->nfev32;
    res->nit_fp32 = p->nit32;
  } else if (p->phase_prec == CM_FP32) {
    res->nit_fp32 = st.it;
  }
  return CM_OK;
}

int cm_apply_periodic_noalloc(int nx, int ny, double sx, double sy, double young, double poisson,
                              int op, const double* in, double* out, void* stream) {
  if (!in || !out || (op != CM_OP_DISP && op != CM_OP_FORCE)) return CM_ERR_ARG;
  if (nx < 2 || ny < 2 || !(sx > 0) || !(sy > 0) || !(young > 0)) return CM_ERR_ARG;
  if (nx > CM_NOALLOC_MAX_SIDE || ny > CM_NOALLOC_MAX_SIDE) return CM_ERR_SIZE;
  FftDesc fx, fy;
  if (!make_fft_desc(nx, &fx) || !make_fft_desc(ny, &fy)) return CM_ERR_SIZE;
  const int nyh = ny / 2 + 1;
  Tiles T;
  CKS(choose_tiles(nx, ny, nyh, nx, ny, sizeof(double2), &T));
  // carve the scratch
  unsigned char* base = nullptr;
  CKS(noalloc_scratch(&base));
  const int nt_row = (nx + T.row_tile - 1) / T.row_tile;
  const int nitems = std::max(nt_row, T.ntile_cols);
  const size_t ncols = (size_t)T.ntile_cols * T.col_tile;
  auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
  size_t off = 0;
  const size_t o_slot = off; off = up(off + sizeof(Slot<double>));
  const size_t o_items = off; off = up(off + sizeof(int2) * nitems);
  const size_t o_twx = off; off = up(off + sizeof(double2) * nx);
  const size_t o_twy = off; off = up(off + sizeof(double2) * ny);
  const size_t o_tab = off; off = up(off + sizeof(double) * nx * ncols);
  const size_t o_spec = off; off = up(off + sizeof(double2) * nx * ncols);
  if (off > CM_NOALLOC_BYTES) return CM_ERR_SIZE;
  Slot<double>* d_slot = (Slot<double>*)(base + o_slot);
  int2* d_items = (int2*)(base + o_items);
  double2* d_twx = (double2*)(base + o_twx);
  double2* d_twy = (double2*)(base + o_twy);
  double* d_tab = (double*)(base + o_tab);
  double2* d_spec = (double2*)(base + o_spec);
  double* d_G = (double*)d_spec;  // the unscaled table lives in the spectrum until the transform
  Slot<double> sv;
  memset(&sv, 0, sizeof(sv));
  sv.nx = nx; sv.ny = ny; sv.nyh = nyh; sv.tx = nx; sv.ty = ny;
  sv.row_tile = T.row_tile; sv.col_tile = T.col_tile; sv.lw = T.lw; sv.comp_rows = T.comp_rows;
  sv.nt_rowt = nt_row; sv.nt_rowd = nt_row; sv.nt_col = T.ntile_cols; sv.nt_comp = 0;
  sv.dv_ny = make_fastdiv(ny); sv.dv_nyh = make_fastdiv(nyh); sv.dv_ty = make_fastdiv(ny);
  sv.fx = fx; sv.fy = fy; sv.twx = d_twx; sv.twy = d_twy; sv.spec = d_spec;
  sv.tab[0] = d_tab; sv.tab[1] = d_tab; sv.table_sel = 0;
  sv.in = in; sv.out = out;
  sv.in_rows = nx; sv.in_cols = ny; sv.in_ld = ny;
  sv.out_rows = nx; sv.out_cols = ny; sv.out_ld = ny;
  cudaStream_t s = (cudaStream_t)stream;
  set_smem_attrs<double>();
  const long nh = (long)nx * nyh;
  k_noalloc_setup<<<grid_for(std::max<long>(nitems, std::max(nx, ny))), 256, 0, s>>>(
      d_slot, sv, d_items, nitems, d_twx, nx, d_twy, ny);
  const double Es = young / (1 - poisson * poisson);
  k_table_periodic<<<grid_for(nh), 256, 0, s>>>(d_G, nx, ny, nyh, sx, sy, Es, young, poisson,
                                                 CM_Q0_DEFAULT, 0.0, 0.0, 2);
  const double area = (sx / nx) * (sy / ny);
  const double N = (double)nx * (double)ny;
  k_noalloc_table<<<grid_for(nh), 256, 0, s>>>(d_G, d_tab, nx, nyh, T.lw, op, 1.0 / (area * N), area / N);
  k_row_fwd<double, MODE_PLAIN><<<nt_row, T.threads_row, T.smem_row, s>>>(d_slot, d_items);
  k_col<double, MODE_PLAIN><<<T.ntile_cols, T.threads_col, T.smem_col, s>>>(d_slot, d_items);
  k_row_inv<double, MODE_PLAIN><<<nt_row, T.threads_row, T.smem_row, s>>>(d_slot, d_items);
  g_launches += 6;
  CK(cudaGetLastError());
  return CM_OK;
}

int cm_fft_forward(cm_plan* p, const double* in, int in_rows, int in_cols, int in_ld, double* out,
                   void* stream) {
  if (!p || !in || !out) return CM_ERR_ARG;
  if (in_rows < 0 || in_rows > p->nx || in_cols < 0 || in_cols > p->ny || in_ld < in_cols)
    return CM_ERR_SHAPE;
  cudaStream_t s = stream ? (cudaStream_t)stream : p->stream;
  CKS(launch_plain<double>(p, p->w64, MODE_FWD, 0, in, in_rows, in_cols, in_ld, nullptr, 0, 0, 0, s));
  const long n = (long)(p->nx / 2 + 1) * p->ny;
  k_spec_to_ref<<<grid_for(n), 256, 0, s>>>(p->w64.spec, (double2*)out, p->nx, p->ny,
                                            p->w64.tiles.lw);
  g_launches += 1;
  CK(cudaGetLastError());
  return CM_OK;
}

int cm_kspace_apply(cm_plan* p, int op, double scale, const double* k_in, double* k_out, void* stream) {
  if (!p || !k_in || !k_out || (op != CM_OP_DISP && op != CM_OP_FORCE)) return CM_ERR_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : p->stream;
  const long n = (long)(p->nx / 2 + 1) * p->ny;
  k_kspace_apply<<<grid_for(n), 256, 0, s>>>(p->G, (const double2*)k_in, (double2*)k_out, p->nx,
                                             p->ny, op, scale);
  g_launches += 1;
  CK(cudaGetLastError());
  return CM_OK;
}

int cm_kspace_dot(cm_plan* p, const double* ka, const double* kb, double* out, void* stream) {
  if (!p || !ka || !kb || !out) return CM_ERR_ARG;
  cudaStream_t s = stream ? (cudaStream_t)stream : p->stream;
  const long n = (long)(p->nx / 2 + 1) * p->ny;
  const int blocks = (int)std::max(1L, std::min((n + 255) / 256, 1184L));
  // the solver's reduction scratch holds at least max(nx, tiles) * 32 doubles
  if (blocks > p->w64.partial_blocks * CM_MAX_PARTIAL_VALS) return CM_ERR_SIZE;
  k_kspace_dot<<<blocks, 256, 0, s>>>((const double2*)ka, (const double2*)kb, p->nx, p->ny,
                                      p->w64.partials);
  g_launches += 1;
  std::vector<double> part(blocks);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(part.data(), p->w64.partials, blocks * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double acc = 0.0;
  for (double v : part) acc += v;
  *out = acc / ((double)p->nx * (double)p->ny);
  return CM_OK;
}

int cm_tuning_set_tiles(int precision, int length, int tile_elems) {
  if ((precision != CM_FP64 && precision != CM_FP32) || length < 1 || tile_elems < 0) return CM_ERR_ARG;
  const int pi = precision == CM_FP64 ? 0 : 1;
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto& v = g_tune_elems[pi];
  for (size_t i = 0; i < v.size(); ++i)
    if (v[i].first == length) {
      v.erase(v.begin() + i);
      break;
    }
  if (tile_elems > 0) v.emplace_back(length, tile_elems);
  return CM_OK;
}

int cm_tuning_set_batch_threads(int precision, int threads) {
  if ((precision != CM_FP64 && precision != CM_FP32)) return CM_ERR_ARG;
  if (threads < 32 || threads > CM_FFT_THREADS || (threads & 31)) return CM_ERR_ARG;
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_batch_threads[precision == CM_FP64 ? 0 : 1] = threads;
  return CM_OK;
}

int cm_tuning_set_batch_persistent(int enable) {
  if (enable != 0 && enable != 1) return CM_ERR_ARG;
  g_batch_persistent.store(enable);
  return CM_OK;
}

int cm_tuning_get(int precision, int length, int* tile_elems, int* batch_threads) {
  if ((precision != CM_FP64 && precision != CM_FP32) || length < 1) return CM_ERR_ARG;
  const size_t csize = precision == CM_FP64 ? 16 : 8;
  const int dflt = (int)std::min<size_t>(CM_SMEM_ROW / (2 * csize), 2048);
  if (tile_elems) *tile_elems = tuned_elems(csize, length, dflt);
  if (batch_threads) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    *batch_threads = g_batch_threads[precision == CM_FP64 ? 0 : 1];
  }
  return CM_OK;
}

int cm_selftest_grid_barrier(int blocks, int phantom, double limit_us, int* gave_up) {
  if (blocks < 1 || phantom < 0 || !(limit_us > 0) || limit_us > 1e7 || !gave_up) return CM_ERR_ARG;
  int dev = 0, nsm = 0, coop = 0, per_sm = 0, khz = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  CK(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_selftest_barrier, 128, 0));
  if (!coop || blocks > per_sm * nsm) return CM_ERR_ARG;  // every block must be resident
  const long long limit = (long long)(limit_us * 1e-3 * khz) + 1;
  struct Buf {
    GridBarrier bar;
    int gave_up;
  };
  Buf* d = nullptr;
  CK(cudaMalloc(&d, sizeof(Buf)));
  Buf h;
  memset(&h, 0, sizeof(h));
  h.bar.count = (unsigned)phantom;
  int rc = CM_OK;
  if (cudaMemcpy(d, &h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) rc = CM_ERR_CUDA;
  if (rc == CM_OK) {
    GridBarrier* bar = &d->bar;
    int* out = &d->gave_up;
    void* args[] = {(void*)&bar, (void*)&limit, (void*)&out};
    g_launches += 1;
    if (cudaLaunchCooperativeKernel((const void*)k_selftest_barrier, dim3(blocks), dim3(128), args, 0,
                                    nullptr) != cudaSuccess ||
        cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = CM_ERR_CUDA;
  }
  if (rc != CM_OK) last_cuda_error() = cudaGetLastError();
  cudaFree(d);
  *gave_up = h.gave_up;
  return rc;
}

int cm_ccg_profile(cm_plan* p, const cm_ccg_params* prm, const double* h, int iters,
                   float* ms_per_kernel, int* n_kernels, const char** names) {
  if (!p || !prm || !h || iters < 1 || !ms_per_kernel) return CM_ERR_ARG;
  SolveInput in{h, nullptr, nullptr, p->ny};
  CcgState fin;
  cm_ccg_params q = *prm;
  q.maxiter = std::max(prm->maxiter, iters + 1);
  if (prm->precision == CM_FP64)
    CKS(run_ccg<double>(p, p->w64, &q, in, 0.0, 0.0, q.maxiter, &fin, iters, ms_per_kernel));
  else
    CKS(run_ccg<float>(p, p->w32, &q, in, 0.0, 0.0, q.maxiter, &fin, iters, ms_per_kernel));
  if (n_kernels) *n_kernels = CM_ITER_KERNELS - 1;
  if (names)
    for (int k = 0; k < CM_ITER_KERNELS - 1; ++k) names[k] = k_iter_names[k];
  return fin.done && fin.it < iters ? CM_ERR_ARG : CM_OK;
}

int cm_ccg_solve_host(cm_plan* p, const cm_ccg_params* prm, const double* h, const double* u0,
                      const double* f0, double* x, double* jac, unsigned char* active,
                      unsigned char* plastic, cm_ccg_result* res) {
  if (!p || !prm || !h || !res) return CM_ERR_ARG;
  const size_t nt = (size_t)p->tx * p->ty, nd = (size_t)p->nx * p->ny;
  double *dh = nullptr, *du = nullptr, *df = nullptr, *dx = nullptr, *dj = nullptr;
  unsigned char *da = nullptr, *dp = nullptr;
  int rc = CM_OK;
  cudaStream_t s = p->stream;
  auto cleanup = [&]() {
    cudaFree(dh); cudaFree(du); cudaFree(df); cudaFree(dx); cudaFree(dj); cudaFree(da); cudaFree(dp);
  };
  if (cudaMalloc(&dh, nt * 8) != cudaSuccess) { cleanup(); return CM_ERR_OOM; }
  if (u0 && cudaMalloc(&du, nd * 8) != cudaSuccess) { cleanup(); return CM_ERR_OOM; }
  if (f0 && cudaMalloc(&df, nd * 8) != cudaSuccess) { cleanup(); return CM_ERR_OOM; }
  if (x && cudaMalloc(&dx, nd * 8) != cudaSuccess) { cleanup(); return CM_ERR_OOM; }
  if (jac && cudaMalloc(&dj, nt * 8) != cudaSuccess) { cleanup(); return CM_ERR_OOM; }
  if (active && cudaMalloc(&da, nt) != cudaSuccess) { cleanup(); return CM_ERR_OOM; }
  if (plastic && cudaMalloc(&dp, nt) != cudaSuccess) { cleanup(); return CM_ERR_OOM; }
  if (cudaMemcpyAsync(dh, h, nt * 8, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      (u0 && cudaMemcpyAsync(du, u0, nd * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) ||
      (f0 && cudaMemcpyAsync(df, f0, nd * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)) {
    cleanup();
    return CM_ERR_CUDA;
  }
  rc = cm_ccg_solve(p, prm, dh, du, df, dx, dj, da, dp, res);
  if (rc == CM_OK) {
    if ((x && cudaMemcpyAsync(x, dx, nd * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        (jac && cudaMemcpyAsync(jac, dj, nt * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        (active && cudaMemcpyAsync(active, da, nt, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        (plastic && cudaMemcpyAsync(plastic, dp, nt, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        cudaStreamSynchronize(s) != cudaSuccess)
      rc = CM_ERR_CUDA;
  }
  cleanup();
  return rc;
}

}  // extern "C"
