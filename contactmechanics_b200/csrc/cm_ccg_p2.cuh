// Row passes of one CCG iteration for a single solve on a power-of-two
// domain, in the shape of the operator passes of cm_op_p2.cuh: arguments by
// value, blocks of 2*NP rows walking their tiles with a grid stride, the
// pair-major spectrum stored and loaded straight from the transform
// registers (the column pass splits and packs the row pairs).  The
// solver's element-wise work rides on the transforms with the formulas of
// the per-pass kernels of cm_kernels.cuh:
//
//   k_ccg_row_fwd<MODE_T>  search direction t (ConstrainedConjugateGradients.py
//                          :276-279), sum c g t, rows of the topography;
//   k_ccg_row_fwd<MODE_F>  final force of the iteration (:362-389), its sum
//                          and maximum;
//   k_ccg_row_inv<MODE_T>  r = G t, sum r t -> step length (:287-294);
//   k_ccg_row_inv<MODE_F>  u = G f on the whole domain, max |du|, maximum
//                          penetration, convergence test (:391-434), and the
//                          next iteration's start (the statistics of
//                          k_ccg_begin, :239-270, 300-318), so an iteration
//                          after the first launches no k_ccg_begin.
//
// The column pass between them is k_op_col with the solve's state attached.
// Each block accumulates its tiles' reductions and writes one partial; the
// last block to finish runs the scalar step (tile_finish).
#pragma once
#include "cm_op_p2.cuh"

template <typename R, int MODE, int LOGN>
__global__ void __launch_bounds__(OpShape<R, LOGN>::THREADS, OpShape<R, LOGN>::MINB)
k_ccg_row_fwd(CcgArgs<R> a) {
  typedef typename CT<R>::C C;
  typedef OpShape<R, LOGN> Sh;
  typedef typename Sh::P P;
  constexpr int N = P::N, NP = Sh::NP, ROWS = 2 * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long mbar;
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = Sh::ONEBUF ? tws : tws + N;
  C* bufB = bufA + smem_padded(NP * N);
  pdl_trigger();
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  const C* tw = stage_twiddles<LOGN, Sh::LR, Sh::THREADS, Sh::ONEBUF>(tws, a.op.twy);
  pdl_wait();
  CcgState* st = a.st;
  if (st->done) return;
  if (MODE == MODE_T && st->branch != 0) return;
  CcgView cv;
  load_view(st, cv);
  __syncthreads();
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const int tx = a.tx, ty = a.ty, ny = N;
  unsigned mphase = 0;
  const int ntiles = (tx + ROWS - 1) / ROWS;
  R* __restrict__ fio = a.f[MODE == MODE_T ? cv.par : (cv.par ^ 1)];
  const R* __restrict__ u_in = a.u;
  const R* __restrict__ h_in = a.h;
  R* __restrict__ t_io = a.t;
  const R off = (R)cv.offset;
  const R hdn = neg_down<R>(cv.H);
  const bool need_gap = (MODE == MODE_T) || cv.apply_nc;
  // The tile's input rows (f, then u and h for the gap, then t) are brought
  // into the transform buffers by bulk copies when there are at least three
  // fields and all of them fit (field j of row r at stg[(j * ROWS + r) * ty]);
  // otherwise they are loaded per element.
  R* stg = reinterpret_cast<R*>(bufA);
  const int nfield = 1 + (need_gap ? 2 : 0) + (MODE == MODE_T ? 1 : 0);
  const int nst = nfield >= 3 && (size_t)nfield * ROWS * ty * sizeof(R) <= Sh::STAGE ? nfield : 0;
  const int jt = need_gap ? 3 : 1;  // field index of t
  // reductions accumulate over the block's tiles; one partial per block
  double acc = 0.0;
  R amax = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int x0 = tile * ROWS, xa = x0 + 2 * s;
    if (nst > 0) {
      if (threadIdx.x == 0) {
        fence_async_shared();
        fence_async_global();
        const int nr = min(ROWS, tx - x0);
        const unsigned rb = (unsigned)(ty * sizeof(R));
        mbar_expect_tx(&mbar, (unsigned)(nst * nr) * rb);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (j >= nst) break;
          const R* src = j == 0 ? fio : j == jt ? t_io : j == 1 ? u_in : h_in;
          const int ld = (j == 1 && need_gap) ? ny : ty;
          for (int r = 0; r < nr; ++r)
            bulk_g2s(stg + (size_t)(j * ROWS + r) * ty, src + (size_t)(x0 + r) * ld, rb, &mbar);
        }
      }
      const bool ok = __syncthreads_and(mbar_wait(&mbar, mphase)) != 0;
      mphase ^= 1u;
      if (!ok) {
        // copies read valid rows and always complete; the wait is bounded all the same
        if (threadIdx.x == 0) {
          mbar_wait(&mbar, mphase ^ 1u);
          st->status = CMS_TIMEOUT;
          st->done = 1;
        }
        return;
      }
    }
    // the element-wise step of element (x, y): search direction t (MODE_T)
    // or the iteration's final force (MODE_F), stored and returned
    auto step = [&](int x, int y, R fv, R uv, R hv, R tv) -> R {
      const size_t ic = (size_t)x * ty + y;
      if (MODE == MODE_T) {
        const bool c = (fv < 0) && (!cv.has_h || fv > hdn);
        const R g = (uv - hv) - off;
        const R tn = c ? (R)(g + (R)cv.beta * tv) : (R)0;
        t_io[ic] = tn;
        if (c) acc += (double)g * (double)tn;
        return tn;
      } else {
        double f = cv.uniform ? cv.funif : cv.scale * (double)fv;
        const bool flowing = cv.has_h && fv <= hdn;
        if (flowing) f = -cv.H;
        if (cv.apply_nc) {
          const R g = (uv - hv) - off;
          const bool nc = ((fv == (R)0) && g < 0) || (flowing && g > 0);
          if (nc) f += cv.tau * (double)g;
        }
        const R fr = (R)f;
        fio[ic] = fr;
        acc += (double)fr;
        amax = fmax(amax, fabs(fr));
        return fr;
      }
    };
    R out[2][Sh::E];
    if (nst == nfield) {
      // every input in shared memory
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const int x = xa + w, r = 2 * s + w;
#pragma unroll
        for (int q = 0; q < Sh::E; ++q) {
          const int y = tt + q * P::TPS;
          out[w][q] = 0;
          if (x >= tx || y >= ty) continue;
          const R* row = stg + (size_t)r * ty + y;
          out[w][q] = step(x, y, row[0], need_gap ? row[(size_t)ROWS * ty] : (R)0,
                           need_gap ? row[(size_t)2 * ROWS * ty] : (R)0,
                           MODE == MODE_T ? row[(size_t)jt * ROWS * ty] : (R)0);
        }
      }
    } else {
      // every input of the thread's 2E elements first, then the
      // element-wise step and its stores
      R fv2[2][Sh::E], uv2[2][Sh::E], hv2[2][Sh::E], tv2[2][Sh::E];
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const int x = xa + w;
#pragma unroll
        for (int q = 0; q < Sh::E; ++q) {
          const int y = tt + q * P::TPS;
          fv2[w][q] = 0; uv2[w][q] = 0; hv2[w][q] = 0; tv2[w][q] = 0;
          if (x >= tx || y >= ty) continue;
          const size_t ic = (size_t)x * ty + y;
          fv2[w][q] = fio[ic];
          if (need_gap) {
            uv2[w][q] = u_in[(size_t)x * ny + y];
            hv2[w][q] = h_in[ic];
          }
          if (MODE == MODE_T) tv2[w][q] = t_io[ic];
        }
      }
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const int x = xa + w;
#pragma unroll
        for (int q = 0; q < Sh::E; ++q) {
          const int y = tt + q * P::TPS;
          out[w][q] = 0;
          if (x >= tx || y >= ty) continue;
          out[w][q] = step(x, y, fv2[w][q], uv2[w][q], hv2[w][q], tv2[w][q]);
        }
      }
    }
    if (nst > 0) __syncthreads();  // the transform reuses the staging buffers
    C v[Sh::E];
#pragma unroll
    for (int q = 0; q < Sh::E; ++q) v[q] = cmake<C>(out[0][q], out[1][q]);
    fft_len<C, false, LOGN, Sh::LR, Sh::ONEBUF, Sh::ONESTG>(v, bufA, bufB, s * N, 1, tt, tw);
    if (xa < tx) {
      C* __restrict__ srow = a.op.spec + (size_t)(xa >> 1) * N;
#pragma unroll
      for (int q = 0; q < Sh::E; ++q) srow[kfreq<LOGN, Sh::LR>(tt, q)] = v[q];
    }
    __syncthreads();  // buffers free for the next tile
  }
  if (MODE == MODE_T) {
    double vr[1] = {acc};
    const int kinds[1] = {RED_SUM};
    tile_finish<1>(a.partials, a.counter, blockIdx.x, gridDim.x, vr, kinds,
                   [&](double (&r)[1]) { st->sum_cgt = r[0]; });
  } else {
    double vr[2] = {acc, (double)amax};
    const int kinds[2] = {RED_SUM, RED_MAX};
    tile_finish<2>(a.partials, a.counter, blockIdx.x, gridDim.x, vr, kinds,
                   [&](double (&r)[2]) { fin_force(*st, r); });
  }
}

// shape of the inverse row passes: the displacement pass (MODE_F) of FP32
// solves has its own elements per thread
template <typename R, int MODE, int LOGN>
using InvShape = OpShape<R, LOGN,
                         (MODE == MODE_F && sizeof(R) == 4 && LOGN <= 12) ? CM_ROW_LR_INVF_F32
                                                                          : OpShape<R, LOGN>::LR>;

template <typename R, int MODE, int LOGN>
__global__ void __launch_bounds__(InvShape<R, MODE, LOGN>::THREADS, InvShape<R, MODE, LOGN>::MINB)
k_ccg_row_inv(CcgArgs<R> a) {
  typedef typename CT<R>::C C;
  typedef InvShape<R, MODE, LOGN> Sh;
  typedef typename Sh::P P;
  constexpr int N = P::N, NP = Sh::NP, ROWS = 2 * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = Sh::ONEBUF ? tws : tws + N;
  C* bufB = bufA + smem_padded(NP * N);
  pdl_trigger();
  const C* tw = stage_twiddles<LOGN, Sh::LR, Sh::THREADS, Sh::ONEBUF>(tws, a.op.twy);
  pdl_wait();
  CcgState* st = a.st;
  if (st->done) return;
  if (MODE == MODE_T && st->branch != 0) return;
  CcgView cv;
  load_view(st, cv);
  __syncthreads();
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const int tx = a.tx, ty = a.ty, nx = a.op.nx;
  const int rows_total = (MODE == MODE_T) ? tx : a.u_rows;
  const int ntiles = (rows_total + ROWS - 1) / ROWS;
  const R off = (R)cv.offset;
  const R hdn = neg_down<R>(cv.H);
  const R* __restrict__ fa_buf = a.f[cv.par];
  R* __restrict__ u_io = a.u;
  const R* __restrict__ h_in = a.h;
  const R* __restrict__ t_in = a.t;
  const unsigned char* __restrict__ gneg = a.gneg;
  // reductions accumulate over the block's tiles; one partial per block
  double a0 = 0.0;                                // MODE_T: sum r t
  R du = 0, pmax = -INFINITY;                     // MODE_F: extrema, exact in R
  R gmax = -INFINITY, gmin = INFINITY;
  int n_c = 0, n_cg = 0;                          // counts, exact in int
  double s_cg = 0, s_cg2 = 0;                     // sums of g and g^2 over the CG area
  const R* __restrict__ fn_buf = a.f[cv.par ^ 1];
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int x0 = tile * ROWS;
    const int xa = x0 + 2 * s;
    if (MODE == MODE_F && threadIdx.x == 0) {
      // the rows the epilogue reads (u, h and both force buffers) requested
      // into L2 before the tile's gather and transform: where the whole
      // domain is topography the epilogue's loads otherwise wait on DRAM one
      // row batch at a time (periodic 3072^2 FP32: 352 -> 192 us a launch)
      prefetch_l2(u_io + (size_t)x0 * N, (size_t)min(ROWS, rows_total - x0) * N * sizeof(R));
      const int nt = min(ROWS, tx - x0);
      if (nt > 0) {
        const size_t off = (size_t)x0 * ty, bytes = (size_t)nt * ty * sizeof(R);
        prefetch_l2(h_in + off, bytes);
        prefetch_l2(fa_buf + off, bytes);
        prefetch_l2(fn_buf + off, bytes);
      }
    }
    C v[Sh::E];
    {
      const C* __restrict__ srow = a.op.spec + (size_t)(xa >> 1) * N;
      const bool have = xa < rows_total;
#pragma unroll
      for (int q = 0; q < Sh::E; ++q) v[q] = have ? srow[kfreq<LOGN, Sh::LR>(tt, q)] : czero<C>();
    }
    fft_len<C, true, LOGN, Sh::LR, Sh::ONEBUF, Sh::ONESTG>(v, bufA, bufB, s * N, 1, tt, tw);
    if (MODE == MODE_T) {
#pragma unroll
      for (int q = 0; q < Sh::E; ++q) {
        const int y = tt + q * P::TPS;
        if (y >= ty) continue;
        if (xa < tx) a0 += (double)v[q].x * (double)t_in[(size_t)xa * ty + y];
        if (xa + 1 < tx) a0 += (double)v[q].y * (double)t_in[(size_t)(xa + 1) * ty + y];
      }
    } else {
      // u on the whole domain, max |du| and the maximum penetration; on the
      // topography also the start-of-iteration statistics of the next
      // iteration (k_ccg_begin: contact areas, sum of the gaps over the CG
      // area, extreme gaps; ConstrainedConjugateGradients.py:239-270) from
      // the new displacement and the iteration's final force f[par ^ 1]
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const int x = xa + w;
        if (x >= rows_total) continue;
        // every input of the row's E elements first, then the stores
        R uo[Sh::E], hv[Sh::E], fn[Sh::E];
        bool cc[Sh::E];
#pragma unroll
        for (int q = 0; q < Sh::E; ++q) {
          const int y = tt + q * P::TPS;
          hv[q] = 0; fn[q] = 0; cc[q] = false;
          uo[q] = u_io[(size_t)x * N + y];
          if (x < tx && y < ty) {
            const size_t ic = (size_t)x * ty + y;
            hv[q] = h_in[ic];
            fn[q] = fn_buf[ic];
            if (cv.branch == 0) {
              const R fa = fa_buf[ic];
              cc[q] = (fa < 0) && (!cv.has_h || fa > hdn);
            } else {
              cc[q] = gneg[ic] != 0;
            }
          }
        }
#pragma unroll
        for (int q = 0; q < Sh::E; ++q) {
          const int y = tt + q * P::TPS;
          const R val = w ? v[q].y : v[q].x;
          du = fmax(du, fabs(val - uo[q]));
          u_io[(size_t)x * N + y] = val;
          if (x < tx && y < ty) {
            const R pen = (hv[q] + off) - val;
            pmax = fmax(pmax, cc[q] ? pen : (R)0);
            const bool c0 = fn[q] < 0;
            const bool c = c0 && (!cv.has_h || fn[q] > hdn);
            const R g = val - hv[q];
            n_c += c0;
            n_cg += c;
            if (c) s_cg += (double)g;
            // the reference sums c g^2 over the whole topography, so a NaN
            // gap outside the contact set makes G NaN as well
            if (c) s_cg2 += (double)g * (double)g;
            else if (isnan(g)) s_cg2 += (double)g;
            gmax = fmax(gmax, g);
            gmin = fmin(gmin, g);
          }
        }
      }
    }
    __syncthreads();  // buffers free for the next tile
  }
  if (MODE == MODE_T) {
    double vr[1] = {a0};
    const int kinds[1] = {RED_SUM};
    tile_finish<1>(a.partials, a.counter, blockIdx.x, gridDim.x, vr, kinds,
                   [&](double (&r)[1]) { fin_tau(*st, r); });
  } else {
    double vr[8] = {(double)du, (double)pmax, (double)n_c, (double)n_cg, s_cg, (double)gmax,
                    (double)gmin, s_cg2};
    const int kinds[8] = {RED_MAX, RED_MAX, RED_SUM, RED_SUM, RED_SUM, RED_MAX, RED_MIN, RED_SUM};
    const int fuse = a.fuse_gsum;
    tile_finish<8>(a.partials, a.counter, blockIdx.x, gridDim.x, vr, kinds, [&](double (&r)[8]) {
      ccg_converge(*st, r[0], r[1]);
      if (!st->done) {
        double b[5] = {r[2], r[3], r[4], r[5], r[6]};
        fin_begin(*st, b);
        if (fuse && st->branch == 0) {
          // G = sum over c of (g - offset)^2 from the sums over c of g^2
          // and g (each g^2 of an FP32 gap is exact in FP64); near
          // convergence this loses about eps64 * sum g^2 / G, far below the
          // FP32 gaps' own rounding
          const double off = st->offset;
          double G = r[7] - 2.0 * off * r[4] + (double)st->A_cg * off * off;
          if (G < 0) G = 0;  // rounding (a NaN stays NaN)
          double gv[1] = {G};
          fin_gsum(*st, gv);
        }
      }
    });
  }
}

// ---------------------------------------------------------------------------
// Element-wise passes of the single-solve path, vectorised.  The topography
// fields (h, f, t: tx x ty, rows of a length ty >= 64 that is a multiple of
// four) and the
// displacement (u: rows of length ny on the domain) are read in 16-byte
// vectors of V = 16 / sizeof(R) consecutive elements of one row; every
// thread has U vectors of each field in flight, the grid is one resident
// wave that strides over the vectors, and each block writes one reduction
// partial.  The arithmetic per element is that of the per-tile kernels of
// cm_kernels.cuh (same formulas, same precision).
// ---------------------------------------------------------------------------
template <typename R>
struct alignas(16) Vec16 {
  static constexpr int V = 16 / sizeof(R);
  R v[V];
};

#define CM_EW_THREADS 256

// vector j of the topography: element index (topography) and displacement
// index.  P2: the vectors per topography row are a power of two (a shift
// finds the row), else a multiply-shift division does.
template <bool P2>
struct EwIndex {
  int lvr;      // log2 of the vectors per topography row (P2)
  FastDiv vpr;  // vectors per topography row
  int ny;       // displacement row length
  int V;
  CM_DEVINL void at(long j, size_t& ic, size_t& iu) const {
    long x, y;
    if constexpr (P2) {
      x = j >> lvr;
      y = (j - (x << lvr)) * V;
    } else {
      x = fdiv(vpr, (int)j);
      y = (j - x * (long)vpr.d) * V;
    }
    ic = (size_t)j * V;
    iu = (size_t)x * ny + y;
  }
};

template <bool P2, typename R>
CM_DEVINL EwIndex<P2> ew_index(const CcgArgs<R>& a) {
  EwIndex<P2> e;
  e.V = Vec16<R>::V;
  e.vpr = a.ew_vpr;
  e.lvr = __ffs(e.vpr.d) - 1;
  e.ny = a.ny;
  return e;
}

// whether the element-wise passes of a solve take the shift (EwIndex<true>)
template <typename R>
inline bool ew_pow2(const CcgArgs<R>& a) { return (a.ew_vpr.d & (a.ew_vpr.d - 1)) == 0; }

// G = sum over the CG area of g^2 (ConstrainedConjugateGradients.py:273-279)
template <typename R, int U, bool P2>
__global__ void __launch_bounds__(CM_EW_THREADS) k_ew_gsum(CcgArgs<R> a) {
  typedef Vec16<R> VR;
  constexpr int V = VR::V;
  const EwIndex<P2> ix = ew_index<P2>(a);
  const long nvec = (long)a.tx * a.ty / V;
  pdl_trigger();
  pdl_wait();
  CcgState* st = a.st;
  if (st->done || st->branch != 0) return;
  const int has_h = st->p.has_h;
  const R hdn = neg_down<R>(st->p.H);
  const R off = (R)st->offset;
  const R* __restrict__ f = a.f[st->parity & 1];
  const R* __restrict__ u = a.u;
  const R* __restrict__ h = a.h;
  double G = 0;
  const long step = (long)gridDim.x * blockDim.x * U;
  for (long j0 = (long)blockIdx.x * blockDim.x * U + threadIdx.x; j0 < nvec; j0 += step) {
    VR fv[U], uv[U], hv[U];
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const long j = j0 + (long)i * blockDim.x;
      if (j >= nvec) continue;
      size_t ic, iu;
      ix.at(j, ic, iu);
      fv[i] = *reinterpret_cast<const VR*>(f + ic);
      uv[i] = *reinterpret_cast<const VR*>(u + iu);
      hv[i] = *reinterpret_cast<const VR*>(h + ic);
    }
#pragma unroll
    for (int i = 0; i < U; ++i) {
      if (j0 + (long)i * blockDim.x >= nvec) continue;
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const R fa = fv[i].v[e];
        const bool c = (fa < 0) && (!has_h || fa > hdn);
        const R g = (uv[i].v[e] - hv[i].v[e]) - off;
        // the reference sums c * g^2 over the whole topography, so a NaN gap
        // outside the contact set makes G NaN as well (0 * NaN)
        if (c) G += (double)g * (double)g;
        else if (isnan(g)) G += (double)g;
      }
    }
  }
  double v[1] = {G};
  const int kinds[1] = {RED_SUM};
  tile_finish<1>(a.partials, a.counter, blockIdx.x, gridDim.x, v, kinds,
                 [&](double (&r)[1]) { fin_gsum(*st, r); });
}

// Force update, projection onto [0, H] and the constraint bookkeeping
// (ConstrainedConjugateGradients.py:296, 320-389)
template <typename R, int U, bool P2>
__global__ void __launch_bounds__(CM_EW_THREADS) k_ew_update(CcgArgs<R> a) {
  typedef Vec16<R> VR;
  constexpr int V = VR::V;
  const EwIndex<P2> ix = ew_index<P2>(a);
  const long nvec = (long)a.tx * a.ty / V;
  pdl_trigger();
  pdl_wait();
  CcgState* st = a.st;
  if (st->done) return;
  const int par = st->parity & 1, has_h = st->p.has_h, branch = st->branch;
  const double H = st->p.H;
  const R off = (R)st->offset;
  const R tau = (R)st->tau;
  const double mix = st->cur_mixfac;
  const R* __restrict__ f = a.f[par];
  R* __restrict__ fo = a.f[par ^ 1];
  const R* __restrict__ t = a.t;
  const R* __restrict__ u = a.u;
  const R* __restrict__ h = a.h;
  unsigned char* __restrict__ gneg = const_cast<unsigned char*>(a.gneg);
  const R hdn = neg_down<R>(H);
  // counts in int and extrema in R are exact (x -> (double)x + H is
  // monotonic, so the minimum of fn + H is the minimum fn plus H); only the
  // force sum is accumulated in FP64
  int a_fl = 0, n_nc = 0;
  R min_fn = INFINITY, max_t = 0;
  double s_fp = 0;
  const long step = (long)gridDim.x * blockDim.x * U;
  for (long j0 = (long)blockIdx.x * blockDim.x * U + threadIdx.x; j0 < nvec; j0 += step) {
    VR fv[U], uv[U], hv[U], tv[U];
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const long j = j0 + (long)i * blockDim.x;
      if (j >= nvec) continue;
      size_t ic, iu;
      ix.at(j, ic, iu);
      fv[i] = *reinterpret_cast<const VR*>(f + ic);
      uv[i] = *reinterpret_cast<const VR*>(u + iu);
      hv[i] = *reinterpret_cast<const VR*>(h + ic);
      if (branch == 0) tv[i] = *reinterpret_cast<const VR*>(t + ic);
    }
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const long j = j0 + (long)i * blockDim.x;
      if (j >= nvec) continue;
      VR out;
      unsigned char gn[V];
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const R fa = fv[i].v[e];
        const R g = (uv[i].v[e] - hv[i].v[e]) - off;
        R fn;
        if (branch == 0) {
          const bool c = (fa < 0) && (!has_h || fa > hdn);
          fn = c ? (R)(fa + tau * tv[i].v[e]) : fa;
        } else {
          fn = (R)((R)(1 - mix) * fa - (g < 0 ? (R)(mix * H) : (R)0));
        }
        const bool tensile = fn >= 0;
        const bool flowing = has_h && fn <= hdn;
        const bool nc = (tensile && g < 0) || (flowing && g > 0);
        if (tensile) max_t = fmax(max_t, fn);
        if (flowing) { a_fl += 1; min_fn = fmin(min_fn, fn); }
        const R fp = tensile ? (R)0 : fn;
        s_fp += (double)fp;
        n_nc += nc;
        out.v[e] = fp;
        gn[e] = g < 0;
      }
      const size_t ic = (size_t)j * V;
      *reinterpret_cast<VR*>(fo + ic) = out;
      if (has_h) {
        if constexpr (V == 4)
          *reinterpret_cast<uchar4*>(gneg + ic) = make_uchar4(gn[0], gn[1], gn[2], gn[3]);
        else
          *reinterpret_cast<uchar2*>(gneg + ic) = make_uchar2(gn[0], gn[1]);
      }
    }
  }
  double v[5] = {(double)a_fl, (double)min_fn + H, (double)max_t, s_fp, (double)n_nc};
  const int kinds[5] = {RED_SUM, RED_MIN, RED_MAX, RED_SUM, RED_SUM};
  tile_finish<5>(a.partials, a.counter, blockIdx.x, gridDim.x, v, kinds,
                 [&](double (&r)[5]) { fin_update(*st, r); });
}
