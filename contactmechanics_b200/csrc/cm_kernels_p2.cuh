// Contact-solve operator passes specialised for power-of-two transform
// lengths (64..4096), built on the register-resident FFT of cm_fft_p2.cuh.
// Same contract, layouts and reductions as the generic k_row_fwd / k_col /
// k_row_inv in MODE_T and MODE_F; the host picks these when both domain
// sides are powers of two in range.
//
// Thread mapping.  Row kernels: thread (s, tt) = (threadIdx.x >> (LOGN-3),
// threadIdx.x & (N/8-1)) owns elements y = tt + q N/8 of the row pair s.
// Column kernel: thread (c, tt) = (threadIdx.x & (W-1), threadIdx.x >> lw)
// owns elements x = tt + q N/8 of column c of the tile.  Global loads and
// stores at fixed q are contiguous across the warp.
#pragma once
#include "cm_fft_p2.cuh"
#include "cm_kernels.cuh"

#define CM_P2_MIN 6
#define CM_P2_MAX 12

template <typename R, int MODE, int LOGN>
__global__ void __launch_bounds__(sizeof(R) == 8 ? CM_FFT_THREADS / 2 : CM_FFT_THREADS)
k_row_fwd_p2(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  if (st->done) return;
  if (MODE == MODE_T && st->branch != 0) return;
  CcgView cv;
  load_view(st, cv);
  const int nx = Sp->nx, nyh = Sp->nyh, ty = Sp->ty, lw = Sp->lw;
  const int row_tile = Sp->row_tile;
  const int x0 = item.y * row_tile;
  const int nrows = min(row_tile, Sp->tx - x0);
  const int npairs = (nrows + 1) >> 1;
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = tws + N;
  C* bufB = bufA + smem_padded((row_tile >> 1) * N);
  stage_tw_p2<LOGN>(tws, Sp->twy);
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const int xa = x0 + 2 * s;
  const bool va_ok = xa < x0 + nrows, vb_ok = xa + 1 < x0 + nrows;
  const R* __restrict__ u = Sp->u;
  const R* __restrict__ h = Sp->h;
  R* __restrict__ fio = Sp->f[MODE == MODE_T ? cv.par : (cv.par ^ 1)];
  R* __restrict__ t = Sp->t;
  const R off = (R)cv.offset;
  double acc = 0.0, amax = 0.0;
  const bool need_gap = (MODE == MODE_T) || cv.apply_nc;
  // prologue: the 16 field values of this thread (2 rows x 8 columns)
  R fv[2][8], uv[2][8], hv[2][8], tv[2][8];
#pragma unroll
  for (int w = 0; w < 2; ++w) {
    const bool ok = w ? vb_ok : va_ok;
    const int x = xa + w;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int y = tt + q * P::TPS;
      fv[w][q] = 0; uv[w][q] = 0; hv[w][q] = 0; tv[w][q] = 0;
      if (ok && y < ty) {
        const size_t ic = (size_t)x * ty + y;
        fv[w][q] = fio[ic];
        if (need_gap) {
          uv[w][q] = u[(size_t)x * N + y];
          hv[w][q] = h[ic];
        }
        if (MODE == MODE_T) tv[w][q] = t[ic];
      }
    }
  }
  C v[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int y = tt + q * P::TPS;
    R out[2] = {0, 0};
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const bool ok = (w ? vb_ok : va_ok) && y < ty;
      if (!ok) continue;
      const size_t ic = (size_t)(xa + w) * ty + y;
      if (MODE == MODE_T) {
        // search direction (ConstrainedConjugateGradients.py:276-279)
        const R fa = fv[w][q];
        const bool c = (fa < 0) && (!cv.has_h || (double)fa > -cv.H);
        const R g = (uv[w][q] - hv[w][q]) - off;
        const R tn = c ? (R)(g + (R)cv.beta * tv[w][q]) : (R)0;
        t[ic] = tn;
        if (c) acc += (double)g * (double)tn;
        out[w] = tn;
      } else {
        // final force of the iteration (:362-389)
        const R fp = fv[w][q];
        double f = cv.uniform ? cv.funif : cv.scale * (double)fp;
        const bool flowing = cv.has_h && (double)fp <= -cv.H;
        if (flowing) f = -cv.H;
        if (cv.apply_nc) {
          const R g = (uv[w][q] - hv[w][q]) - off;
          const bool nc = ((fp == (R)0) && g < 0) || (flowing && g > 0);
          if (nc) f += cv.tau * (double)g;
        }
        const R fr = (R)f;
        fio[ic] = fr;
        acc += (double)fr;
        amax = fmax(amax, fabs((double)fr));
        out[w] = fr;
      }
    }
    v[q] = cmake<C>(out[0], out[1]);
  }
  __syncthreads();  // twiddles staged
  fft_p2<C, false, LOGN>(v, bufA, bufB, s * N, 1, tt, tws);
  __syncthreads();  // transform reads done before bufA is overwritten
#pragma unroll
  for (int q = 0; q < 8; ++q) bufA[spad(s * N + tt + q * P::TPS)] = v[q];
  __syncthreads();
  C* __restrict__ spec = Sp->spec;
  for (int e = threadIdx.x; e < npairs * nyh; e += blockDim.x) {
    const int p = e / nyh, k = e - p * nyh;
    const C z = bufA[spad(p * N + k)];
    const C zm = bufA[spad(p * N + ((N - k) & (N - 1)))];
    const int x = x0 + 2 * p;
    spec[spec_at(x, k, nx, lw)] = cmake<C>((z.x + zm.x) * (R)0.5, (z.y - zm.y) * (R)0.5);
    if (x + 1 < x0 + nrows)
      spec[spec_at(x + 1, k, nx, lw)] = cmake<C>((z.y + zm.y) * (R)0.5, (zm.x - z.x) * (R)0.5);
  }
  if (MODE == MODE_T) {
    double vr[1] = {acc};
    const int kinds[1] = {RED_SUM};
    tile_finish<1>(Sp->partials, Sp->counter, item.y, Sp->nt_rowt, vr, kinds,
                   [&](double (&a)[1]) { st->sum_cgt = a[0]; });
  } else {
    double vr[2] = {acc, amax};
    const int kinds[2] = {RED_SUM, RED_MAX};
    tile_finish<2>(Sp->partials, Sp->counter, item.y, Sp->nt_rowt, vr, kinds,
                   [&](double (&a)[2]) { fin_force(*st, a); });
  }
}

template <typename R, int MODE, int LOGN>
__global__ void __launch_bounds__(sizeof(R) == 8 ? CM_FFT_THREADS / 2 : CM_FFT_THREADS)
k_col_p2(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  const CcgState* st = Sp->st;
  if (st->done) return;
  if (MODE == MODE_T && st->branch != 0) return;
  const int nyh = Sp->nyh, lw = Sp->lw;
  const int W = 1 << lw;
  const int wc = min(W, nyh - item.y * W);
  const int nx_in = Sp->tx;
  const int nx_out = (MODE == MODE_T) ? Sp->tx : N;
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = tws + N;
  C* bufB = bufA + smem_padded(N * W);
  stage_tw_p2<LOGN>(tws, Sp->twx);
  const int c = threadIdx.x & (W - 1), tt = threadIdx.x >> lw;
  C* __restrict__ blk = Sp->spec + (size_t)item.y * N * W;
  const R* __restrict__ tblk = Sp->tab[0] + (size_t)item.y * N * W;
  const bool col_ok = c < wc;
  C v[8];
  R g[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int x = tt + q * P::TPS;
    v[q] = (col_ok && x < nx_in) ? blk[x * W + c] : czero<C>();
    g[q] = col_ok ? __ldg(tblk + x * W + c) : (R)0;
  }
  __syncthreads();  // twiddles staged
  fft_p2<C, false, LOGN>(v, bufA, bufB, c, W, tt, tws);
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = cscale(v[q], g[q]);
  __syncthreads();  // forward reads done before the inverse writes
  fft_p2<C, true, LOGN>(v, bufA, bufB, c, W, tt, tws);
  if (col_ok) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int x = tt + q * P::TPS;
      if (x < nx_out) blk[x * W + c] = v[q];
    }
  }
}

template <typename R, int MODE, int LOGN>
__global__ void __launch_bounds__(sizeof(R) == 8 ? CM_FFT_THREADS / 2 : CM_FFT_THREADS)
k_row_inv_p2(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  if (st->done) return;
  if (MODE == MODE_T && st->branch != 0) return;
  CcgView cv;
  load_view(st, cv);
  const int nx = Sp->nx, nyh = Sp->nyh, ty = Sp->ty, tx = Sp->tx, lw = Sp->lw;
  const int rows_total = (MODE == MODE_T) ? tx : nx;
  const int row_tile = Sp->row_tile;
  const int x0 = item.y * row_tile;
  const int nrows = min(row_tile, rows_total - x0);
  const int npairs = (nrows + 1) >> 1;
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = tws + N;
  C* bufB = bufA + smem_padded((row_tile >> 1) * N);
  stage_tw_p2<LOGN>(tws, Sp->twy);
  const C* __restrict__ spec = Sp->spec;
  struct XY { C X, Y; };
  batched_loop<4>(npairs * nyh, [&](int e) {
    const int p = e / nyh, k = e - p * nyh;
    const int x = x0 + 2 * p;
    XY r;
    r.X = spec[spec_at(x, k, nx, lw)];
    r.Y = (x + 1 < x0 + nrows) ? spec[spec_at(x + 1, k, nx, lw)] : czero<C>();
    return r;
  }, [&](int e, XY r) {
    const int p = e / nyh, k = e - p * nyh;
    C X = r.X, Y = r.Y;
    const bool selfconj = (k == 0) || (2 * k == N);
    if (selfconj) { X.y = 0; Y.y = 0; }
    bufA[spad(p * N + k)] = cmake<C>(X.x - Y.y, X.y + Y.x);
    if (!selfconj) bufA[spad(p * N + N - k)] = cmake<C>(X.x + Y.y, Y.x - X.y);
  });
  __syncthreads();
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const bool s_ok = s < npairs;
  C v[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = s_ok ? bufA[spad(s * N + tt + q * P::TPS)] : czero<C>();
  // the first stage writes bufB while other threads may still read bufA
  fft_p2<C, true, LOGN>(v, bufB, bufA, s * N, 1, tt, tws);
  const int xa = x0 + 2 * s;
  const bool va_ok = s_ok, vb_ok = s_ok && (xa + 1 < x0 + nrows);
  double a0 = 0.0, a1 = -INFINITY;
  if (MODE == MODE_T) {
    const R* __restrict__ t = Sp->t;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int y = tt + q * P::TPS;
      if (y >= ty) continue;
      if (va_ok) a0 += (double)v[q].x * (double)t[(size_t)xa * ty + y];
      if (vb_ok) a0 += (double)v[q].y * (double)t[(size_t)(xa + 1) * ty + y];
    }
    double vr[1] = {a0};
    const int kinds[1] = {RED_SUM};
    tile_finish<1>(Sp->partials, Sp->counter, item.y, Sp->nt_rowt, vr, kinds,
                   [&](double (&a)[1]) { fin_tau(*st, a); });
  } else {
    R* __restrict__ u = Sp->u;
    const R* __restrict__ h = Sp->h;
    const R* __restrict__ fa_buf = Sp->f[cv.par];
    const unsigned char* __restrict__ gneg = Sp->gneg;
    const R off = (R)cv.offset;
    R uo[2][8], hv[2][8], fa[2][8];
    unsigned char gn[2][8];
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const bool ok = w ? vb_ok : va_ok;
      const int x = xa + w;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int y = tt + q * P::TPS;
        uo[w][q] = 0; hv[w][q] = 0; fa[w][q] = 0; gn[w][q] = 0;
        if (!ok) continue;
        uo[w][q] = u[(size_t)x * N + y];
        if (x < tx && y < ty) {
          const size_t ic = (size_t)x * ty + y;
          hv[w][q] = h[ic];
          if (cv.branch == 0) fa[w][q] = fa_buf[ic];
          else gn[w][q] = gneg[ic];
        }
      }
    }
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const bool ok = w ? vb_ok : va_ok;
      if (!ok) continue;
      const int x = xa + w;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int y = tt + q * P::TPS;
        const R val = w ? v[q].y : v[q].x;
        a0 = fmax(a0, (double)fabs(val - uo[w][q]));
        u[(size_t)x * N + y] = val;
        if (x < tx && y < ty) {
          bool cc;
          if (cv.branch == 0) cc = (fa[w][q] < 0) && (!cv.has_h || (double)fa[w][q] > -cv.H);
          else cc = gn[w][q] != 0;
          const R pen = (hv[w][q] + off) - val;
          a1 = fmax(a1, cc ? (double)pen : 0.0);
        }
      }
    }
    double vr[2] = {a0, a1};
    const int kinds[2] = {RED_MAX, RED_MAX};
    tile_finish<2>(Sp->partials, Sp->counter, item.y, Sp->nt_rowd, vr, kinds,
                   [&](double (&a)[2]) { ccg_converge(*st, a[0], a[1]); });
  }
}
