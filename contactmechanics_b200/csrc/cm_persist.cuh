// Persistent cooperative CCG kernel for square power-of-two domains.
//
// One cooperative launch runs up to `max_iters` Polonsky-Keer iterations.
// Every field pass of an iteration (the element-wise reductions, the row and
// column FFT passes of both operator applications, the force update and
// the displacement update) is a grid-stride loop over tiles; each tile
// writes its reduction partials to a tile-indexed array.  Passes are
// separated by a grid barrier; after it every block reduces all partials
// in the same fixed order and advances its own shared-memory copy of the
// solver state with the same scalar step (fin_* of cm_kernels.cuh), so all
// blocks hold bit-identical state and take the same branches, and results
// do not depend on the grid size.  Block 0 writes the state back at exit.
//
// Barrier waits are bounded: a block that waits longer than
// CM_BARRIER_TIMEOUT_CYCLES (or sees another block give up) sets the abort
// flag, marks the solve as timed out and returns; every other block then
// leaves at its next barrier.  Nothing waits unboundedly.
//
// Loads of fields that other blocks write during the launch use ld.global.cg
// (L2, not the SM's L1) so that no block reads a stale line.
#pragma once
#include "cm_kernels_p2.cuh"

#include "cm_launch.h"

#ifndef CM_PERSIST_MIN_BLOCKS_F
#define CM_PERSIST_MIN_BLOCKS_F 1  // resident blocks per SM the FP32 kernel is compiled for
#endif
#ifndef CM_PERSIST_MIN_BLOCKS_D
#define CM_PERSIST_MIN_BLOCKS_D 1
#endif

// Reduce ntiles x NV tile partials in a fixed order; result in thread 0.
template <int NV>
CM_DEVINL void reduce_partials(const double* __restrict__ partials, int ntiles,
                               const int (&kinds)[NV], double (&out)[NV], double* red_sm) {
#pragma unroll
  for (int i = 0; i < NV; ++i) out[i] = red_neutral(kinds[i]);
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) {
#pragma unroll
    for (int i = 0; i < NV; ++i) out[i] = red_apply(kinds[i], out[i], __ldcg(partials + (size_t)t * NV + i));
  }
  block_reduce<NV>(out, kinds, red_sm);
}

// Tile partials with the cross-warp step deferred.  body(t, v) fills the
// thread's values v of tile t; each tile's warp-level tree runs at once and
// its per-warp results wait in shared memory; after up to `slots` tiles (and
// after the last one) every warp finishes one parked tile with block_reduce's
// cross-warp tree and writes its partials.  Same arithmetic in the same order
// as block_reduce per tile, with two block barriers per flush instead of
// three per tile.  red_sm holds CM_RED_SM_VALS doubles, red_tiles
// CM_RED_SLOTS ints.
#define CM_RED_SLOTS 8
#define CM_RED_SM_VALS (CM_RED_SLOTS * 5 * 32)
template <int NV, typename Body>
CM_DEVINL void tile_partials(int ntiles, double* partials, const int (&kinds)[NV], double* red_sm,
                             int* red_tiles, Body body) {
  constexpr int SLOTS = (CM_RED_SLOTS * NV * 32 <= CM_RED_SM_VALS) ? CM_RED_SLOTS : 1;
  static_assert(NV * 32 <= CM_RED_SM_VALS, "reduction buffer too small");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  auto flush = [&](int n) {
    __syncthreads();
    for (int sl = warp; sl < n; sl += nw) {
      const int tile = red_tiles[sl];
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        double x = lane < nw ? red_sm[(sl * NV + i) * 32 + lane] : red_neutral(kinds[i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          x = red_apply(kinds[i], x, __shfl_xor_sync(0xffffffffu, x, o));
        if (lane == 0) partials[(size_t)tile * NV + i] = x;
      }
    }
    __syncthreads();
  };
  int n = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    double v[NV];
    body(t, v);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
        v[i] = red_apply(kinds[i], v[i], __shfl_xor_sync(0xffffffffu, v[i], o));
    }
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < NV; ++i) red_sm[(n * NV + i) * 32 + warp] = v[i];
    }
    if (threadIdx.x == 0) red_tiles[n] = t;
    if (++n == SLOTS) {
      flush(n);
      n = 0;
    }
  }
  if (n > 0) flush(n);
}

// view of the state for the operator phases
CM_DEVINL void view_of(const CcgState& s, CcgView& v) {
  v.par = s.parity;
  v.has_h = s.p.has_h;
  v.uniform = s.uniform;
  v.apply_nc = s.apply_nc;
  v.branch = s.branch;
  v.beta = s.beta;
  v.offset = s.offset;
  v.H = s.p.H;
  v.scale = s.scale;
  v.tau = s.tau;
  v.funif = -s.p.F / s.p.n_surface;
}

// ---------------------------------------------------------------------------
// element-wise phases (one comp tile)
// ---------------------------------------------------------------------------
template <typename R>
CM_DEVINL void ph_begin(const Slot<R>& S, const CcgState& st, int tile, double (&v)[5]) {
  const int ty = S.ty, ny = S.ny, cx0 = tile * S.comp_rows;
  const int cn = min(S.comp_rows, S.tx - cx0) * ty;
  const R* __restrict__ f = S.f[st.parity];
  const int has_h = st.p.has_h;
  const R hdn = neg_down<R>(st.p.H);
  // counts in int and extrema in R are exact; only the sum is accumulated in FP64
  int a_c = 0, a_cg = 0;
  double s_cg = 0;
  R gmax = -INFINITY, gmin = INFINITY;
  struct V3 { R f, u, h; };
  batched_loop<4>(cn, [&](int e) {
    const int r = e / ty, y = e - r * ty;
    return V3{__ldcg(f + (size_t)cx0 * ty + e), __ldcg(S.u + (size_t)(cx0 + r) * ny + y),
              __ldg(S.h + (size_t)cx0 * ty + e)};
  }, [&](int, V3 q) {
    const bool c0 = q.f < 0;
    const bool c = c0 && (!has_h || q.f > hdn);
    const R g = q.u - q.h;
    a_c += c0;
    a_cg += c;
    if (c) s_cg += (double)g;
    gmax = fmax(gmax, g);
    gmin = fmin(gmin, g);
  });
  v[0] = a_c; v[1] = a_cg; v[2] = s_cg; v[3] = gmax; v[4] = gmin;
}

template <typename R>
CM_DEVINL void ph_gsum(const Slot<R>& S, const CcgState& st, int tile, double (&v)[1]) {
  const int ty = S.ty, ny = S.ny, cx0 = tile * S.comp_rows;
  const int cn = min(S.comp_rows, S.tx - cx0) * ty;
  const R* __restrict__ f = S.f[st.parity];
  const int has_h = st.p.has_h;
  const R hdn = neg_down<R>(st.p.H);
  const R off = (R)st.offset;
  double G = 0;
  struct V3 { R f, u, h; };
  batched_loop<4>(cn, [&](int e) {
    const int r = e / ty, y = e - r * ty;
    return V3{__ldcg(f + (size_t)cx0 * ty + e), __ldcg(S.u + (size_t)(cx0 + r) * ny + y),
              __ldg(S.h + (size_t)cx0 * ty + e)};
  }, [&](int, V3 q) {
    const bool c = (q.f < 0) && (!has_h || q.f > hdn);
    const R g = (q.u - q.h) - off;
    if (c) G += (double)g * (double)g;
  });
  v[0] = G;
}

template <typename R>
CM_DEVINL void ph_bisect(const Slot<R>& S, const CcgState& st, int tile, double (&cnt)[CM_BIS_CAND]) {
  const int ty = S.ty, ny = S.ny, cx0 = tile * S.comp_rows;
  const int cn = min(S.comp_rows, S.tx - cx0) * ty;
  const int ncand = (st.bs_iter < 0) ? 1 : CM_BIS_CAND;
#pragma unroll
  for (int i = 0; i < CM_BIS_CAND; ++i) cnt[i] = 0;
  struct V2 { R u, h; };
  batched_loop<4>(cn, [&](int e) {
    const int r = e / ty, y = e - r * ty;
    return V2{__ldcg(S.u + (size_t)(cx0 + r) * ny + y), __ldg(S.h + (size_t)cx0 * ty + e)};
  }, [&](int, V2 q) {
    const double g = (double)(q.u - q.h);
#pragma unroll
    for (int i = 0; i < CM_BIS_CAND; ++i)
      if (i < ncand) cnt[i] += (g - st.bs_cand[i] < 0.0) ? 1.0 : 0.0;
  });
}

template <typename R>
CM_DEVINL void ph_update(const Slot<R>& S, const CcgState& st, int tile, double (&v)[5]) {
  const int ty = S.ty, ny = S.ny, cx0 = tile * S.comp_rows;
  const int cn = min(S.comp_rows, S.tx - cx0) * ty;
  const int par = st.parity, has_h = st.p.has_h, branch = st.branch;
  const double H = st.p.H;
  const R off = (R)st.offset;
  const R tau = (R)st.tau;
  const double mix = st.cur_mixfac;
  const R* __restrict__ f = S.f[par];
  R* __restrict__ fo = S.f[par ^ 1];
  const R hdn = neg_down<R>(H);
  // counts in int and extrema in R are exact (x -> (double)x + H is monotonic,
  // so the minimum of fn + H is the minimum fn plus H); only the sum is FP64
  int a_fl = 0, n_nc = 0;
  R min_fn = INFINITY, max_t = 0;
  double s_fp = 0;
  struct V4 { R f, u, h, t; };
  batched_loop<4>(cn, [&](int e) {
    const int r = e / ty, y = e - r * ty;
    const size_t ic = (size_t)cx0 * ty + e;
    return V4{__ldcg(f + ic), __ldcg(S.u + (size_t)(cx0 + r) * ny + y), __ldg(S.h + ic),
              branch == 0 ? __ldcg(S.t + ic) : (R)0};
  }, [&](int e, V4 q) {
    const size_t ic = (size_t)cx0 * ty + e;
    const R g = (q.u - q.h) - off;
    R fn;
    if (branch == 0) {
      const bool c = (q.f < 0) && (!has_h || q.f > hdn);
      fn = c ? (R)(q.f + tau * q.t) : q.f;
    } else {
      fn = (R)((R)(1 - mix) * q.f - (g < 0 ? (R)(mix * H) : (R)0));
    }
    const bool tensile = fn >= 0;
    const bool flowing = has_h && fn <= hdn;
    const bool nc = (tensile && g < 0) || (flowing && g > 0);
    if (tensile) max_t = fmax(max_t, fn);
    if (flowing) { a_fl += 1; min_fn = fmin(min_fn, fn); }
    const R fp = tensile ? (R)0 : fn;
    s_fp += (double)fp;
    n_nc += nc;
    fo[ic] = fp;
    if (has_h) S.gneg[ic] = g < 0;
  });
  v[0] = a_fl; v[1] = (double)min_fn + H; v[2] = max_t; v[3] = s_fp; v[4] = n_nc;
}

// ---------------------------------------------------------------------------
// operator phases (one row tile / column tile), LOGN = log2 of the side
// ---------------------------------------------------------------------------
template <typename R, int MODE, int LOGN>
CM_DEVINL void ph_row_fwd(const Slot<R>& S, const CcgView& cv, int tile,
                          typename CT<R>::C* tws, typename CT<R>::C* bufA,
                          typename CT<R>::C* bufB, double (&vr)[2]) {
  typedef typename CT<R>::C C;
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  const int nx = S.nx, nyh = S.nyh, ty = S.ty, lw = S.lw, row_tile = S.row_tile;
  const int x0 = tile * row_tile;
  const int nrows = min(row_tile, S.tx - x0);
  const int npairs = (nrows + 1) >> 1;
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const int xa = x0 + 2 * s;
  const bool va_ok = xa < x0 + nrows, vb_ok = xa + 1 < x0 + nrows;
  R* __restrict__ fio = S.f[MODE == MODE_T ? cv.par : (cv.par ^ 1)];
  const R off = (R)cv.offset;
  const R hdn = neg_down<R>(cv.H);
  double acc = 0.0;
  R amax = 0;  // exact in R
  const bool need_gap = (MODE == MODE_T) || cv.apply_nc;
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
        fv[w][q] = __ldcg(fio + ic);
        if (need_gap) {
          uv[w][q] = __ldcg(S.u + (size_t)x * N + y);
          hv[w][q] = __ldg(S.h + ic);
        }
        if (MODE == MODE_T) tv[w][q] = __ldcg(S.t + ic);
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
        const R fa = fv[w][q];
        const bool c = (fa < 0) && (!cv.has_h || fa > hdn);
        const R g = (uv[w][q] - hv[w][q]) - off;
        const R tn = c ? (R)(g + (R)cv.beta * tv[w][q]) : (R)0;
        S.t[ic] = tn;
        if (c) acc += (double)g * (double)tn;
        out[w] = tn;
      } else {
        const R fp = fv[w][q];
        double f = cv.uniform ? cv.funif : cv.scale * (double)fp;
        const bool flowing = cv.has_h && fp <= hdn;
        if (flowing) f = -cv.H;
        if (cv.apply_nc) {
          const R g = (uv[w][q] - hv[w][q]) - off;
          const bool nc = ((fp == (R)0) && g < 0) || (flowing && g > 0);
          if (nc) f += cv.tau * (double)g;
        }
        const R fr = (R)f;
        fio[ic] = fr;
        acc += (double)fr;
        amax = fmax(amax, fabs(fr));
        out[w] = fr;
      }
    }
    v[q] = cmake<C>(out[0], out[1]);
  }
  fft_p2<C, false, LOGN>(v, bufA, bufB, s * N, 1, tt, tws);
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 8; ++q) bufA[spad(s * N + tt + q * P::TPS)] = v[q];
  __syncthreads();
  C* __restrict__ spec = S.spec;
  for (int e = threadIdx.x; e < npairs * nyh; e += blockDim.x) {
    const int p = e / nyh, k = e - p * nyh;
    const C z = bufA[spad(p * N + k)];
    const C zm = bufA[spad(p * N + ((N - k) & (N - 1)))];
    const int x = x0 + 2 * p;
    spec[spec_at(x, k, nx, lw)] = cmake<C>((z.x + zm.x) * (R)0.5, (z.y - zm.y) * (R)0.5);
    if (x + 1 < x0 + nrows)
      spec[spec_at(x + 1, k, nx, lw)] = cmake<C>((z.y + zm.y) * (R)0.5, (zm.x - z.x) * (R)0.5);
  }
  __syncthreads();  // bufA reads done before the next tile reuses it
  vr[0] = acc;
  vr[1] = amax;
}

template <typename R, int MODE, int LOGN>
CM_DEVINL void ph_col(const Slot<R>& S, int tile, typename CT<R>::C* tws, typename CT<R>::C* bufA,
                      typename CT<R>::C* bufB) {
  typedef typename CT<R>::C C;
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  const int nyh = S.nyh, lw = S.lw;
  const int W = 1 << lw;
  const int wc = min(W, nyh - tile * W);
  const int nx_in = S.tx;
  const int nx_out = (MODE == MODE_T) ? S.tx : N;
  const int c = threadIdx.x & (W - 1), tt = threadIdx.x >> lw;
  C* __restrict__ blk = S.spec + (size_t)tile * N * W;
  const R* __restrict__ tblk = S.tab[0] + (size_t)tile * N * W;
  const bool col_ok = c < wc;
  C v[8];
  R g[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int x = tt + q * P::TPS;
    v[q] = (col_ok && x < nx_in) ? __ldcg(blk + x * W + c) : czero<C>();
    g[q] = col_ok ? __ldg(tblk + x * W + c) : (R)0;
  }
  fft_p2<C, false, LOGN>(v, bufA, bufB, c, W, tt, tws);
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = cscale(v[q], g[q]);
  __syncthreads();
  fft_p2<C, true, LOGN>(v, bufA, bufB, c, W, tt, tws);
  if (col_ok) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int x = tt + q * P::TPS;
      if (x < nx_out) blk[x * W + c] = v[q];
    }
  }
  __syncthreads();
}

// Stage of one column tile: its spectrum block (N x W complex, of which the
// first `rows` rows are copied; the transform treats the others as zero) and
// its Green's table block (N x W reals).
template <typename R>
struct ColStage {
  typedef typename CT<R>::C C;
  static __host__ __device__ size_t bytes(int n, int w) { return (size_t)n * w * (sizeof(C) + sizeof(R)); }
};

// Issue (one thread) the bulk copies of column tile `tile` into `stage`.
template <typename R, int LOGN>
CM_DEVINL void col_issue(const Slot<R>& S, int tile, unsigned char* stage, unsigned long long* mbar) {
  typedef typename CT<R>::C C;
  constexpr int N = 1 << LOGN;
  const int W = 1 << S.lw;
  // the forward input holds the topography's rows only (the rest are zero);
  // rounded up to whole 16-byte units, still inside the N x W block
  const unsigned b_spec = (unsigned)min((S.tx * W * sizeof(C) + 15) & ~(size_t)15, N * W * sizeof(C));
  const unsigned b_tab = (unsigned)(N * W * sizeof(R));
  mbar_expect_tx(mbar, b_spec + b_tab);
  bulk_g2s(stage, S.spec + (size_t)tile * N * W, b_spec, mbar);
  bulk_g2s(stage + (size_t)N * W * sizeof(C), S.tab[0] + (size_t)tile * N * W, b_tab, mbar);
}

// Column pass of one tile from its staged copy (see ph_col).
template <typename R, int MODE, int LOGN>
CM_DEVINL void ph_col_staged(const Slot<R>& S, int tile, const unsigned char* stage,
                             typename CT<R>::C* tws, typename CT<R>::C* bufA, typename CT<R>::C* bufB) {
  typedef typename CT<R>::C C;
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  const int nyh = S.nyh, lw = S.lw;
  const int W = 1 << lw;
  const int wc = min(W, nyh - tile * W);
  const int nx_in = S.tx;
  const int nx_out = (MODE == MODE_T) ? S.tx : N;
  const int c = threadIdx.x & (W - 1), tt = threadIdx.x >> lw;
  C* __restrict__ blk = S.spec + (size_t)tile * N * W;
  const C* __restrict__ sblk = reinterpret_cast<const C*>(stage);
  const R* __restrict__ stab = reinterpret_cast<const R*>(stage + (size_t)N * W * sizeof(C));
  const bool col_ok = c < wc;
  C v[8];
  R g[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int x = tt + q * P::TPS;
    v[q] = (x < nx_in) ? sblk[x * W + c] : czero<C>();
    g[q] = stab[x * W + c];
  }
  fft_p2<C, false, LOGN>(v, bufA, bufB, c, W, tt, tws);
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = cscale(v[q], g[q]);
  __syncthreads();
  fft_p2<C, true, LOGN>(v, bufA, bufB, c, W, tt, tws);
  if (col_ok) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int x = tt + q * P::TPS;
      if (x < nx_out) blk[x * W + c] = v[q];
    }
  }
  __syncthreads();
}

template <typename R, int MODE, int LOGN>
CM_DEVINL void ph_row_inv(const Slot<R>& S, const CcgView& cv, int tile,
                          typename CT<R>::C* tws, typename CT<R>::C* bufA,
                          typename CT<R>::C* bufB, double (&vr)[2]) {
  typedef typename CT<R>::C C;
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  const int nx = S.nx, nyh = S.nyh, ty = S.ty, tx = S.tx, lw = S.lw, row_tile = S.row_tile;
  const int rows_total = (MODE == MODE_T) ? tx : nx;
  const int x0 = tile * row_tile;
  const int nrows = min(row_tile, rows_total - x0);
  const int npairs = (nrows + 1) >> 1;
  const C* __restrict__ spec = S.spec;
  struct XY { C X, Y; };
  batched_loop<4>(npairs * nyh, [&](int e) {
    const int p = e / nyh, k = e - p * nyh;
    const int x = x0 + 2 * p;
    XY r;
    r.X = __ldcg(spec + spec_at(x, k, nx, lw));
    r.Y = (x + 1 < x0 + nrows) ? __ldcg(spec + spec_at(x + 1, k, nx, lw)) : czero<C>();
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
  fft_p2<C, true, LOGN>(v, bufB, bufA, s * N, 1, tt, tws);
  const int xa = x0 + 2 * s;
  const bool va_ok = s_ok, vb_ok = s_ok && (xa + 1 < x0 + nrows);
  double a0 = 0.0, a1 = -INFINITY;
  if (MODE == MODE_T) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int y = tt + q * P::TPS;
      if (y >= ty) continue;
      if (va_ok) a0 += (double)v[q].x * (double)__ldcg(S.t + (size_t)xa * ty + y);
      if (vb_ok) a0 += (double)v[q].y * (double)__ldcg(S.t + (size_t)(xa + 1) * ty + y);
    }
  } else {
    const R* __restrict__ fa_buf = S.f[cv.par];
    const R off = (R)cv.offset;
    const R hdn = neg_down<R>(cv.H);
    R du = 0, pmax = -INFINITY;  // extrema, exact in R
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
        uo[w][q] = __ldcg(S.u + (size_t)x * N + y);
        if (x < tx && y < ty) {
          const size_t ic = (size_t)x * ty + y;
          hv[w][q] = __ldg(S.h + ic);
          if (cv.branch == 0) fa[w][q] = __ldcg(fa_buf + ic);
          else gn[w][q] = __ldcg(S.gneg + ic);
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
        du = fmax(du, fabs(val - uo[w][q]));
        S.u[(size_t)x * N + y] = val;
        if (x < tx && y < ty) {
          bool cc;
          if (cv.branch == 0) cc = (fa[w][q] < 0) && (!cv.has_h || fa[w][q] > hdn);
          else cc = gn[w][q] != 0;
          const R pen = (hv[w][q] + off) - val;
          pmax = fmax(pmax, cc ? pen : (R)0);
        }
      }
    }
    a0 = du;
    a1 = pmax;
  }
  __syncthreads();  // shared buffers free before the next tile
  vr[0] = a0;
  vr[1] = a1;
}

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------
CM_DEVINL unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Column pass over this block's tiles, two stages deep: the bulk copies of
// the next tile run while the current one is transformed.  Returns false if
// a copy did not complete in time (after waiting, bounded, for the other
// stage's copy so that none is in flight when the block leaves).
template <typename R, int MODE, int LOGN>
CM_DEVINL bool col_pass(const Slot<R>& S, typename CT<R>::C* tws, typename CT<R>::C* bufA,
                        typename CT<R>::C* bufB, unsigned char* (&stage)[2],
                        unsigned long long* mbar, unsigned& mphase) {
  const int G = gridDim.x;
  int t = blockIdx.x;
  if (t >= S.nt_col) return true;
  if (threadIdx.x == 0) {
    fence_async_global();
    col_issue<R, LOGN>(S, t, stage[0], &mbar[0]);
  }
  int b = 0;
  for (; t < S.nt_col; t += G) {
    const bool next = t + G < S.nt_col;
    if (next && threadIdx.x == 0) col_issue<R, LOGN>(S, t + G, stage[b ^ 1], &mbar[b ^ 1]);
    // every thread waits; the outcome is made block-uniform before any
    // thread proceeds to the transform's barriers
    const bool ok = __syncthreads_and(mbar_wait(&mbar[b], (mphase >> b) & 1u)) != 0;
    if (!ok) {
      if (next) mbar_wait(&mbar[b ^ 1], (mphase >> (b ^ 1)) & 1u);
      return false;
    }
    mphase ^= 1u << b;
    ph_col_staged<R, MODE, LOGN>(S, t, stage[b], tws, bufA, bufB);
    b ^= 1;
  }
  return true;
}

// stamps (optional, PH_COUNT entries, zeroed by the caller): block 0 adds
// the nanoseconds from the previous grid barrier to the end of each phase's
// barrier, so every phase is charged its tile work, its wait for the slowest
// block and the reduction that follows the previous barrier.
template <typename R, int LOGN>
__global__ void __launch_bounds__(CM_FFT_THREADS / 2,
                                  sizeof(R) == 8 ? CM_PERSIST_MIN_BLOCKS_D : CM_PERSIST_MIN_BLOCKS_F)
k_ccg_persist(const Slot<R>* __restrict__ slot, GridBarrier* bar, int max_iters, int bisect_passes,
              unsigned long long* stamps) {
  typedef typename CT<R>::C C;
  constexpr int N = 1 << LOGN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ CcgState st;
  __shared__ int bar_ok;
  __shared__ double red_sm[CM_RED_SM_VALS > 32 * CM_BIS_CAND ? CM_RED_SM_VALS : 32 * CM_BIS_CAND];
  __shared__ int red_tiles[CM_RED_SLOTS];
  __shared__ Slot<R> S;
  {
    const int nS = (int)(sizeof(Slot<R>) / sizeof(int));
    for (int i = threadIdx.x; i < nS; i += blockDim.x)
      reinterpret_cast<int*>(&S)[i] = reinterpret_cast<const int*>(slot)[i];
    __syncthreads();
    const int nst = (int)(sizeof(CcgState) / sizeof(int));
    for (int i = threadIdx.x; i < nst; i += blockDim.x)
      reinterpret_cast<int*>(&st)[i] = __ldcg(reinterpret_cast<const int*>(S.st) + i);
  }
  unsigned gen = 0;
  if (threadIdx.x == 0) gen = atomicAdd(&bar->gen, 0u);
  C* tws = reinterpret_cast<C*>(smem_raw);  // one table: square domain
  C* bufA = tws + N;
  const int ebuf = smem_padded(max((S.row_tile >> 1) * N, (1 << S.lw) * N));
  C* bufB = bufA + ebuf;
  // two stages of column tiles, filled by bulk copies (see persist_smem_bytes)
  unsigned char* stage[2];
  {
    const size_t o = ((size_t)(N + 2 * ebuf) * sizeof(C) + 127) & ~(size_t)127;
    stage[0] = smem_raw + o;
    stage[1] = stage[0] + ((ColStage<R>::bytes(N, 1 << S.lw) + 127) & ~(size_t)127);
  }
  __shared__ __align__(8) unsigned long long mbar[2];
  unsigned mphase = 0;  // bit b: parity of stage b's next completion
  if (threadIdx.x == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
  }
  stage_tw_p2<LOGN>(tws, S.twy);
  __syncthreads();
  double* partials = S.partials;
  bool alive = true;
  const bool timed = stamps != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
  unsigned long long t_last = timed ? global_ns() : 0ull;
  auto abort_solve = [&]() {
    alive = false;
    if (threadIdx.x == 0) {
      atomicExch(&bar->abort, 1u);
      if (blockIdx.x == 0) {
        st.status = CMS_TIMEOUT;
        st.done = 1;
      }
    }
  };
  auto barrier = [&](int phase) -> bool {
    const bool ok = grid_barrier(bar, gen, &bar_ok);
    if (timed) {
      const unsigned long long t = global_ns();
      stamps[phase] += t - t_last;
      t_last = t;
    }
    if (!ok) {
      alive = false;
      if (threadIdx.x == 0 && blockIdx.x == 0) {
        st.status = CMS_TIMEOUT;
        st.done = 1;
      }
      return false;
    }
    return true;
  };
  for (int iter = 0; iter < max_iters && alive && !st.done; ++iter) {
    // ---- start of the iteration
    {
      double v[5];
      const int kinds[5] = {RED_SUM, RED_SUM, RED_SUM, RED_MAX, RED_MIN};
      tile_partials<5>(S.nt_comp, partials, kinds, red_sm, red_tiles,
                       [&](int t, double (&tv)[5]) { ph_begin<R>(S, st, t, tv); });
      if (!barrier(PH_BEGIN)) break;
      reduce_partials<5>(partials, S.nt_comp, kinds, v, red_sm);
      if (threadIdx.x == 0) fin_begin(st, v);
      __syncthreads();
    }
    // ---- offset bisection of a load-controlled mixing step
    for (int pass = 0; pass < bisect_passes && st.branch == 1 && st.bs_active && !st.done; ++pass) {
      double v[CM_BIS_CAND];
      int kinds[CM_BIS_CAND];
#pragma unroll
      for (int i = 0; i < CM_BIS_CAND; ++i) kinds[i] = RED_SUM;
      tile_partials<CM_BIS_CAND>(S.nt_comp, partials, kinds, red_sm, red_tiles,
                       [&](int t, double (&tv)[CM_BIS_CAND]) { ph_bisect<R>(S, st, t, tv); });
      if (!barrier(PH_BISECT)) break;
      reduce_partials<CM_BIS_CAND>(partials, S.nt_comp, kinds, v, red_sm);
      if (threadIdx.x == 0) fin_bisect(st, v);
      __syncthreads();
    }
    if (!alive || st.done) break;
    CcgView cv;
    if (st.branch == 0) {
      // ---- G, conjugation factor
      {
        double v[1];
        const int kinds[1] = {RED_SUM};
        tile_partials<1>(S.nt_comp, partials, kinds, red_sm, red_tiles,
                         [&](int t, double (&tv)[1]) { ph_gsum<R>(S, st, t, tv); });
        if (!barrier(PH_GSUM)) break;
        reduce_partials<1>(partials, S.nt_comp, kinds, v, red_sm);
        if (threadIdx.x == 0) fin_gsum(st, v);
        __syncthreads();
      }
      // ---- r = G * t
      view_of(st, cv);
      {
        double v[2];
        const int kinds[2] = {RED_SUM, RED_MAX};
        tile_partials<2>(S.nt_rowt, partials, kinds, red_sm, red_tiles,
                         [&](int t, double (&tv)[2]) { ph_row_fwd<R, MODE_T, LOGN>(S, cv, t, tws, bufA, bufB, tv); });
        if (!barrier(PH_ROW_FWD_T)) break;
        reduce_partials<2>(partials, S.nt_rowt, kinds, v, red_sm);
        if (threadIdx.x == 0) st.sum_cgt = v[0];
        __syncthreads();
      }
      if (!col_pass<R, MODE_T, LOGN>(S, tws, bufA, bufB, stage, mbar, mphase)) { abort_solve(); break; }
      if (!barrier(PH_COL_T)) break;
      {
        double v[2];
        const int kinds[2] = {RED_SUM, RED_MAX};
        tile_partials<2>(S.nt_rowt, partials, kinds, red_sm, red_tiles,
                         [&](int t, double (&tv)[2]) { ph_row_inv<R, MODE_T, LOGN>(S, cv, t, tws, bufA, bufB, tv); });
        if (!barrier(PH_ROW_INV_T)) break;
        reduce_partials<2>(partials, S.nt_rowt, kinds, v, red_sm);
        if (threadIdx.x == 0) {
          double a[1] = {v[0]};
          fin_tau(st, a);
        }
        __syncthreads();
      }
    }
    // ---- force update, projection, constraint bookkeeping
    {
      double v[5];
      const int kinds[5] = {RED_SUM, RED_MIN, RED_MAX, RED_SUM, RED_SUM};
      tile_partials<5>(S.nt_comp, partials, kinds, red_sm, red_tiles,
                       [&](int t, double (&tv)[5]) { ph_update<R>(S, st, t, tv); });
      if (!barrier(PH_UPDATE)) break;
      reduce_partials<5>(partials, S.nt_comp, kinds, v, red_sm);
      if (threadIdx.x == 0) fin_update(st, v);
      __syncthreads();
    }
    // ---- u = G * f
    view_of(st, cv);
    {
      double v[2];
      const int kinds[2] = {RED_SUM, RED_MAX};
      tile_partials<2>(S.nt_rowt, partials, kinds, red_sm, red_tiles,
                       [&](int t, double (&tv)[2]) { ph_row_fwd<R, MODE_F, LOGN>(S, cv, t, tws, bufA, bufB, tv); });
      if (!barrier(PH_ROW_FWD_F)) break;
      reduce_partials<2>(partials, S.nt_rowt, kinds, v, red_sm);
      if (threadIdx.x == 0) fin_force(st, v);
      __syncthreads();
    }
    if (!col_pass<R, MODE_F, LOGN>(S, tws, bufA, bufB, stage, mbar, mphase)) { abort_solve(); break; }
    if (!barrier(PH_COL_F)) break;
    {
      double v[2];
      const int kinds[2] = {RED_MAX, RED_MAX};
      tile_partials<2>(S.nt_rowd, partials, kinds, red_sm, red_tiles,
                       [&](int t, double (&tv)[2]) { ph_row_inv<R, MODE_F, LOGN>(S, cv, t, tws, bufA, bufB, tv); });
      if (!barrier(PH_ROW_INV_F)) break;
      reduce_partials<2>(partials, S.nt_rowd, kinds, v, red_sm);
      if (threadIdx.x == 0) ccg_converge(st, v[0], v[1]);
      __syncthreads();
    }
  }
  // every block holds the same state; block 0 publishes it
  if (blockIdx.x == 0) {
    __syncthreads();
    const int nst = (int)(sizeof(CcgState) / sizeof(int));
    for (int i = threadIdx.x; i < nst; i += blockDim.x)
      reinterpret_cast<int*>(S.st)[i] = reinterpret_cast<const int*>(&st)[i];
  }
}

// Host stub of k_ccg_persist for square 2^logn domains (declared in cm_launch.h).
template <typename R>
const void* persist_kernel(int logn) {
  switch (logn) {
#define CM_CASE(L) case L: return (const void*)k_ccg_persist<R, L>;
    CM_P2_CASES(CM_CASE)
#undef CM_CASE
    default: return nullptr;
  }
}
