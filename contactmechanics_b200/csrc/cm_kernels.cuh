// Kernels of the FFT Green's-function operator and the Polonsky-Keer loop.
//
// Operator (evaluate_disp / evaluate_force), three passes per application:
//   k_row_fwd : rows of the real field -> half spectrum along y.  Two real
//               rows are packed into one complex FFT and separated after.
//               In a contact solve the prologue computes the field on the
//               fly (search direction t, or the final force f).
//   k_col     : per column block: FFT along x, multiply by the real Green's
//               table, inverse FFT along x.  Rows of the free (Hockney)
//               domain beyond the topography are zero-filled, not read.
//   k_row_inv : half spectrum -> real rows.  In a contact solve the epilogue
//               consumes the result (sum r*t, or the displacement update
//               with its max|du| / max penetration reductions) instead of
//               writing an extra field.
// CCG element-wise kernels (k_ccg_*) run over the topography region.
//
// Every reduction is deterministic: per-tile partials in a fixed tile
// order, reduced by the last tile of the slot (atomic ticket, no waiting).
#pragma once
#include "cm_slot.cuh"

#define CM_THREADS 256

enum {
  MODE_PLAIN = 0,  // operator on caller buffers
  MODE_T = 1,      // CCG: r = G * t  (forward prologue builds t)
  MODE_F = 2,      // CCG: u = G * f  (forward prologue builds the final f)
  MODE_FWD = 3,    // forward transform only (Green's table construction)
};

// ---------------------------------------------------------------------------
// last-tile reduction
// ---------------------------------------------------------------------------
template <int NV, typename R, typename Fin>
CM_DEVINL void tile_finish(const Slot<R>& S, int tile, int ntiles, double (&v)[NV],
                           const int (&kinds)[NV], Fin fin) {
  __shared__ double red_sm[32 * NV];
  __shared__ int am_last;
  block_reduce<NV>(v, kinds, red_sm);
  if (threadIdx.x == 0) {
    double* P = S.partials + (size_t)tile * NV;
#pragma unroll
    for (int i = 0; i < NV; ++i) P[i] = v[i];
    __threadfence();
    const unsigned prev = atomicAdd(S.counter, 1u);
    am_last = (prev == (unsigned)(ntiles - 1));
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = red_neutral(kinds[i]);
  for (int tt = threadIdx.x; tt < ntiles; tt += blockDim.x) {
#pragma unroll
    for (int i = 0; i < NV; ++i)
      acc[i] = red_apply(kinds[i], acc[i], __ldcg(S.partials + (size_t)tt * NV + i));
  }
  block_reduce<NV>(acc, kinds, red_sm);
  if (threadIdx.x == 0) {
    fin(acc);
    *S.counter = 0;
  }
}

// ---------------------------------------------------------------------------
// operator passes
// ---------------------------------------------------------------------------
template <typename R, int MAXE, int MODE>
__global__ void __launch_bounds__(CM_THREADS)
k_row_fwd(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  CcgState* st = S.st;
  int par = 0, has_h = 0, uniform = 0, apply_nc = 0;
  double beta = 0, offset = 0, H = 0, scale = 1, tau = 0, funif = 0;
  if (MODE == MODE_T || MODE == MODE_F) {
    if (st->done) return;
    if (MODE == MODE_T && st->branch != 0) return;
    par = st->parity;
    has_h = st->p.has_h;
    H = st->p.H;
    offset = st->offset;
    beta = st->beta;
    scale = st->scale;
    tau = st->tau;
    uniform = st->uniform;
    apply_nc = st->apply_nc;
    funif = -st->p.F / st->p.n_surface;
  }
  const int ny = S.ny, nyh = S.nyh, ty = S.ty;
  const int rows_total = (MODE == MODE_PLAIN || MODE == MODE_FWD) ? S.in_rows : S.tx;
  const int x0 = item.y * S.row_tile;
  const int nrows = min(S.row_tile, rows_total - x0);
  const int npairs = (nrows + 1) >> 1;
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scratch = buf + npairs * ny;
  double acc = 0.0;
  const R* fin = (MODE == MODE_T) ? S.f[par] : S.f[par ^ 1];

  for (int e = threadIdx.x; e < npairs * ny; e += blockDim.x) {
    const int p = e / ny, y = e - p * ny;
    R vv[2] = {0, 0};
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const int x = x0 + 2 * p + w;
      if (x >= x0 + nrows) continue;
      if (MODE == MODE_PLAIN || MODE == MODE_FWD) {
        if (y < S.in_cols) vv[w] = S.in[(size_t)x * S.in_ld + y];
      } else if (y < ty) {
        const size_t ic = (size_t)x * ty + y;
        const size_t iu = (size_t)x * ny + y;
        if (MODE == MODE_T) {
          const R fa = fin[ic];
          const bool c = (fa < 0) && (!has_h || (double)fa > -H);
          const R g = (S.u[iu] - S.h[ic]) - (R)offset;
          const R tn = c ? (R)(g + (R)beta * S.t[ic]) : (R)0;
          S.t[ic] = tn;
          if (c) acc += (double)g * (double)tn;
          vv[w] = tn;
        } else {  // MODE_F
          const R fp = fin[ic];
          double v = uniform ? funif : scale * (double)fp;
          const bool flowing = has_h && (double)fp <= -H;
          if (flowing) v = -H;
          if (apply_nc) {
            const R g = (S.u[iu] - S.h[ic]) - (R)offset;
            const bool nc = ((fp == (R)0) && g < 0) || (flowing && g > 0);
            if (nc) v += tau * (double)g;
          }
          const R vr = (R)v;
          S.f[par ^ 1][ic] = vr;
          acc += (double)vr;
          vv[w] = vr;
        }
      }
    }
    buf[e] = cmake<C>(vv[0], vv[1]);
  }
  __syncthreads();
  fft_smem<C, false, MAXE>(buf, scratch, S.fy, npairs, ny, 1, false, S.twy);
  for (int e = threadIdx.x; e < npairs * nyh; e += blockDim.x) {
    const int p = e / nyh, k = e - p * nyh;
    const C z = buf[p * ny + k];
    const C zm = buf[p * ny + (k == 0 ? 0 : ny - k)];
    const int xa = x0 + 2 * p;
    S.spec[(size_t)xa * nyh + k] = cmake<C>((z.x + zm.x) * (R)0.5, (z.y - zm.y) * (R)0.5);
    if (xa + 1 < x0 + nrows)
      S.spec[(size_t)(xa + 1) * nyh + k] = cmake<C>((z.y + zm.y) * (R)0.5, (zm.x - z.x) * (R)0.5);
  }
  if (MODE == MODE_T || MODE == MODE_F) {
    double v[1] = {acc};
    const int kinds[1] = {RED_SUM};
    tile_finish<1>(S, item.y, S.nt_rowt, v, kinds, [&](double (&a)[1]) {
      if (MODE == MODE_T) st->sum_cgt = a[0];
      else st->total_force = -a[0];
    });
  }
}

template <typename R, int MAXE, int MODE>
__global__ void __launch_bounds__(CM_THREADS)
k_col(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  if (MODE == MODE_T || MODE == MODE_F) {
    if (S.st->done) return;
    if (MODE == MODE_T && S.st->branch != 0) return;
  }
  const int nx = S.nx, nyh = S.nyh;
  const int k0 = item.y * S.col_tile;
  const int wc = min(S.col_tile, nyh - k0);
  int nx_in, nx_out;
  const R* tab;
  if (MODE == MODE_PLAIN || MODE == MODE_FWD) {
    nx_in = S.in_rows;
    nx_out = (MODE == MODE_FWD) ? nx : S.out_rows;
    tab = S.tab[S.table_sel];
  } else {
    nx_in = S.tx;
    nx_out = (MODE == MODE_T) ? S.tx : nx;
    tab = S.tab[0];
  }
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scratch = buf + nx * wc;
  const int total = nx * wc;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int x = e / wc, c = e - x * wc;
    buf[e] = (x < nx_in) ? S.spec[(size_t)x * nyh + k0 + c] : czero<C>();
  }
  __syncthreads();
  fft_smem<C, false, MAXE>(buf, scratch, S.fx, wc, 1, wc, true, S.twx);
  if (MODE != MODE_FWD) {
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int x = e / wc, c = e - x * wc;
      buf[e] = cscale(buf[e], __ldg(tab + (size_t)x * nyh + k0 + c));
    }
    __syncthreads();
    fft_smem<C, true, MAXE>(buf, scratch, S.fx, wc, 1, wc, true, S.twx);
  }
  for (int e = threadIdx.x; e < nx_out * wc; e += blockDim.x) {
    const int x = e / wc, c = e - x * wc;
    S.spec[(size_t)x * nyh + k0 + c] = buf[e];
  }
}

template <typename R, int MAXE, int MODE>
__global__ void __launch_bounds__(CM_THREADS)
k_row_inv(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  CcgState* st = S.st;
  int par = 0, has_h = 0, branch = 0;
  double offset = 0, H = 0;
  if (MODE == MODE_T || MODE == MODE_F) {
    if (st->done) return;
    branch = st->branch;
    if (MODE == MODE_T && branch != 0) return;
    par = st->parity;
    has_h = st->p.has_h;
    H = st->p.H;
    offset = st->offset;
  }
  const int ny = S.ny, nyh = S.nyh, ty = S.ty, tx = S.tx;
  const int rows_total = (MODE == MODE_PLAIN) ? S.out_rows : (MODE == MODE_T ? tx : S.nx);
  const int x0 = item.y * S.row_tile;
  const int nrows = min(S.row_tile, rows_total - x0);
  const int npairs = (nrows + 1) >> 1;
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scratch = buf + npairs * ny;
  for (int e = threadIdx.x; e < npairs * nyh; e += blockDim.x) {
    const int p = e / nyh, k = e - p * nyh;
    const int xa = x0 + 2 * p;
    C X = S.spec[(size_t)xa * nyh + k];
    C Y = (xa + 1 < x0 + nrows) ? S.spec[(size_t)(xa + 1) * nyh + k] : czero<C>();
    const bool selfconj = (k == 0) || (2 * k == ny);
    if (selfconj) { X.y = 0; Y.y = 0; }
    buf[p * ny + k] = cmake<C>(X.x - Y.y, X.y + Y.x);
    if (!selfconj) buf[p * ny + ny - k] = cmake<C>(X.x + Y.y, Y.x - X.y);
  }
  __syncthreads();
  fft_smem<C, true, MAXE>(buf, scratch, S.fy, npairs, ny, 1, false, S.twy);
  double a0 = 0.0, a1 = 0.0;  // MODE_T: sum r t ; MODE_F: max|du|, max penetration
  if (MODE == MODE_F) { a0 = 0.0; a1 = -INFINITY; }
  const R* fa_buf = S.f[par];
  for (int e = threadIdx.x; e < npairs * ny; e += blockDim.x) {
    const int p = e / ny, y = e - p * ny;
    const C z = buf[e];
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const int x = x0 + 2 * p + w;
      if (x >= x0 + nrows) continue;
      const R val = w ? z.y : z.x;
      if (MODE == MODE_PLAIN) {
        if (y < S.out_cols) S.out[(size_t)x * S.out_ld + y] = val;
      } else if (MODE == MODE_T) {
        if (y < ty) a0 += (double)val * (double)S.t[(size_t)x * ty + y];
      } else {  // MODE_F: displacement update
        const size_t iu = (size_t)x * ny + y;
        const R uo = S.u[iu];
        a0 = fmax(a0, (double)fabs(val - uo));
        S.u[iu] = val;
        if (x < tx && y < ty) {
          const size_t ic = (size_t)x * ty + y;
          bool c;
          if (branch == 0) {
            const R fa = fa_buf[ic];
            c = (fa < 0) && (!has_h || (double)fa > -H);
          } else {
            c = S.gneg[ic] != 0;
          }
          const R pen = (S.h[ic] + (R)offset) - val;
          a1 = fmax(a1, c ? (double)pen : 0.0);
        }
      }
    }
  }
  if (MODE == MODE_T) {
    double v[1] = {a0};
    const int kinds[1] = {RED_SUM};
    tile_finish<1>(S, item.y, S.nt_rowt, v, kinds, [&](double (&a)[1]) {
      // step length (ConstrainedConjugateGradients.py:287-294)
      double tau = 0.0;
      if (st->A_cg > 0) {
        const double xx = -a[0];
        if (xx > 0.0) tau = st->sum_cgt / xx;
        else st->G = 0.0;
      }
      st->tau = tau;
      st->cur_mixfac = st->p.mixfac;
    });
  } else if (MODE == MODE_F) {
    double v[2] = {a0, a1};
    const int kinds[2] = {RED_MAX, RED_MAX};
    tile_finish<2>(S, item.y, S.nt_rowd, v, kinds, [&](double (&a)[2]) {
      // convergence test (ConstrainedConjugateGradients.py:391-434, 491-492)
      CcgState& s = *st;
      const CcgParams& P = s.p;
      s.maxdu = a[0];
      s.nfev += (s.branch == 0) ? 2 : 1;
      s.G_old = s.G;
      s.rms_pen = (s.A_cg > 0) ? sqrt(s.G / (double)s.A_cg) : sqrt(s.G);
      s.max_pen = fmax(0.0, a[1]);
      const double tf = s.total_force;
      bool conv = true;
      if (P.load_control) conv = conv && fabs((tf - P.F) / tf) < P.thermotol;
      else if (s.have_last_tf) conv = conv && fabs((tf - s.last_tf) / tf) < P.thermotol;
      s.last_tf = tf;
      s.have_last_tf = 1;
      const double mh = P.max_surface + s.offset;
      if (P.load_control && s.have_last_mh) conv = conv && fabs((mh - s.last_mh) / mh) < P.thermotol;
      s.last_mh = mh;
      s.have_last_mh = 1;
      if (s.mode == CMM_MIX)
        conv = conv && s.maxdu < P.pentol && s.max_pres < P.forcetol && s.pad_pres < P.forcetol;
      else
        conv = conv && s.rms_pen < P.pentol && s.max_pen < P.pentol && s.maxdu < P.pentol &&
               s.max_pres < P.forcetol && s.pad_pres < P.forcetol;
      s.parity ^= 1;
      if (conv) {
        s.status = CMS_CONVERGED;
        s.done = 1;
      } else if (isnan(s.G) || isnan(s.rms_pen)) {
        s.status = CMS_NAN;
        s.done = 1;
      } else if (s.it >= P.maxiter) {
        s.status = CMS_MAXITER;
        s.done = 1;
      } else {
        s.it += 1;
      }
    });
  }
}

// ---------------------------------------------------------------------------
// CCG element-wise kernels over the topography region
// ---------------------------------------------------------------------------
#define CM_COMP_LOOP(S, tile)                                              \
  const int cx0 = (tile) * (S).comp_rows;                                  \
  const int crows = min((S).comp_rows, (S).tx - cx0);                      \
  const int cn = crows * (S).ty;                                           \
  for (int e = threadIdx.x; e < cn; e += blockDim.x)

// Start of an iteration: contact areas, raw-gap sums, step kind and offset
// (ConstrainedConjugateGradients.py:239-270, 300-318).
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_begin(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  CcgState* st = S.st;
  if (st->done) return;
  const int par = st->parity, has_h = st->p.has_h;
  const double H = st->p.H;
  const R* f = S.f[par];
  double a_c = 0, a_cg = 0, s_cg = 0, gmax = -INFINITY, gmin = INFINITY;
  CM_COMP_LOOP(S, item.y) {
    const int r = e / S.ty, y = e - r * S.ty;
    const size_t ic = (size_t)(cx0 + r) * S.ty + y;
    const R fa = f[ic];
    const bool c0 = fa < 0;
    const bool c = c0 && (!has_h || (double)fa > -H);
    const R g = S.u[(size_t)(cx0 + r) * S.ny + y] - S.h[ic];
    a_c += c0;
    a_cg += c;
    if (c) s_cg += (double)g;
    gmax = fmax(gmax, (double)g);
    gmin = fmin(gmin, (double)g);
  }
  double v[5] = {a_c, a_cg, s_cg, gmax, gmin};
  const int kinds[5] = {RED_SUM, RED_SUM, RED_SUM, RED_MAX, RED_MIN};
  tile_finish<5>(S, item.y, S.nt_comp, v, kinds, [&](double (&a)[5]) {
    CcgState& s = *st;
    const CcgParams& P = s.p;
    s.A_contact = (long long)a[0];
    s.A_cg = (long long)a[1];
    s.sum_cg = a[2];
    s.gmax = a[3];
    s.gmin = a[4];
    const bool cg = !P.has_h || (s.A_contact > 0 && (double)s.A_cg / (double)s.A_contact > 0.01 &&
                                 s.mixsteps <= 0);
    s.bs_active = 0;
    if (cg) {
      s.branch = 0;
      if (s.mode == CMM_MIX) s.mode = CMM_SD;
      if (P.load_control) s.offset = (s.A_cg > 0) ? s.sum_cg / (double)s.A_cg : 0.0;
    } else {
      s.branch = 1;
      if (s.mode != CMM_MIX) {
        s.mixsteps = P.minmixsteps;
        s.mode = CMM_MIX;
      }
      if (P.load_control) {
        // scipy.optimize.bisect(f, a=max g, b=min g); first pass evaluates f(a)
        s.bs_active = 1;
        s.bs_iter = -1;
        s.bs_xa = s.gmax;
        s.bs_dm = s.gmin - s.gmax;
        s.bs_cand[0] = s.gmax;
      }
    }
  });
}

// G = sum over the CG area of g^2 and the conjugation factor (:273-279).
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_gsum(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  CcgState* st = S.st;
  if (st->done || st->branch != 0) return;
  const int par = st->parity, has_h = st->p.has_h;
  const double H = st->p.H;
  const R off = (R)st->offset;
  const R* f = S.f[par];
  double G = 0;
  CM_COMP_LOOP(S, item.y) {
    const int r = e / S.ty, y = e - r * S.ty;
    const size_t ic = (size_t)(cx0 + r) * S.ty + y;
    const R fa = f[ic];
    const bool c = (fa < 0) && (!has_h || (double)fa > -H);
    const R g = (S.u[(size_t)(cx0 + r) * S.ny + y] - S.h[ic]) - off;
    if (c) G += (double)g * (double)g;
  }
  double v[1] = {G};
  const int kinds[1] = {RED_SUM};
  tile_finish<1>(S, item.y, S.nt_comp, v, kinds, [&](double (&a)[1]) {
    CcgState& s = *st;
    s.G = a[0];
    s.beta = (s.delta > 0 && s.G_old > 0) ? (double)s.delta * (s.G / s.G_old) : 0.0;
  });
}

// One pass of the load-controlled offset bisection of the mixing step
// (ConstrainedConjugateGradients.py:316-318).  Counts #(g < x) for up to 31
// candidate midpoints, i.e. the next five levels of scipy's bisection tree,
// then replays scipy's bisection on those counts bit for bit.
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_bisect(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  CcgState* st = S.st;
  if (st->done || st->branch != 1 || !st->bs_active) return;
  __shared__ double cand[CM_BIS_CAND];
  const int ncand = (st->bs_iter < 0) ? 1 : CM_BIS_CAND;
  if (threadIdx.x < ncand) cand[threadIdx.x] = st->bs_cand[threadIdx.x];
  __syncthreads();
  double cnt[CM_BIS_CAND];
#pragma unroll
  for (int i = 0; i < CM_BIS_CAND; ++i) cnt[i] = 0;
  CM_COMP_LOOP(S, item.y) {
    const int r = e / S.ty, y = e - r * S.ty;
    const size_t ic = (size_t)(cx0 + r) * S.ty + y;
    const double g = (double)(S.u[(size_t)(cx0 + r) * S.ny + y] - S.h[ic]);
#pragma unroll
    for (int i = 0; i < CM_BIS_CAND; ++i)
      if (i < ncand) cnt[i] += (g - cand[i] < 0.0) ? 1.0 : 0.0;
  }
  int kinds[CM_BIS_CAND];
#pragma unroll
  for (int i = 0; i < CM_BIS_CAND; ++i) kinds[i] = RED_SUM;
  tile_finish<CM_BIS_CAND>(S, item.y, S.nt_comp, cnt, kinds, [&](double (&a)[CM_BIS_CAND]) {
    CcgState& s = *st;
    const double H = s.p.H, F = s.p.F;
    const double xtol = 2e-12, rtol = 8.881784197001252e-16;
    const int maxit = 100;
    if (s.bs_iter < 0) {
      const double fa = a[0] * H - F;
      const double fb = 0.0 * H - F;  // nothing lies below min g
      s.bs_fa = fa;
      if (fa * fb > 0) {
        s.status = CMS_BISECT_SIGN;
        s.done = 1;
        s.bs_active = 0;
        return;
      }
      if (fa == 0) { s.offset = s.bs_xa; s.bs_active = 0; return; }
      if (fb == 0) { s.offset = s.gmin; s.bs_active = 0; return; }
      s.bs_iter = 0;
    } else {
      int node = 1;
      double xa = s.bs_xa, dm = s.bs_dm;
      for (int lev = 0; lev < 5; ++lev) {
        dm *= 0.5;
        const double xm = xa + dm;
        const double fm = a[node - 1] * H - F;
        s.bs_iter += 1;
        if (fm * s.bs_fa >= 0) { xa = xm; node = 2 * node + 1; }
        else node = 2 * node;
        if (fm == 0 || fabs(dm) < xtol + rtol * fabs(xm)) {
          s.offset = xm;
          s.bs_active = 0;
          return;
        }
        if (s.bs_iter >= maxit) {
          s.status = CMS_BISECT_SIGN + 1;  // bisection did not converge
          s.done = 1;
          s.bs_active = 0;
          return;
        }
      }
      s.bs_xa = xa;
      s.bs_dm = dm;
    }
    // candidate midpoints of the next five levels, heap-indexed from 1
    double xa_n[CM_BIS_CAND + 1], xm_n[CM_BIS_CAND + 1];
    double dml = s.bs_dm;
    int lev_start = 1;
    for (int lev = 0; lev < 5; ++lev) {
      dml *= 0.5;
      for (int i = lev_start; i < 2 * lev_start; ++i) {
        xa_n[i] = (i == 1) ? s.bs_xa : ((i & 1) ? xm_n[i >> 1] : xa_n[i >> 1]);
        xm_n[i] = xa_n[i] + dml;
        s.bs_cand[i - 1] = xm_n[i];
      }
      lev_start *= 2;
    }
  });
}

// Force update, projection onto [0, H], constraint bookkeeping
// (ConstrainedConjugateGradients.py:296, 320-389).
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_update(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  const int2 item = items[blockIdx.x];
  const Slot<R>& S = slots[item.x];
  CcgState* st = S.st;
  if (st->done) return;
  const int par = st->parity, has_h = st->p.has_h, branch = st->branch;
  const double H = st->p.H;
  const R off = (R)st->offset;
  const R tau = (R)st->tau;
  const double mix = st->cur_mixfac;
  const R* f = S.f[par];
  R* fo = S.f[par ^ 1];
  double a_fl = 0, min_fl = INFINITY, max_t = 0, s_fp = 0, n_nc = 0;
  CM_COMP_LOOP(S, item.y) {
    const int r = e / S.ty, y = e - r * S.ty;
    const size_t ic = (size_t)(cx0 + r) * S.ty + y;
    const R fa = f[ic];
    const R g = (S.u[(size_t)(cx0 + r) * S.ny + y] - S.h[ic]) - off;
    R fn;
    if (branch == 0) {
      const bool c = (fa < 0) && (!has_h || (double)fa > -H);
      fn = c ? (R)(fa + tau * S.t[ic]) : fa;
    } else {
      fn = (R)((R)(1 - mix) * fa - (g < 0 ? (R)(mix * H) : (R)0));
    }
    const bool tensile = fn >= 0;
    const bool flowing = has_h && (double)fn <= -H;
    const bool nc = (tensile && g < 0) || (flowing && g > 0);
    if (tensile) max_t = fmax(max_t, (double)fn);
    if (flowing) { a_fl += 1; min_fl = fmin(min_fl, (double)fn + H); }
    const R fp = tensile ? (R)0 : fn;
    s_fp += (double)fp;
    n_nc += nc;
    fo[ic] = fp;
    if (has_h) S.gneg[ic] = g < 0;
  }
  double v[5] = {a_fl, min_fl, max_t, s_fp, n_nc};
  const int kinds[5] = {RED_SUM, RED_MIN, RED_MAX, RED_SUM, RED_SUM};
  tile_finish<5>(S, item.y, S.nt_comp, v, kinds, [&](double (&a)[5]) {
    CcgState& s = *st;
    const CcgParams& P = s.p;
    s.A_fl = (long long)a[0];
    s.n_nc = (long long)a[4];
    double mp = a[2];
    if (P.has_h && s.A_fl > 0) mp = fmax(mp, -a[1]);
    s.max_pres = mp;
    s.pad_pres = 0.0;  // the force is structurally zero on the padding
    s.uniform = 0;
    s.scale = 1.0;
    if (P.load_control) {
      const double total = -a[3];
      if (total != 0) s.scale = P.F / total;
      else s.uniform = 1;
    }
    if (s.branch == 1) {
      s.cur_mixfac *= P.mixdecfac;
      if (s.mixsteps > 0) s.mixsteps -= 1;
      s.delta = 0;
      s.G = 0;
      s.apply_nc = 0;
    } else if (s.n_nc > 0) {
      s.apply_nc = 1;
      s.delta = 0;
      s.mode = CMM_SD;
    } else {
      s.apply_nc = 0;
      s.delta = 1;
      s.mode = CMM_CG;
    }
  });
}
