// Kernels of the FFT Green's-function operator and the Polonsky-Keer loop.
//
// Operator (evaluate_disp / evaluate_force), three passes per application:
//   k_row_fwd : rows of the real field -> half spectrum along y.  Two real
//               rows are packed into one complex FFT and separated after.
//               In a contact solve the prologue computes the field on the
//               fly (search direction t, or the final force f).
//   k_col     : per column tile: FFT along x, multiply by the real Green's
//               table, inverse FFT along x.  Rows of the free (Hockney)
//               domain beyond the topography are zero-filled, not read.
//   k_row_inv : half spectrum -> real rows.  In a contact solve the epilogue
//               consumes the result (sum r*t, or the displacement update
//               with its max|du| / max penetration reductions) instead of
//               writing an extra field.
// CCG element-wise kernels (k_ccg_*) run over the topography region.
//
// Layout of the half spectrum and of the Green's tables in HBM: column tiles
// of width W = 2^lw.  Element (x, k) lives at ((k >> lw) * nx + x) * W +
// (k & (W-1)), so a column tile is one contiguous block (read and written
// whole by k_col) and a row tile of R rows touches contiguous R*W runs.
//
// Every reduction is deterministic: partials (one per tile, or one per block
// when the blocks walk several tiles) reduced in a fixed order by the last
// one to finish (atomic ticket, no waiting).
#pragma once
#include "cm_slot.cuh"

#define CM_THREADS 256      // element-wise kernels
#define CM_FFT_THREADS 512  // upper bound for the transform kernels

enum {
  MODE_PLAIN = 0,  // operator on caller buffers
  MODE_T = 1,      // CCG: r = G * t  (forward prologue builds t)
  MODE_F = 2,      // CCG: u = G * f  (forward prologue builds the final f)
  MODE_FWD = 3,    // forward transform only (Green's table construction)
};

CM_DEVINL size_t spec_at(int x, int k, int nx, int lw) {
  return (((size_t)(k >> lw) * nx + x) << lw) + (k & ((1 << lw) - 1));
}

// ---------------------------------------------------------------------------
// last-tile reduction
// ---------------------------------------------------------------------------
template <int NV, typename Fin>
CM_DEVINL void tile_finish(double* __restrict__ partials, unsigned int* counter, int tile,
                           int ntiles, double (&v)[NV], const int (&kinds)[NV], Fin fin) {
  __shared__ double red_sm[32 * NV];
  __shared__ int am_last;
  block_reduce<NV>(v, kinds, red_sm);
  if (threadIdx.x == 0) {
    double* P = partials + (size_t)tile * NV;
#pragma unroll
    for (int i = 0; i < NV; ++i) P[i] = v[i];
    __threadfence();
    const unsigned prev = atomicAdd(counter, 1u);
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
      acc[i] = red_apply(kinds[i], acc[i], __ldcg(partials + (size_t)tt * NV + i));
  }
  block_reduce<NV>(acc, kinds, red_sm);
  if (threadIdx.x == 0) {
    fin(acc);
    *counter = 0;
  }
}

#ifndef CM_BARRIER_SLEEP_NS
#define CM_BARRIER_SLEEP_NS 32  // back-off between polls of the barrier word
#endif

CM_DEVINL unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

CM_DEVINL unsigned ld_relaxed_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// All blocks of the grid meet; returns false if the wait gave up (after
// limit_cycles SM clock cycles, or when another block gave up first and set
// the abort word).
CM_DEVINL bool grid_barrier(GridBarrier* bar, unsigned& gen, int* ok_sm,
                            long long limit_cycles = CM_BARRIER_TIMEOUT_CYCLES) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g = gen;
    __threadfence();
    const unsigned arrived = atomicAdd(&bar->count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicExch(&bar->gen, g + 1);
    } else {
      const long long t0 = clock64();
      while (true) {
        if (ld_acquire_gpu(&bar->gen) != g) break;
        if (ld_relaxed_gpu(&bar->abort) != 0u) { ok = 0; break; }
        if (clock64() - t0 > limit_cycles) {
          atomicExch(&bar->abort, 1u);
          ok = 0;
          break;
        }
        if (CM_BARRIER_SLEEP_NS > 0) __nanosleep(CM_BARRIER_SLEEP_NS);
      }
    }
    __threadfence();
    gen = g + 1;
    *ok_sm = ok;
  }
  __syncthreads();
  return *ok_sm != 0;
}

// stage the FFT descriptor and twiddle table of length n in shared memory
template <typename C>
CM_DEVINL void stage_fft(FftDesc& fd, const FftDesc& src, C* tws, const C* __restrict__ tw, int n) {
  const int nint = (int)(sizeof(FftDesc) / sizeof(int));
  for (int i = threadIdx.x; i < nint; i += blockDim.x)
    reinterpret_cast<int*>(&fd)[i] = reinterpret_cast<const int*>(&src)[i];
  for (int i = threadIdx.x; i < n; i += blockDim.x) tws[i] = __ldg(tw + i);
}

// The largest R not above -H: for any R value x, (double)x > -H exactly when
// x > neg_down<R>(H), and (double)x <= -H exactly when x <= neg_down<R>(H),
// so the hardness tests run in the field's own type.
template <typename R> CM_DEVINL R neg_down(double H);
template <> CM_DEVINL float neg_down<float>(double H) { return __double2float_rd(-H); }
template <> CM_DEVINL double neg_down<double>(double H) { return -H; }

// scalar state of a contact solve that the operator prologues/epilogues use
struct CcgView {
  int par, has_h, uniform, apply_nc, branch;
  double beta, offset, H, scale, tau, funif;
};

CM_DEVINL void load_view(const CcgState* st, CcgView& v) {
  v.par = st->parity;
  v.has_h = st->p.has_h;
  v.uniform = st->uniform;
  v.apply_nc = st->apply_nc;
  v.branch = st->branch;
  v.beta = st->beta;
  v.offset = st->offset;
  v.H = st->p.H;
  v.scale = st->scale;
  v.tau = st->tau;
  v.funif = -st->p.F / st->p.n_surface;
}

// ---------------------------------------------------------------------------
// scalar steps between the field passes (shared by every execution path)
// ---------------------------------------------------------------------------
// Step kind and offset (ConstrainedConjugateGradients.py:239-270, 300-318).
CM_DEVINL void fin_begin(CcgState& s, double (&a)[5]) {
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

}

// G and the conjugation factor (:273-279).
CM_DEVINL void fin_gsum(CcgState& s, double (&a)[1]) {
  s.G = a[0];
  s.beta = (s.delta > 0 && s.G_old > 0) ? (double)s.delta * (s.G / s.G_old) : 0.0;

}

// Replays five levels of scipy's bisection on the counts of one pass (:316-318).
CM_DEVINL void fin_bisect(CcgState& s, double (&a)[CM_BIS_CAND]) {
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

}

// Step length (:287-294).
CM_DEVINL void fin_tau(CcgState& s, double (&a)[1]) {
  // step length (ConstrainedConjugateGradients.py:287-294)
  double tau = 0.0;
  if (s.A_cg > 0) {
    const double xx = -a[0];
    if (xx > 0.0) tau = s.sum_cgt / xx;
    else s.G = 0.0;
  }
  s.tau = tau;
  s.cur_mixfac = s.p.mixfac;

}

// Load scaling, hardness cap and restart bookkeeping after the projection (:334-389).
CM_DEVINL void fin_update(CcgState& s, double (&a)[5]) {
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

}

// Total force of the iteration's final forces and their maximum magnitude.
CM_DEVINL void fin_force(CcgState& s, double (&a)[2]) {
  s.total_force = -a[0];
  s.fmax = a[1];

}

// ---------------------------------------------------------------------------
// operator passes
// ---------------------------------------------------------------------------
// Loads of fields that other blocks of the same launch may have written
// (the persistent batch kernel runs every pass of a solve in one launch)
// bypass L1; tables and twiddles are constant and read through it.
template <typename T> CM_DEVINL T ldf(const T* p) { return __ldcg(p); }

// Row tile `tile` of the forward pass: the tile's rows of the field (the
// caller's buffer, or the CCG prologue's search direction / final force),
// packed-pair FFTs along y, half spectrum to the column-tile layout.  fd /
// tws hold the staged descriptor and twiddles of length ny; buf and scratch
// row_tile/2 * ny elements each.  acc / amax collect this thread's share of
// the tile's sums (MODE_T: sum g t over the CG set; MODE_F: sum f, max |f|).
template <typename R, int MODE>
CM_DEVINL void row_fwd_tile(const Slot<R>* __restrict__ Sp, const CcgView& cv, int tile,
                            const FftDesc& fd, const typename CT<R>::C* tws,
                            typename CT<R>::C* buf, typename CT<R>::C* scratch, double& acc,
                            double& amax) {
  typedef typename CT<R>::C C;
  const int nx = Sp->nx, ny = Sp->ny, nyh = Sp->nyh, ty = Sp->ty, lw = Sp->lw;
  const int rows_total = (MODE == MODE_PLAIN || MODE == MODE_FWD) ? Sp->in_rows : Sp->tx;
  const int row_tile = Sp->row_tile;
  const int x0 = tile * row_tile;
  const int nrows = min(row_tile, rows_total - x0);
  const int npairs = (nrows + 1) >> 1;
  const FastDiv dny = Sp->dv_ny, dnyh = Sp->dv_nyh;
  C* __restrict__ spec = Sp->spec;

  if (MODE == MODE_PLAIN || MODE == MODE_FWD) {
    const R* __restrict__ in = Sp->in;
    const int in_cols = Sp->in_cols, in_ld = Sp->in_ld;
    batched_loop<4>(npairs * ny, [&](int e) {
      const int p = fdiv(dny, e), y = e - p * ny;
      const int xa = x0 + 2 * p;
      R va = 0, vb = 0;
      if (y < in_cols) {
        va = ldf(in + (size_t)xa * in_ld + y);
        if (xa + 1 < x0 + nrows) vb = ldf(in + (size_t)(xa + 1) * in_ld + y);
      }
      return cmake<C>(va, vb);
    }, [&](int e, C v) { buf[e] = v; });
  } else {
    const R* __restrict__ u = Sp->u;
    const R* __restrict__ h = Sp->h;
    R* __restrict__ fio = Sp->f[MODE == MODE_T ? cv.par : (cv.par ^ 1)];
    R* __restrict__ t = Sp->t;
    const R off = (R)cv.offset;
    struct In { R f[2], u[2], h[2], t[2]; };
    batched_loop<2>(npairs * ny, [&](int e) {
      const int p = fdiv(dny, e), y = e - p * ny;
      In v;
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const int x = x0 + 2 * p + w;
        v.f[w] = 0; v.u[w] = 0; v.h[w] = 0; v.t[w] = 0;
        if (x < x0 + nrows && y < ty) {
          const size_t ic = (size_t)x * ty + y;
          v.f[w] = ldf(fio + ic);
          if (MODE == MODE_T || cv.apply_nc) {
            v.u[w] = ldf(u + (size_t)x * ny + y);
            v.h[w] = ldf(h + ic);
          }
          if (MODE == MODE_T) v.t[w] = ldf(t + ic);
        }
      }
      return v;
    }, [&](int e, const In& v) {
      const int p = fdiv(dny, e), y = e - p * ny;
      R vv[2] = {0, 0};
      if (y < ty) {
#pragma unroll
        for (int w = 0; w < 2; ++w) {
          const int x = x0 + 2 * p + w;
          if (x >= x0 + nrows) continue;
          const size_t ic = (size_t)x * ty + y;
          if (MODE == MODE_T) {
            // search direction (ConstrainedConjugateGradients.py:276-279)
            const R fa = v.f[w];
            const bool c = (fa < 0) && (!cv.has_h || (double)fa > -cv.H);
            const R g = (v.u[w] - v.h[w]) - off;
            const R tn = c ? (R)(g + (R)cv.beta * v.t[w]) : (R)0;
            t[ic] = tn;
            if (c) acc += (double)g * (double)tn;
            vv[w] = tn;
          } else {
            // final force of the iteration (:362-389)
            const R fp = v.f[w];
            double fv = cv.uniform ? cv.funif : cv.scale * (double)fp;
            const bool flowing = cv.has_h && (double)fp <= -cv.H;
            if (flowing) fv = -cv.H;
            if (cv.apply_nc) {
              const R g = (v.u[w] - v.h[w]) - off;
              const bool nc = ((fp == (R)0) && g < 0) || (flowing && g > 0);
              if (nc) fv += cv.tau * (double)g;
            }
            const R vr = (R)fv;
            fio[ic] = vr;
            acc += (double)vr;
            amax = fmax(amax, fabs((double)vr));
            vv[w] = vr;
          }
        }
      }
      buf[e] = cmake<C>(vv[0], vv[1]);
    });
  }
  __syncthreads();
  const C* res = fft_smem<C, false>(buf, scratch, fd, npairs, ny, 1, false, tws);
  for (int e = threadIdx.x; e < npairs * nyh; e += blockDim.x) {
    const int p = fdiv(dnyh, e), k = e - p * nyh;
    const C z = res[p * ny + k];
    const C zm = res[p * ny + (k == 0 ? 0 : ny - k)];
    const int xa = x0 + 2 * p;
    spec[spec_at(xa, k, nx, lw)] = cmake<C>((z.x + zm.x) * (R)0.5, (z.y - zm.y) * (R)0.5);
    if (xa + 1 < x0 + nrows)
      spec[spec_at(xa + 1, k, nx, lw)] = cmake<C>((z.y + zm.y) * (R)0.5, (zm.x - z.x) * (R)0.5);
  }
}

template <typename R, int MODE>
__global__ void __launch_bounds__(CM_FFT_THREADS)
k_row_fwd(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc fd;
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  CcgView cv{};
  if (MODE == MODE_T || MODE == MODE_F) {
    if (st->done) return;
    if (MODE == MODE_T && st->branch != 0) return;
    load_view(st, cv);
  }
  const int ny = Sp->ny;
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* buf = tws + ny;
  C* scratch = buf + (Sp->row_tile >> 1) * ny;
  stage_fft(fd, Sp->fy, tws, Sp->twy, ny);
  double acc = 0.0, amax = 0.0;
  row_fwd_tile<R, MODE>(Sp, cv, item.y, fd, tws, buf, scratch, acc, amax);
  if (MODE == MODE_T) {
    double v[1] = {acc};
    const int kinds[1] = {RED_SUM};
    tile_finish<1>(Sp->partials, Sp->counter, item.y, Sp->nt_rowt, v, kinds,
                   [&](double (&a)[1]) { st->sum_cgt = a[0]; });
  } else if (MODE == MODE_F) {
    double v[2] = {acc, amax};
    const int kinds[2] = {RED_SUM, RED_MAX};
    tile_finish<2>(Sp->partials, Sp->counter, item.y, Sp->nt_rowt, v, kinds,
                   [&](double (&a)[2]) { fin_force(*st, a); });
  }
}

// Column tile `tile` (spectrum columns tile*W .. tile*W + W): FFT along x,
// multiply by the Green's table, inverse FFT along x.  fd / tws: staged
// descriptor and twiddles of length nx; buf and scratch nx * W elements each.
template <typename R, int MODE>
CM_DEVINL void col_tile(const Slot<R>* __restrict__ Sp, int tile, const FftDesc& fd,
                        const typename CT<R>::C* tws, typename CT<R>::C* buf,
                        typename CT<R>::C* scratch) {
  typedef typename CT<R>::C C;
  const int nx = Sp->nx, nyh = Sp->nyh, lw = Sp->lw;
  const int W = 1 << lw;
  const int k0 = tile * W;
  const int wc = min(W, nyh - k0);
  int nx_in, nx_out;
  const R* __restrict__ tab;
  if (MODE == MODE_PLAIN || MODE == MODE_FWD) {
    nx_in = Sp->in_rows;
    nx_out = (MODE == MODE_FWD) ? nx : Sp->out_rows;
    tab = Sp->tab[Sp->table_sel];
  } else {
    nx_in = Sp->tx;
    nx_out = (MODE == MODE_T) ? Sp->tx : nx;
    tab = Sp->tab[0];
  }
  // the tile is one contiguous block of nx * W elements in HBM
  C* __restrict__ blk = Sp->spec + (size_t)tile * nx * W;
  const R* __restrict__ tblk = tab + (size_t)tile * nx * W;
  const int total = nx * wc;
  if (wc == W) {
    batched_loop<8>(nx_in * W, [&](int e) { return ldf(blk + e); }, [&](int e, C v) { buf[e] = v; });
    for (int e = nx_in * W + threadIdx.x; e < total; e += blockDim.x) buf[e] = czero<C>();
  } else {
    batched_loop<8>(total, [&](int e) {
      const int x = e / wc, c = e - x * wc;
      return (x < nx_in) ? ldf(blk + x * W + c) : czero<C>();
    }, [&](int e, C v) { buf[e] = v; });
  }
  __syncthreads();
  C* res = fft_smem<C, false>(buf, scratch, fd, wc, 1, wc, true, tws);
  if (MODE != MODE_FWD) {
    batched_loop<8>(total, [&](int e) {
      const int x = e / wc, c = e - x * wc;
      return __ldg(tblk + x * W + c);
    }, [&](int e, R g) { res[e] = cscale(res[e], g); });
    __syncthreads();
    res = fft_smem<C, true>(res, res == buf ? scratch : buf, fd, wc, 1, wc, true, tws);
  }
  if (wc == W) {
    for (int e = threadIdx.x; e < nx_out * W; e += blockDim.x) blk[e] = res[e];
  } else {
    for (int e = threadIdx.x; e < nx_out * wc; e += blockDim.x) {
      const int x = e / wc, c = e - x * wc;
      blk[x * W + c] = res[e];
    }
  }
}

template <typename R, int MODE>
__global__ void __launch_bounds__(CM_FFT_THREADS)
k_col(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc fd;
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  if (MODE == MODE_T || MODE == MODE_F) {
    const CcgState* st = Sp->st;
    if (st->done) return;
    if (MODE == MODE_T && st->branch != 0) return;
  }
  const int nx = Sp->nx;
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* buf = tws + nx;
  C* scratch = buf + nx * (1 << Sp->lw);
  stage_fft(fd, Sp->fx, tws, Sp->twx, nx);
  col_tile<R, MODE>(Sp, item.y, fd, tws, buf, scratch);
}

// Convergence test at the end of an iteration (ConstrainedConjugateGradients.py
// :391-434, 491-492); run by the last tile of the displacement update.
CM_DEVINL void ccg_converge(CcgState& s, double maxdu_in, double maxpen_in) {
  // convergence test (ConstrainedConjugateGradients.py:391-434, 491-492)
  const CcgParams& P = s.p;
  s.rep_area = s.A_contact;
  s.rep_cg_area = s.A_cg;
  s.rep_offset = s.offset;
  s.rep_mode = s.mode;
  s.maxdu = maxdu_in;
  s.nfev += (s.branch == 0) ? 2 : 1;
  s.G_old = s.G;
  s.rms_pen = (s.A_cg > 0) ? sqrt(s.G / (double)s.A_cg) : sqrt(s.G);
  s.max_pen = fmax(0.0, maxpen_in);
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
  const double ftol = fmax(P.forcetol, P.rel_forcetol * s.fmax);
  if (s.mode == CMM_MIX)
    conv = conv && s.maxdu < P.pentol && s.max_pres < ftol && s.pad_pres < ftol;
  else
    conv = conv && s.rms_pen < P.pentol && s.max_pen < P.pentol && s.maxdu < P.pentol &&
           s.max_pres < ftol && s.pad_pres < ftol;
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
}

// Row tile `tile` of the inverse pass: half spectrum -> real rows, then the
// caller's buffer, or the CCG epilogue.  fd / tws / buf / scratch as for
// row_fwd_tile.  a0 / a1 collect this thread's share of the tile's sums
// (MODE_T: sum r t; MODE_F: max |du|, max penetration over the CG set).
template <typename R, int MODE>
CM_DEVINL void row_inv_tile(const Slot<R>* __restrict__ Sp, const CcgView& cv, int tile,
                            const FftDesc& fd, const typename CT<R>::C* tws,
                            typename CT<R>::C* buf, typename CT<R>::C* scratch, double& a0,
                            double& a1) {
  typedef typename CT<R>::C C;
  const int nx = Sp->nx, ny = Sp->ny, nyh = Sp->nyh, ty = Sp->ty, tx = Sp->tx, lw = Sp->lw;
  const int rows_total = (MODE == MODE_PLAIN) ? Sp->out_rows : (MODE == MODE_T ? tx : nx);
  const int row_tile = Sp->row_tile;
  const int x0 = tile * row_tile;
  const int nrows = min(row_tile, rows_total - x0);
  const int npairs = (nrows + 1) >> 1;
  const FastDiv dny = Sp->dv_ny, dnyh = Sp->dv_nyh;
  const C* __restrict__ spec = Sp->spec;
  struct XY { C X, Y; };
  batched_loop<4>(npairs * nyh, [&](int e) {
    const int p = fdiv(dnyh, e), k = e - p * nyh;
    const int xa = x0 + 2 * p;
    XY v;
    v.X = ldf(spec + spec_at(xa, k, nx, lw));
    v.Y = (xa + 1 < x0 + nrows) ? ldf(spec + spec_at(xa + 1, k, nx, lw)) : czero<C>();
    return v;
  }, [&](int e, XY v) {
    const int p = fdiv(dnyh, e), k = e - p * nyh;
    C X = v.X, Y = v.Y;
    const bool selfconj = (k == 0) || (2 * k == ny);
    if (selfconj) { X.y = 0; Y.y = 0; }
    buf[p * ny + k] = cmake<C>(X.x - Y.y, X.y + Y.x);
    if (!selfconj) buf[p * ny + ny - k] = cmake<C>(X.x + Y.y, Y.x - X.y);
  });
  __syncthreads();
  const C* res = fft_smem<C, true>(buf, scratch, fd, npairs, ny, 1, false, tws);
  if (MODE == MODE_PLAIN) {
    R* __restrict__ out = Sp->out;
    const int out_cols = Sp->out_cols, out_ld = Sp->out_ld;
    for (int e = threadIdx.x; e < npairs * ny; e += blockDim.x) {
      const int p = fdiv(dny, e), y = e - p * ny;
      if (y >= out_cols) continue;
      const C z = res[e];
      const int xa = x0 + 2 * p;
      out[(size_t)xa * out_ld + y] = z.x;
      if (xa + 1 < x0 + nrows) out[(size_t)(xa + 1) * out_ld + y] = z.y;
    }
  } else if (MODE == MODE_T) {
    const R* __restrict__ t = Sp->t;
    struct T2 { R a, b; };
    batched_loop<4>(npairs * ny, [&](int e) {
      const int p = fdiv(dny, e), y = e - p * ny;
      const int xa = x0 + 2 * p;
      T2 v{0, 0};
      if (y < ty) {
        v.a = ldf(t + (size_t)xa * ty + y);
        if (xa + 1 < x0 + nrows) v.b = ldf(t + (size_t)(xa + 1) * ty + y);
      }
      return v;
    }, [&](int e, T2 v) {
      const C z = res[e];
      a0 += (double)z.x * (double)v.a + (double)z.y * (double)v.b;
    });
  } else {
    R* __restrict__ u = Sp->u;
    const R* __restrict__ h = Sp->h;
    const R* __restrict__ fa_buf = Sp->f[cv.par];
    const unsigned char* __restrict__ gneg = Sp->gneg;
    const R off = (R)cv.offset;
    struct UF { R uo[2], fa[2], h[2]; unsigned char gn[2]; };
    batched_loop<2>(npairs * ny, [&](int e) {
      const int p = fdiv(dny, e), y = e - p * ny;
      UF v;
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const int x = x0 + 2 * p + w;
        v.uo[w] = 0; v.fa[w] = 0; v.h[w] = 0; v.gn[w] = 0;
        if (x >= x0 + nrows) continue;
        v.uo[w] = ldf(u + (size_t)x * ny + y);
        if (x < tx && y < ty) {
          const size_t ic = (size_t)x * ty + y;
          v.h[w] = ldf(h + ic);
          if (cv.branch == 0) v.fa[w] = ldf(fa_buf + ic);
          else v.gn[w] = ldf(gneg + ic);
        }
      }
      return v;
    }, [&](int e, const UF& v) {
      const int p = fdiv(dny, e), y = e - p * ny;
      const C z = res[e];
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const int x = x0 + 2 * p + w;
        if (x >= x0 + nrows) continue;
        const R val = w ? z.y : z.x;
        a0 = fmax(a0, (double)fabs(val - v.uo[w]));
        u[(size_t)x * ny + y] = val;
        if (x < tx && y < ty) {
          bool c;
          if (cv.branch == 0) c = (v.fa[w] < 0) && (!cv.has_h || (double)v.fa[w] > -cv.H);
          else c = v.gn[w] != 0;
          const R pen = (v.h[w] + off) - val;
          a1 = fmax(a1, c ? (double)pen : 0.0);
        }
      }
    });
  }
}

template <typename R, int MODE>
__global__ void __launch_bounds__(CM_FFT_THREADS)
k_row_inv(const Slot<R>* __restrict__ slots, const int2* __restrict__ items) {
  typedef typename CT<R>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FftDesc fd;
  const int2 item = items[blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  CcgView cv{};
  if (MODE == MODE_T || MODE == MODE_F) {
    if (st->done) return;
    if (MODE == MODE_T && st->branch != 0) return;
    load_view(st, cv);
  }
  const int ny = Sp->ny;
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* buf = tws + ny;
  C* scratch = buf + (Sp->row_tile >> 1) * ny;
  stage_fft(fd, Sp->fy, tws, Sp->twy, ny);
  double a0 = 0.0, a1 = -INFINITY;  // MODE_T: sum r t ; MODE_F: max|du|, max penetration
  row_inv_tile<R, MODE>(Sp, cv, item.y, fd, tws, buf, scratch, a0, a1);
  if (MODE == MODE_T) {
    double v[1] = {a0};
    const int kinds[1] = {RED_SUM};
    tile_finish<1>(Sp->partials, Sp->counter, item.y, Sp->nt_rowt, v, kinds,
                   [&](double (&a)[1]) { fin_tau(*st, a); });
  } else if (MODE == MODE_F) {
    double v[2] = {a0, a1};
    const int kinds[2] = {RED_MAX, RED_MAX};
    tile_finish<2>(Sp->partials, Sp->counter, item.y, Sp->nt_rowd, v, kinds,
                   [&](double (&a)[2]) { ccg_converge(*st, a[0], a[1]); });
  }
}

// ---------------------------------------------------------------------------
// CCG element-wise kernels over the topography region
// ---------------------------------------------------------------------------
// Fields of one comp tile (rows [cx0, cx0+crows) of the topography) in registers.
template <typename R>
struct CompTile {
  int cx0, cn, ty, ny;
  FastDiv dty;
  const R* __restrict__ u;
  const R* __restrict__ h;
  CM_DEVINL CompTile(const Slot<R>* Sp, int tile) {
    ty = Sp->ty;
    ny = Sp->ny;
    dty = Sp->dv_ty;
    cx0 = tile * Sp->comp_rows;
    cn = min(Sp->comp_rows, Sp->tx - cx0) * ty;
    u = Sp->u;
    h = Sp->h;
  }
  // topography index and displacement index of element e of the tile
  CM_DEVINL void at(int e, size_t& ic, size_t& iu) const {
    const int r = fdiv(dty, e), y = e - r * ty;
    ic = (size_t)cx0 * ty + e;
    iu = (size_t)(cx0 + r) * ny + y;
  }
};

// The element-wise passes run in one of two shapes.  With strided == 0 a
// block takes work item items[blockIdx.x] (a (solve, tile) pair: batched
// solves share a launch) and writes one partial per tile.  With strided = n
// > 0 every item is a tile of the one solve of items[0], the block walks
// tiles blockIdx.x, blockIdx.x + gridDim.x, ... < n and writes one partial
// for all of them (fewer blocks and partials for a single solve).
struct EwTiles {
  int first, end, step, part, nparts;
  CM_DEVINL EwTiles(int2 item, int strided, int nt_comp) {
    if (strided > 0) {
      first = blockIdx.x; end = strided; step = gridDim.x;
      part = blockIdx.x; nparts = gridDim.x;
    } else {
      first = item.y; end = item.y + 1; step = 1;
      part = item.y; nparts = nt_comp;
    }
  }
};

// Start of an iteration over one comp tile: contact areas and raw-gap sums
// (counts in int and extrema in R are exact; only the sum is FP64).
template <typename R>
CM_DEVINL void begin_tile(const Slot<R>* __restrict__ Sp, int tile, const R* __restrict__ f,
                          int has_h, R hdn, int& a_c, int& a_cg, double& s_cg, R& gmax, R& gmin) {
  struct V3 { R f, u, h; };
  const CompTile<R> T(Sp, tile);
  batched_loop<sizeof(R) == 8 ? 4 : 8>(T.cn, [&](int e) {
    size_t ic, iu;
    T.at(e, ic, iu);
    return V3{ldf(f + ic), ldf(T.u + iu), ldf(T.h + ic)};
  }, [&](int, V3 v) {
    const bool c0 = v.f < 0;
    const bool c = c0 && (!has_h || v.f > hdn);
    const R g = v.u - v.h;
    a_c += c0;
    a_cg += c;
    if (c) s_cg += (double)g;
    gmax = fmax(gmax, g);
    gmin = fmin(gmin, g);
  });
}

// Start of an iteration: contact areas, raw-gap sums, step kind and offset
// (ConstrainedConjugateGradients.py:239-270, 300-318).
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_begin(const Slot<R>* __restrict__ slots, const int2* __restrict__ items, int strided) {
  const int2 item = items[strided > 0 ? 0 : blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  // the slot (geometry, field pointers) is constant during a solve: read it
  // before waiting for the previous kernel
  const EwTiles W(item, strided, Sp->nt_comp);
  R* const f0 = Sp->f[0];
  R* const f1 = Sp->f[1];
  pdl_trigger();
  pdl_wait();
  if (st->done) return;
  const int has_h = st->p.has_h;
  const R hdn = neg_down<R>(st->p.H);
  const R* __restrict__ f = (st->parity & 1) ? f1 : f0;
  int a_c = 0, a_cg = 0;
  double s_cg = 0;
  R gmax = -INFINITY, gmin = INFINITY;
  for (int tile = W.first; tile < W.end; tile += W.step)
    begin_tile<R>(Sp, tile, f, has_h, hdn, a_c, a_cg, s_cg, gmax, gmin);
  double v[5] = {(double)a_c, (double)a_cg, s_cg, (double)gmax, (double)gmin};
  const int kinds[5] = {RED_SUM, RED_SUM, RED_SUM, RED_MAX, RED_MIN};
  tile_finish<5>(Sp->partials, Sp->counter, W.part, W.nparts, v, kinds,
                 [&](double (&a)[5]) { fin_begin(*st, a); });
}

// G over one comp tile: sum over the CG area of g^2.
template <typename R>
CM_DEVINL void gsum_tile(const Slot<R>* __restrict__ Sp, int tile, const R* __restrict__ f,
                         int has_h, R hdn, R off, double& G) {
  struct V3 { R f, u, h; };
  const CompTile<R> T(Sp, tile);
  batched_loop<sizeof(R) == 8 ? 4 : 8>(T.cn, [&](int e) {
    size_t ic, iu;
    T.at(e, ic, iu);
    return V3{ldf(f + ic), ldf(T.u + iu), ldf(T.h + ic)};
  }, [&](int, V3 v) {
    const bool c = (v.f < 0) && (!has_h || v.f > hdn);
    const R g = (v.u - v.h) - off;
    // the reference sums c * g^2 over the whole topography, so a NaN gap
    // outside the contact set makes G NaN as well (0 * NaN)
    if (c) G += (double)g * (double)g;
    else if (isnan(g)) G += (double)g;
  });
}

// G = sum over the CG area of g^2 and the conjugation factor (:273-279).
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_gsum(const Slot<R>* __restrict__ slots, const int2* __restrict__ items, int strided) {
  const int2 item = items[strided > 0 ? 0 : blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  const EwTiles W(item, strided, Sp->nt_comp);
  R* const f0 = Sp->f[0];
  R* const f1 = Sp->f[1];
  pdl_trigger();
  pdl_wait();
  if (st->done || st->branch != 0) return;
  const int has_h = st->p.has_h;
  const R hdn = neg_down<R>(st->p.H);
  const R off = (R)st->offset;
  const R* __restrict__ f = (st->parity & 1) ? f1 : f0;
  double G = 0;
  for (int tile = W.first; tile < W.end; tile += W.step) gsum_tile<R>(Sp, tile, f, has_h, hdn, off, G);
  double v[1] = {G};
  const int kinds[1] = {RED_SUM};
  tile_finish<1>(Sp->partials, Sp->counter, W.part, W.nparts, v, kinds,
                 [&](double (&a)[1]) { fin_gsum(*st, a); });
}

// One pass of the load-controlled offset bisection of the mixing step
// (ConstrainedConjugateGradients.py:316-318).  Counts #(g < x) for up to 31
// candidate midpoints, i.e. the next five levels of scipy's bisection tree,
// then replays scipy's bisection on those counts bit for bit.
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_bisect(const Slot<R>* __restrict__ slots, const int2* __restrict__ items, int strided) {
  const int2 item = items[strided > 0 ? 0 : blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  const EwTiles W(item, strided, Sp->nt_comp);
  pdl_trigger();
  pdl_wait();
  if (st->done || st->branch != 1 || !st->bs_active) return;
  __shared__ double cand[CM_BIS_CAND];
  __shared__ double cand_lo, cand_hi;
  const int ncand = (st->bs_iter < 0) ? 1 : CM_BIS_CAND;
  if (threadIdx.x < ncand) cand[threadIdx.x] = st->bs_cand[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    double lo = cand[0], hi = cand[0];
    for (int i = 1; i < ncand; ++i) {
      lo = fmin(lo, cand[i]);
      hi = fmax(hi, cand[i]);
    }
    cand_lo = lo;
    cand_hi = hi;
  }
  __syncthreads();
  // g below every candidate counts for all of them, g at or above every
  // candidate for none (for doubles, g - c < 0 exactly when g < c); only gaps
  // inside the candidates' bracket, which shrinks 32-fold per pass, are
  // compared one by one
  const double lo = cand_lo, hi = cand_hi;
  int below_all = 0;
  int icnt[CM_BIS_CAND];  // counts: exact in int
#pragma unroll
  for (int i = 0; i < CM_BIS_CAND; ++i) icnt[i] = 0;
  struct V2 { R u, h; };
  for (int tile = W.first; tile < W.end; tile += W.step) {
    const CompTile<R> T(Sp, tile);
    batched_loop<4>(T.cn, [&](int e) {
      size_t ic, iu;
      T.at(e, ic, iu);
      return V2{T.u[iu], T.h[ic]};
    }, [&](int, V2 v) {
      const double g = (double)(v.u - v.h);
      if (g < lo) {
        ++below_all;
      } else if (g < hi) {
#pragma unroll
        for (int i = 0; i < CM_BIS_CAND; ++i)
          if (i < ncand) icnt[i] += (g - cand[i] < 0.0) ? 1 : 0;
      }
    });
  }
  double cnt[CM_BIS_CAND];
#pragma unroll
  for (int i = 0; i < CM_BIS_CAND; ++i) cnt[i] = (double)(icnt[i] + (i < ncand ? below_all : 0));
  int kinds[CM_BIS_CAND];
#pragma unroll
  for (int i = 0; i < CM_BIS_CAND; ++i) kinds[i] = RED_SUM;
  tile_finish<CM_BIS_CAND>(Sp->partials, Sp->counter, W.part, W.nparts, cnt, kinds,
                           [&](double (&a)[CM_BIS_CAND]) { fin_bisect(*st, a); });
}

// All the bisection passes of one iteration in one launch (single solves):
// the blocks walk the solve's tiles as k_ccg_bisect's strided shape does,
// the last block of each pass advances the bisection (fin_bisect), and a
// grid barrier separates the passes, so an iteration without a mixing step
// costs one launch instead of CM_BISECT_PASSES.  Launched cooperatively
// (every block resident); the barrier's waits are bounded.
template <typename R>
__global__ void __launch_bounds__(CM_THREADS)
k_ccg_bisect_passes(const Slot<R>* __restrict__ slots, const int2* __restrict__ items, int ntiles,
                    GridBarrier* bar) {
  const Slot<R>* __restrict__ Sp = slots + items[0].x;
  CcgState* st = Sp->st;
  pdl_trigger();
  pdl_wait();
  __shared__ double cand[CM_BIS_CAND];
  __shared__ double cand_lo, cand_hi;
  __shared__ int go, ncand_s, ok_sm;
  unsigned gen = 0;
  if (threadIdx.x == 0) gen = ld_acquire_gpu(&bar->gen);
  for (int pass = 0; pass < CM_BISECT_PASSES; ++pass) {
    if (threadIdx.x == 0) {
      // the state as the previous pass's last block left it, past this SM's L1
      go = __ldcg(&st->done) == 0 && __ldcg(&st->branch) == 1 && __ldcg(&st->bs_active) != 0;
      ncand_s = __ldcg(&st->bs_iter) < 0 ? 1 : CM_BIS_CAND;
    }
    __syncthreads();
    if (!go) break;
    const int ncand = ncand_s;
    if (threadIdx.x < ncand) cand[threadIdx.x] = __ldcg(&st->bs_cand[threadIdx.x]);
    __syncthreads();
    if (threadIdx.x == 0) {
      double lo = cand[0], hi = cand[0];
      for (int i = 1; i < ncand; ++i) {
        lo = fmin(lo, cand[i]);
        hi = fmax(hi, cand[i]);
      }
      cand_lo = lo;
      cand_hi = hi;
    }
    __syncthreads();
    const double lo = cand_lo, hi = cand_hi;
    int below_all = 0;
    int icnt[CM_BIS_CAND];
#pragma unroll
    for (int i = 0; i < CM_BIS_CAND; ++i) icnt[i] = 0;
    struct V2 { R u, h; };
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      const CompTile<R> T(Sp, tile);
      batched_loop<4>(T.cn, [&](int e) {
        size_t ic, iu;
        T.at(e, ic, iu);
        return V2{T.u[iu], T.h[ic]};
      }, [&](int, V2 v) {
        const double g = (double)(v.u - v.h);
        if (g < lo) {
          ++below_all;
        } else if (g < hi) {
#pragma unroll
          for (int i = 0; i < CM_BIS_CAND; ++i)
            if (i < ncand) icnt[i] += (g - cand[i] < 0.0) ? 1 : 0;
        }
      });
    }
    double cnt[CM_BIS_CAND];
#pragma unroll
    for (int i = 0; i < CM_BIS_CAND; ++i) cnt[i] = (double)(icnt[i] + (i < ncand ? below_all : 0));
    int kinds[CM_BIS_CAND];
#pragma unroll
    for (int i = 0; i < CM_BIS_CAND; ++i) kinds[i] = RED_SUM;
    tile_finish<CM_BIS_CAND>(Sp->partials, Sp->counter, blockIdx.x, gridDim.x, cnt, kinds,
                             [&](double (&a)[CM_BIS_CAND]) { fin_bisect(*st, a); });
    if (!grid_barrier(bar, gen, &ok_sm)) {
      if (threadIdx.x == 0) {
        st->status = CMS_TIMEOUT;
        st->done = 1;
      }
      break;
    }
  }
}

// Reduction values of the force update (counts in int and extrema in R are
// exact: x -> (double)x + H is monotonic, so the minimum of fn + H is the
// minimum fn plus H; only the sum is FP64).
template <typename R>
struct UpdateAcc {
  int a_fl = 0, n_nc = 0;
  R min_fn = INFINITY, max_t = 0;
  double s_fp = 0;
};

// Force update and projection over one comp tile: f (start of the
// iteration) -> fo.
template <typename R>
CM_DEVINL void update_tile(const Slot<R>* __restrict__ Sp, int tile, const R* __restrict__ f,
                           R* __restrict__ fo, int has_h, int branch, double H, R hdn, R off,
                           R tau, double mix, UpdateAcc<R>& A) {
  const R* __restrict__ t = Sp->t;
  unsigned char* __restrict__ gneg = Sp->gneg;
  struct V4 { R f, u, h, t; };
  const CompTile<R> T(Sp, tile);
  batched_loop<sizeof(R) == 8 ? 4 : 8>(T.cn, [&](int e) {
    size_t ic, iu;
    T.at(e, ic, iu);
    return V4{ldf(f + ic), ldf(T.u + iu), ldf(T.h + ic), branch == 0 ? ldf(t + ic) : (R)0};
  }, [&](int e, V4 v) {
    const size_t ic = (size_t)T.cx0 * T.ty + e;
    const R fa = v.f;
    const R g = (v.u - v.h) - off;
    R fn;
    if (branch == 0) {
      const bool c = (fa < 0) && (!has_h || fa > hdn);
      fn = c ? (R)(fa + tau * v.t) : fa;
    } else {
      fn = (R)((R)(1 - mix) * fa - (g < 0 ? (R)(mix * H) : (R)0));
    }
    const bool tensile = fn >= 0;
    const bool flowing = has_h && fn <= hdn;
    const bool nc = (tensile && g < 0) || (flowing && g > 0);
    if (tensile) A.max_t = fmax(A.max_t, fn);
    if (flowing) { A.a_fl += 1; A.min_fn = fmin(A.min_fn, fn); }
    const R fp = tensile ? (R)0 : fn;
    A.s_fp += (double)fp;
    A.n_nc += nc;
    fo[ic] = fp;
    if (has_h) gneg[ic] = g < 0;
  });
}

// Force update, projection onto [0, H], constraint bookkeeping
// (ConstrainedConjugateGradients.py:296, 320-389).
template <typename R>
__global__ void __launch_bounds__(CM_THREADS, sizeof(R) == 4 ? 4 : 3)
k_ccg_update(const Slot<R>* __restrict__ slots, const int2* __restrict__ items, int strided) {
  const int2 item = items[strided > 0 ? 0 : blockIdx.x];
  const Slot<R>* __restrict__ Sp = slots + item.x;
  CcgState* st = Sp->st;
  const EwTiles W(item, strided, Sp->nt_comp);
  R* const f0 = Sp->f[0];
  R* const f1 = Sp->f[1];
  pdl_trigger();
  pdl_wait();
  if (st->done) return;
  const int par = st->parity & 1, has_h = st->p.has_h, branch = st->branch;
  const double H = st->p.H;
  const R off = (R)st->offset;
  const R tau = (R)st->tau;
  const double mix = st->cur_mixfac;
  const R* __restrict__ f = par ? f1 : f0;
  R* __restrict__ fo = par ? f0 : f1;
  const R hdn = neg_down<R>(H);
  UpdateAcc<R> A;
  for (int tile = W.first; tile < W.end; tile += W.step)
    update_tile<R>(Sp, tile, f, fo, has_h, branch, H, hdn, off, tau, mix, A);
  double v[5] = {(double)A.a_fl, (double)A.min_fn + H, (double)A.max_t, A.s_fp, (double)A.n_nc};
  const int kinds[5] = {RED_SUM, RED_MIN, RED_MAX, RED_SUM, RED_SUM};
  tile_finish<5>(Sp->partials, Sp->counter, W.part, W.nparts, v, kinds,
                 [&](double (&a)[5]) { fin_update(*st, a); });
}

// ---------------------------------------------------------------------------
// solve preparation and results (per comp tile)
// ---------------------------------------------------------------------------
// heights -> working precision over one comp tile; max, min and sum of the
// FP64 heights.
template <typename R>
CM_DEVINL void h_prep_tile(const Slot<R>* __restrict__ Sp, int tile, const double* __restrict__ h64,
                           double& mx, double& mn, double& sm) {
  const CompTile<R> T(Sp, tile);
  R* __restrict__ h = const_cast<R*>(Sp->h);
  const size_t base = (size_t)T.cx0 * T.ty;
  for (int e = threadIdx.x; e < T.cn; e += blockDim.x) {
    const double hv = h64[base + e];
    h[base + e] = (R)hv;
    mx = fmax(mx, hv);
    mn = fmin(mn, hv);
    sm += hv;
  }
}

CM_DEVINL void fin_h_prep(CcgState& s, double (&a)[3]) {
  s.p.max_surface = a[0];
  s.gmin = a[1];  // scratch until the loop starts
  s.sum_cg = a[2];
}

// sum of squared deviations from the mean height over one comp tile
template <typename R>
CM_DEVINL void h_var_tile(const Slot<R>* __restrict__ Sp, int tile, const double* __restrict__ h64,
                          double mean, double& v2) {
  const CompTile<R> T(Sp, tile);
  const size_t base = (size_t)T.cx0 * T.ty;
  for (int e = threadIdx.x; e < T.cn; e += blockDim.x) {
    const double d = h64[base + e] - mean;
    v2 += d * d;
  }
}

// rms height and the reference's default penetration tolerance
// (ConstrainedConjugateGradients.py:150-162); FP32 phases widen pentol.
CM_DEVINL void fin_h_var(CcgState& s, double (&a)[1], int pentol_auto, double rel_pentol, int tx,
                         int ty) {
  if (pentol_auto) {
    const double rms = sqrt(a[0] / s.p.n_surface);
    double pt = rms / (10.0 * (0.5 * ((double)tx + (double)ty)));
    if (pt == 0) pt = (s.p.offset0 + s.sum_cg / s.p.n_surface) / 1000;
    if (pt == 0) pt = 1e-3;
    s.p.pentol = pt;
  }
  if (rel_pentol > 0) s.p.pentol = fmax(s.p.pentol, rel_pentol * (s.p.max_surface - s.gmin));
  s.gmin = 0;
  s.sum_cg = 0;
}

// initial displacement at domain index i: given or zero, lifted onto the
// surface on the topography region (ConstrainedConjugateGradients.py:168-201)
template <typename R>
CM_DEVINL void init_u_at(const Slot<R>& S, const double* __restrict__ u0, double offset, long i) {
  const int x = (int)(i / S.ny), y = (int)(i % S.ny);
  double u = u0 ? u0[i] : 0.0;
  if (x < S.tx && y < S.ty) {
    const double lo = (double)ldf(S.h + (size_t)x * S.ty + y) + offset;
    u = (u < lo) ? lo : u;
  }
  S.u[i] = (R)u;
}

// result.jac, active_set, plastic over one comp tile, with the sums of the
// elastic energy and the contact areas (ConstrainedConjugateGradients.py
// :454-475, 494-509)
template <typename R>
CM_DEVINL void result_tile(const Slot<R>* __restrict__ Sp, int tile, int par, int has_h,
                           int mixing, double H, double* jac, unsigned char* active,
                           unsigned char* plastic, double (&v)[4]) {
  const R* __restrict__ ff = Sp->f[par];       // final force
  const R* __restrict__ fa = Sp->f[par ^ 1];   // force at the start of the last iteration
  const unsigned char* __restrict__ gneg = Sp->gneg;
  const CompTile<R> T(Sp, tile);
  for (int e = threadIdx.x; e < T.cn; e += blockDim.x) {
    size_t ic, iu;
    T.at(e, ic, iu);
    const R f = ldf(ff + ic);
    const R u = ldf(T.u + iu);
    v[0] += (double)f * (double)u;
    if (jac) jac[ic] = -(double)f;
    v[1] += (f < 0);
    bool act;
    if (mixing) act = ldf(gneg + ic) != 0;
    else {
      const R a = ldf(fa + ic);
      act = (a < 0) && (!has_h || (double)a > -H);
    }
    v[2] += act;
    if (active) active[ic] = act;
    if (has_h) {
      const bool p = ldf(gneg + ic) != 0;
      v[3] += p;
      if (plastic) plastic[ic] = p;
    }
  }
}

CM_DEVINL void fin_result(CcgState& s, double (&a)[4]) {
  s.sum_cgt = -a[0] / 2;  // result.fun
  s.A_contact = (long long)a[1];
  s.A_cg = (long long)a[2];
  s.A_fl = (long long)a[3];
}
