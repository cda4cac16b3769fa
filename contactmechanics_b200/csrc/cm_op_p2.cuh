// The elastic operator u = IFFT(T . FFT(f)) (FFTElasticHalfSpace.py:573-611,
// free :1141-1197) for power-of-two domains (sides 64..4096), as three
// bandwidth-oriented passes over caller buffers:
//
//   k_op_row_fwd  rows x < in_rows: packed real-to-complex row transforms
//                 (two rows per complex transform), half spectrum written
//                 into the plan's column-tiled spectrum;
//   k_op_col16    every column tile: forward transform along x (input rows
//                 >= in_rows are zero), times the real Green's table,
//                 inverse transform, rows < out_rows written back;
//   k_op_row_inv  rows x < out_rows: complex-to-real row transforms, output
//                 columns < out_cols written to the caller's buffer.
//
// Arguments travel by value (no descriptor upload), so a call is a plain
// sequence of three launches on the caller's stream.  Blocks walk their
// tiles with a grid stride, so the twiddle tables are staged once per block.
// A block covers 2*NP rows (row passes, N/E threads per transform with E =
// 8 elements per thread by default) or several column tiles (column pass,
// N/16 threads per transform), the register-resident engines of
// cm_fft_p2.cuh.  Spectrum stores and gathers are ordered so that a warp
// touches whole rows-of-a-tile runs: (row, column-in-tile) fastest, which in
// the plan's layout ((k >> lw) * nx + x) * W + (k & (W-1)) are contiguous.
#pragma once
#include "cm_fft_p2.cuh"
#include "cm_kernels.cuh"
#include "cm_launch.h"

// resident blocks per SM the FP64 row passes are compiled for: two blocks
// of 256 threads (at most 128 registers a thread) hide more latency than one
#ifndef CM_FP64_ROW_MINB
#define CM_FP64_ROW_MINB 2
#endif

// threads of an FP64 column-pass block (at least one transform): 128, so
// that two blocks fit an SM's shared memory at length 2048
#ifndef CM_COL16_FP64_BASE
#define CM_COL16_FP64_BASE 128
#endif

// threads of an FP32 row-pass block (at least one transform) and the
// resident blocks per SM it is compiled for
#ifndef CM_ROW_F32_BASE
#define CM_ROW_F32_BASE 512
#endif
#ifndef CM_ROW_F32_MINB
#define CM_ROW_F32_MINB 2
#endif

// threads of an FP32 column-pass block and its resident blocks per SM
#ifndef CM_COL16_F32_BASE
#define CM_COL16_F32_BASE 256
#endif
#ifndef CM_COL16_F32_MINB
#define CM_COL16_F32_MINB 2
#endif

// log2 of the elements per thread of the row passes' transforms (3: the
// radix-8 engine, 4: the radix-16 one)
#ifndef CM_ROW_LR_F32
#define CM_ROW_LR_F32 3
#endif
#ifndef CM_ROW_LR_F64
#define CM_ROW_LR_F64 3
#endif

// threads of one block of the row passes for transform length 2^LOGN
template <typename R, int LOGN>
struct OpShape {
  static constexpr int N = 1 << LOGN;
  static constexpr int LR = sizeof(R) == 8 ? CM_ROW_LR_F64 : CM_ROW_LR_F32;
  static constexpr int E = 1 << LR;  // elements per thread
  static constexpr int TPS = N >> LR;
  static constexpr int BASE = (sizeof(R) == 8 ? 256 : CM_ROW_F32_BASE) >> (LR - 3);
  static constexpr int THREADS = TPS > BASE ? TPS : BASE;
  static constexpr int NP = THREADS / TPS;  // sequences (row pairs, columns) per block
  static constexpr int MINB = sizeof(R) == 8 ? CM_FP64_ROW_MINB : CM_ROW_F32_MINB;
  // block strides of a row-pair gather whose loads are issued together (the
  // gather of a row tile with column tiles W <= N/8 takes at most five); the
  // FP64 passes have the registers to spare, the FP32 ones do not
  static constexpr int GATHER = sizeof(R) == 8 ? 5 : 1;
  static constexpr int LNP = NP >= 512 ? 9 : NP >= 256 ? 8 : NP >= 128 ? 7 : NP >= 64 ? 6 : NP >= 32 ? 5
                             : NP >= 16 ? 4 : NP >= 8 ? 3 : NP >= 4 ? 2 : NP >= 2 ? 1 : 0;
  static size_t smem() {
    return (size_t)(N + 2 * smem_padded(NP * N)) * sizeof(typename CT<R>::C);
  }
};

// Gathers the half spectra of the row pairs x0 + 2p, x0 + 2p + 1 (p < NP,
// rows >= rows_total read as zero) from the column-tiled spectrum and packs
// each pair into one full-length complex sequence in buf (Z = X + iY with the
// Hermitian halves filled in).  Element e = ((kb * NP) + p) * W + kw; the
// loads of U consecutive strides are issued before any of them is used, so a
// thread has 2U loads in flight.
template <typename C, int LOGN, int NP, int LNP, int U>
CM_DEVINL void gather_row_pairs(C* buf, const C* __restrict__ spec, int nx, int nyh, int lw,
                                int x0, int rows_total) {
  constexpr int N = 1 << LOGN;
  const int W = 1 << lw, nkb = (nyh + W - 1) >> lw;
  const int total = nkb * NP * W;
  const int T = blockDim.x;
  for (int e0 = threadIdx.x; e0 < total; e0 += U * T) {
    C X[U], Y[U];
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const int e = e0 + i * T;
      const int kw = e & (W - 1);
      const int p = (e >> lw) & (NP - 1);
      const int kb = e >> (lw + LNP);
      const int k = kb * W + kw, xa = x0 + 2 * p;
      X[i] = czero<C>();
      Y[i] = czero<C>();
      if (e >= total || k >= nyh || xa >= rows_total) continue;
      const size_t ia = ((size_t)kb * nx + xa) * W + kw;
      X[i] = spec[ia];
      if (xa + 1 < rows_total) Y[i] = spec[ia + W];
    }
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const int e = e0 + i * T;
      const int kw = e & (W - 1);
      const int p = (e >> lw) & (NP - 1);
      const int kb = e >> (lw + LNP);
      const int k = kb * W + kw, xa = x0 + 2 * p;
      if (e >= total || k >= nyh || xa >= rows_total) continue;
      C x = X[i], y = Y[i];
      const bool selfconj = (k == 0) || (2 * k == N);
      if (selfconj) { x.y = 0; y.y = 0; }
      buf[spad(p * N + k)] = cmake<C>(x.x - y.y, x.y + y.x);
      if (!selfconj) buf[spad(p * N + N - k)] = cmake<C>(x.x + y.y, y.x - x.y);
    }
  }
}

template <typename R, int LOGN>
__global__ void __launch_bounds__(OpShape<R, LOGN>::THREADS, OpShape<R, LOGN>::MINB)
k_op_row_fwd(OpArgs<R> a) {
  typedef typename CT<R>::C C;
  typedef P2PlanR<LOGN, OpShape<R, LOGN>::LR> P;
  typedef OpShape<R, LOGN> Sh;
  constexpr int N = P::N, NP = Sh::NP, ROWS = 2 * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = tws + N;
  C* bufB = bufA + smem_padded(NP * N);
  pdl_trigger();
  stage_tw_p2r<LOGN, Sh::LR>(tws, a.twy);
  pdl_wait();
  __syncthreads();
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const int W = 1 << a.lw, nkb = (a.nyh + W - 1) >> a.lw;
  const int ntiles = (a.in_rows + ROWS - 1) / ROWS;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int x0 = tile * ROWS, xa = x0 + 2 * s;
    C v[Sh::E];
#pragma unroll
    for (int q = 0; q < Sh::E; ++q) {
      const int y = tt + q * P::TPS;
      R ra = 0, rb = 0;
      if (y < a.in_cols) {
        if (xa < a.in_rows) ra = __ldg(a.in + (size_t)xa * a.in_ld + y);
        if (xa + 1 < a.in_rows) rb = __ldg(a.in + (size_t)(xa + 1) * a.in_ld + y);
      }
      v[q] = cmake<C>(ra, rb);
    }
    fft_p2r<C, false, LOGN, Sh::LR>(v, bufA, bufB, s * N, 1, tt, tws);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Sh::E; ++q) bufA[spad(s * N + tt + q * P::TPS)] = v[q];
    __syncthreads();
    // split the packed transforms; e = ((kb * ROWS) + r) * W + kw
    const int total = nkb * ROWS * W;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int kw = e & (W - 1);
      const int r = (e >> a.lw) & (ROWS - 1);
      const int kb = e >> (a.lw + Sh::LNP + 1);
      const int k = kb * W + kw, x = x0 + r;
      if (k >= a.nyh || x >= a.in_rows) continue;
      const int p = r >> 1;
      const C z = bufA[spad(p * N + k)];
      const C zm = bufA[spad(p * N + ((N - k) & (N - 1)))];
      const C val = (r & 1) ? cmake<C>((z.y + zm.y) * (R)0.5, (zm.x - z.x) * (R)0.5)
                            : cmake<C>((z.x + zm.x) * (R)0.5, (z.y - zm.y) * (R)0.5);
      a.spec[((size_t)kb * a.nx + x) * W + kw] = val;
    }
    __syncthreads();  // bufA free for the next tile
  }
}

// Column pass with 16 elements per thread (radix-16 stages, fft_p2r): two
// shared-memory exchanges per transform of length 2048 instead of the three
// of the 8-element engine.
template <typename R, int LOGN>
struct OpShape16 {
  static constexpr int N = 1 << LOGN;
  static constexpr int TPS = N / 16;
  static constexpr int BASE = sizeof(R) == 8 ? CM_COL16_FP64_BASE : CM_COL16_F32_BASE;
  static constexpr int THREADS = TPS > BASE ? TPS : BASE;
  static constexpr int NP = THREADS / TPS;  // columns per block
  static constexpr int MINB = sizeof(R) == 4 ? CM_COL16_F32_MINB : (BASE < 256 ? 2 : 1);
  static size_t smem() {
    return (size_t)(N + 2 * smem_padded(NP * N)) * sizeof(typename CT<R>::C);
  }
};

template <typename R, int LOGN>
__global__ void __launch_bounds__(OpShape16<R, LOGN>::THREADS, OpShape16<R, LOGN>::MINB)
k_op_col16(OpArgs<R> a) {
  typedef typename CT<R>::C C;
  typedef P2PlanR<LOGN, 4> P;
  typedef OpShape16<R, LOGN> Sh;
  constexpr int N = P::N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = tws + N;
  C* bufB = bufA + smem_padded(Sh::NP * N);
  pdl_trigger();
  stage_tw_p2r<LOGN, 4>(tws, a.twx);
  pdl_wait();
  if (a.st && (a.st->done || (a.cg_only && a.st->branch != 0))) return;
  __syncthreads();
  const int lw = a.lw, W = 1 << lw;
  const int c = threadIdx.x & (W - 1);
  const int tt = (threadIdx.x >> lw) & (P::TPS - 1);
  const int j = threadIdx.x >> (lw + P::LTPS);
  const int tiles_per_block = blockDim.x >> (lw + P::LTPS);
  const int ngroups = (a.ntile_cols + tiles_per_block - 1) / tiles_per_block;
  const int base = j * N * W + c;
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const int tile = grp * tiles_per_block + j;
    const bool tile_ok = tile < a.ntile_cols;
    const int wc = tile_ok ? min(W, a.nyh - tile * W) : 0;
    const bool col_ok = c < wc;
    C* __restrict__ blk = a.spec + (size_t)tile * N * W;
    const R* __restrict__ tblk = a.tab + (size_t)tile * N * W;
    C v[16];
    R g[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int x = tt + q * P::TPS;
      v[q] = (col_ok && x < a.in_rows) ? blk[x * W + c] : czero<C>();
      g[q] = col_ok ? __ldg(tblk + x * W + c) : (R)0;
    }
    fft_p2r<C, false, LOGN, 4>(v, bufA, bufB, base, W, tt, tws);
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = cscale(v[q], g[q]);
    __syncthreads();
    fft_p2r<C, true, LOGN, 4>(v, bufA, bufB, base, W, tt, tws);
    if (col_ok) {
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int x = tt + q * P::TPS;
        if (x < a.out_rows) blk[x * W + c] = v[q];
      }
    }
    __syncthreads();  // buffers free for the next group
  }
}

template <typename R, int LOGN>
__global__ void __launch_bounds__(OpShape<R, LOGN>::THREADS, OpShape<R, LOGN>::MINB)
k_op_row_inv(OpArgs<R> a) {
  typedef typename CT<R>::C C;
  typedef P2PlanR<LOGN, OpShape<R, LOGN>::LR> P;
  typedef OpShape<R, LOGN> Sh;
  constexpr int N = P::N, NP = Sh::NP, ROWS = 2 * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = tws + N;
  C* bufB = bufA + smem_padded(NP * N);
  pdl_trigger();
  stage_tw_p2r<LOGN, Sh::LR>(tws, a.twy);
  pdl_wait();
  __syncthreads();
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const int ntiles = (a.out_rows + ROWS - 1) / ROWS;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int x0 = tile * ROWS;
    gather_row_pairs<C, LOGN, NP, Sh::LNP, Sh::GATHER>(bufA, a.spec, a.nx, a.nyh, a.lw, x0, a.out_rows);
    __syncthreads();
    C v[Sh::E];
#pragma unroll
    for (int q = 0; q < Sh::E; ++q) v[q] = bufA[spad(s * N + tt + q * P::TPS)];
    fft_p2r<C, true, LOGN, Sh::LR>(v, bufB, bufA, s * N, 1, tt, tws);
    const int xa = x0 + 2 * s;
#pragma unroll
    for (int q = 0; q < Sh::E; ++q) {
      const int y = tt + q * P::TPS;
      if (y >= a.out_cols) continue;
      if (xa < a.out_rows) a.out[(size_t)xa * a.out_ld + y] = v[q].x;
      if (xa + 1 < a.out_rows) a.out[(size_t)(xa + 1) * a.out_ld + y] = v[q].y;
    }
    __syncthreads();  // buffers free for the next tile
  }
}
