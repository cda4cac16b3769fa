// The elastic operator u = IFFT(T . FFT(f)) (FFTElasticHalfSpace.py:573-611,
// free :1141-1197) for power-of-two domains (sides 64..8192), as three
// passes over caller buffers:
//
//   k_op_row_fwd  row pairs (2p, 2p+1) with rows < in_rows: one complex
//                 transform of z = f[2p] + i f[2p+1] per pair, stored as it
//                 comes out of the registers: Z_p(k), k = 0..ny-1, at
//                 spec[p * ny + k] (the pair-major spectrum);
//   k_op_col      every column k = 0..ny/2 of the half spectrum: the column
//                 X_x(k) of row x = 2p + b is split off the pair transforms
//                 in registers (X_2p(k) = (Z_p(k) + conj Z_p(ny-k)) / 2,
//                 X_2p+1(k) = (Z_p(k) - conj Z_p(ny-k)) / 2i; rows >= in_rows
//                 are zero), transformed along x, multiplied by the real
//                 Green's table, transformed back, and packed again for the
//                 inverse row transforms: W_p(k) = Xh_2p(k) + i Xh_2p+1(k) and
//                 W_p(ny-k) = conj Xh_2p(k) + i conj Xh_2p+1(k), pairs with rows
//                 < out_rows written back in place;
//   k_op_row_inv  row pairs with rows < out_rows: one inverse complex
//                 transform of W_p per pair straight from the spectrum; the
//                 real part is row 2p, the imaginary part row 2p+1.
//
// The row passes thus read and write the spectrum in whole rows from the
// transform registers, with no shared-memory split or pack pass; the split
// and the pack are arithmetic in the column pass, whose two rows of a pair
// sit in neighbouring threads (a shuffle exchanges them).  A column group
// covers W consecutive columns (W = 32 bytes of complex values, so every
// spectrum access of a warp fills whole 32-byte sectors; fewer when the
// shared memory of a long column does not allow it).
//
// Arguments travel by value (no descriptor upload), so a call is a plain
// sequence of three launches on the caller's stream.  Blocks walk their
// tiles with a grid stride, so the twiddle tables are staged once per block;
// the transforms are the register-resident engines of cm_fft_p2.cuh (row
// passes and column pass 2^LR elements per thread).
#pragma once
#include "cm_fft_p2.cuh"
#include "cm_kernels.cuh"
#include "cm_launch.h"

// resident blocks per SM the FP64 row passes are compiled for: two blocks
// of 256 threads (at most 128 registers a thread) hide more latency than one
#ifndef CM_FP64_ROW_MINB
#define CM_FP64_ROW_MINB 2
#endif

// threads of an FP32 row-pass block (at least one transform) and the
// resident blocks per SM it is compiled for
#ifndef CM_ROW_F32_BASE
#define CM_ROW_F32_BASE 512
#endif
#ifndef CM_ROW_F32_MINB
#define CM_ROW_F32_MINB 2
#endif

// threads of a column-pass block when a column group is smaller
#ifndef CM_COL_BASE
#define CM_COL_BASE 256
#endif

// log2 of the elements per thread of the column pass's transforms
#ifndef CM_COL_LR_F32
#define CM_COL_LR_F32 4
#endif
#ifndef CM_COL_LR_F64
#define CM_COL_LR_F64 4
#endif

// log2 of the columns of a column group (at most; fewer when its shared
// memory does not fit): 32 bytes of complex values
#ifndef CM_COL_LW_F32
#define CM_COL_LW_F32 2
#endif
#ifndef CM_COL_LW_F64
#define CM_COL_LW_F64 1
#endif

// log2 of the elements per thread of the solver's displacement pass
// (k_ccg_row_inv<MODE_F>): its epilogue reads four fields per element, so it
// keeps eight elements per thread and twice the resident warps
#ifndef CM_ROW_LR_INVF_F32
#define CM_ROW_LR_INVF_F32 3
#endif

// log2 of the elements per thread of the row passes' transforms (3: the
// radix-8 engine, 4: the radix-16 one)
#ifndef CM_ROW_LR_F32
#define CM_ROW_LR_F32 4
#endif
#ifndef CM_ROW_LR_F64
#define CM_ROW_LR_F64 3
#endif

// log2 of the elements per thread of each power-of-two part of a length
// 3 * 2^m (three parts, so a thread holds three times as many), and the
// threads of a row-pass block for those lengths.  Four elements a part in
// FP32 too: the solver passes' epilogues then keep their fields in
// registers (mixed solves 8-20 % faster than with eight, periodic 768..3072).
#ifndef CM_T3_LR_F32
#define CM_T3_LR_F32 2
#endif
#ifndef CM_T3_LR_F64
#define CM_T3_LR_F64 2
#endif
#ifndef CM_T3_ROW_BASE
#define CM_T3_ROW_BASE 256
#endif

// default log2 elements per thread (per part) of the row passes for length
// code L (cm_fft_p2.cuh): FP64 transforms of length 2^13 take 16 elements
// per thread (512 threads a sequence)
template <typename R>
constexpr int row_lr(int code) {
  return code >= 32 ? (sizeof(R) == 8 ? CM_T3_LR_F64 : CM_T3_LR_F32)
                    : sizeof(R) == 8 ? (code >= 13 ? 4 : CM_ROW_LR_F64) : CM_ROW_LR_F32;
}

// threads of one block of the row passes for the transform of length code
// LOGN (2^LOGN, or 3 * 2^m for LOGN = CM_T3(m)) with 2^LRV elements of each
// power-of-two part per thread.  ONEBUF: the ping-pong buffers and the
// staged twiddles do not fit a block's shared memory (FP64 at 2^13), so the
// transform runs on one buffer with the twiddles read from global memory;
// ONESTG: one buffer and the staged twiddles fit (FP64 at 3 * 2^11).
template <typename R, int LOGN, int LRV = row_lr<R>(LOGN)>
struct OpShape {
  typedef typename CT<R>::C C;
  typedef FftLen<LOGN, LRV> P;
  static constexpr int N = P::N;
  static constexpr int LR = LRV;
  static constexpr int E = P::E;  // elements per thread
  static constexpr int TPS = P::TPS;
  static constexpr int BASE = P::F == 3 ? CM_T3_ROW_BASE
                                        : (sizeof(R) == 8 ? 256 : CM_ROW_F32_BASE) >> (LR - 3);
  static constexpr int THREADS = TPS > BASE ? TPS : BASE;
  static constexpr int NP = THREADS / TPS;  // row pairs per block
  static constexpr size_t BUF = (size_t)(NP * N + ((NP * N) >> 3) + 1) * sizeof(C);
  static constexpr bool TWO = N * sizeof(C) + 2 * BUF <= CM_SMEM_DYN_MAX;
  // ONESTG: one buffer with the twiddles staged (FP64 at 3 * 2^11)
  static constexpr bool ONESTG = !TWO && N * sizeof(C) + BUF <= CM_SMEM_DYN_MAX;
  static constexpr bool ONEBUF = !TWO && !ONESTG;
  static constexpr size_t SMEM = TWO ? N * sizeof(C) + 2 * BUF : ONESTG ? N * sizeof(C) + BUF : BUF;
  static constexpr size_t STAGE = TWO ? 2 * BUF : BUF;  // bytes for staging input rows
  // resident blocks per SM the kernels are compiled for; one when a block
  // holds more than half of the shared memory
  static constexpr int MINB = SMEM > CM_SMEM_DYN_MAX / 2 ? 1
                              : sizeof(R) == 8 ? CM_FP64_ROW_MINB : CM_ROW_F32_MINB;
  static size_t smem() { return SMEM; }
};

// Column pass for columns of length code LOGX: 16 elements per thread for
// 2^LOGX (3 x 2^LR for 3 * 2^m), groups of W = 2^LW columns with the column
// index fastest across threads.
template <typename R, int LOGX>
struct ColShape {
  typedef typename CT<R>::C C;
  static constexpr int LR = LenCode<LOGX>::F == 3 ? (sizeof(R) == 8 ? CM_T3_LR_F64 : CM_T3_LR_F32)
                            : sizeof(R) == 8 ? CM_COL_LR_F64 : CM_COL_LR_F32;
  typedef FftLen<LOGX, LR> P;
  static constexpr int NX = P::N;
  static constexpr int E = P::E;  // elements per thread
  static constexpr int TPS = P::TPS;
  static constexpr size_t smem_for(int lw) {
    return (size_t)(NX + 2 * (((NX << lw)) + ((NX << lw) >> 3) + 1)) * sizeof(C);
  }
  // 32 bytes of complex values per column group, fewer if the group's
  // ping-pong buffers do not fit
  static constexpr int LW_PREF = sizeof(C) == 8 ? CM_COL_LW_F32 : CM_COL_LW_F64;
  static constexpr int LW = smem_for(LW_PREF) <= CM_SMEM_DYN_MAX ? LW_PREF
                            : smem_for(LW_PREF - 1) <= CM_SMEM_DYN_MAX ? LW_PREF - 1 : 0;
  static constexpr int W = 1 << LW;
  static constexpr int GROUP = W * TPS;
  static constexpr int THREADS = GROUP > CM_COL_BASE ? GROUP : CM_COL_BASE;
  static constexpr int NG = THREADS / GROUP;  // column groups per block
  static constexpr size_t BUF = (size_t)(NG * NX * W + ((NG * NX * W) >> 3) + 1) * sizeof(C);
  // one buffer when even one column's ping-pong buffers do not fit: with the
  // twiddles staged where they fit beside it (ONESTG: FP64 at 3 * 2^11),
  // else read from the global table (ONEBUF: FP64 at 2^13)
  static constexpr bool TWO = NX * sizeof(C) + 2 * BUF <= CM_SMEM_DYN_MAX;
  static constexpr bool ONESTG = !TWO && NX * sizeof(C) + BUF <= CM_SMEM_DYN_MAX;
  static constexpr bool ONEBUF = !TWO && !ONESTG;
  static constexpr size_t SMEM = TWO ? NX * sizeof(C) + 2 * BUF : ONESTG ? NX * sizeof(C) + BUF : BUF;
  static size_t smem() { return SMEM; }
};

template <typename R, int LOGN>
__global__ void __launch_bounds__(OpShape<R, LOGN>::THREADS, OpShape<R, LOGN>::MINB)
k_op_row_fwd(OpArgs<R> a) {
  typedef typename CT<R>::C C;
  typedef OpShape<R, LOGN> Sh;
  typedef typename Sh::P P;
  constexpr int N = P::N, NP = Sh::NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = Sh::ONEBUF ? tws : tws + N;
  C* bufB = bufA + smem_padded(NP * N);
  pdl_trigger();
  const C* tw = stage_twiddles<LOGN, Sh::LR, Sh::THREADS, Sh::ONEBUF>(tws, a.twy);
  pdl_wait();
  __syncthreads();
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const int npairs = (a.in_rows + 1) >> 1;
  for (int p0 = blockIdx.x * NP; p0 < npairs; p0 += gridDim.x * NP) {
    const int p = p0 + s, xa = 2 * p;
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
    fft_len<C, false, LOGN, Sh::LR, Sh::ONEBUF, Sh::ONESTG>(v, bufA, bufB, s * N, 1, tt, tw);
    if (p < npairs) {
      C* __restrict__ row = a.spec + (size_t)p * N;
#pragma unroll
      for (int q = 0; q < Sh::E; ++q) row[kfreq<LOGN, Sh::LR>(tt, q)] = v[q];
    }
    __syncthreads();  // buffers free for the next pairs
  }
}

// Loads of one column unit k of the pair-major spectrum (rows x = 2p + b of
// the thread's elements x = tt + q TPS, b = tt & 1): both rows of a pair load
// Z_p(k) and Z_p(ny - k) (neighbouring lanes, one request) and each splits
// off its own row.  Rows >= in_rows are zero.
template <typename C, int TPS, int E>
CM_DEVINL void col_split_load(C (&v)[E], const C* __restrict__ spec, int ny, int k, int km, int tt,
                              int in_rows, bool ok) {
  typedef decltype(v[0].x) R;
  const int b = tt & 1;
  const C* __restrict__ sk = spec + k + (size_t)(tt >> 1) * ny;
  const C* __restrict__ skm = spec + km + (size_t)(tt >> 1) * ny;
  const int pstep = (TPS / 2) * ny;
  constexpr int CH = E % 8 == 0 ? 8 : 4;  // loads in flight per chunk
#pragma unroll
  for (int h = 0; h < E; h += CH) {
    C z[CH], zm[CH];
#pragma unroll
    for (int q = h; q < h + CH; ++q) {
      const int x = tt + q * TPS;
      z[q - h] = czero<C>();
      zm[q - h] = czero<C>();
      if (ok && x < in_rows) {
        z[q - h] = sk[(size_t)q * pstep];
        zm[q - h] = skm[(size_t)q * pstep];
      }
    }
#pragma unroll
    for (int q = h; q < h + CH; ++q) {
      const C zk = z[q - h], zn = zm[q - h];
      v[q] = b ? cmake<C>((zk.y + zn.y) * (R)0.5, (zn.x - zk.x) * (R)0.5)
               : cmake<C>((zk.x + zn.x) * (R)0.5, (zk.y - zn.y) * (R)0.5);
    }
  }
}

// Pack the filtered column back into the pair-major spectrum: the even row of
// a pair writes W_p(k) = Xh_2p + i Xh_2p+1 (real parts only for the
// self-conjugate columns 0 and ny/2), the odd row W_p(ny - k); pairs with
// rows < out_rows.
template <typename C, int TPS, int W, int E>
CM_DEVINL void col_pack_store(const C (&v)[E], C* __restrict__ spec, int ny, int k, int km, int tt,
                              int out_rows, bool ok) {
  const int b = tt & 1;
  const int pairs_out = (out_rows + 1) >> 1;
  const bool selfc = (k == 0) || (2 * k == ny);
  const bool writes = ok && !(b && selfc);
  C* __restrict__ dst = spec + (b ? km : k) + (size_t)(tt >> 1) * ny;
  const int pstep = (TPS / 2) * ny;
#pragma unroll
  for (int q = 0; q < E; ++q) {
    const C a = v[q];
    C o;
    o.x = __shfl_xor_sync(0xffffffffu, a.x, W);
    o.y = __shfl_xor_sync(0xffffffffu, a.y, W);
    const int pp = (tt >> 1) + q * (TPS / 2);
    if (!writes || pp >= pairs_out) continue;
    dst[(size_t)q * pstep] = !b ? (selfc ? cmake<C>(a.x, o.x) : cmake<C>(a.x - o.y, a.y + o.x))
                                : cmake<C>(o.x + a.y, a.x - o.y);
  }
}

template <typename R, int LOGX>
__global__ void __launch_bounds__(ColShape<R, LOGX>::THREADS, 1)
k_op_col(OpArgs<R> a) {
  typedef typename CT<R>::C C;
  typedef ColShape<R, LOGX> Sh;
  typedef typename Sh::P P;
  constexpr int NX = P::N, W = Sh::W, LW = Sh::LW, E = Sh::E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = Sh::ONEBUF ? tws : tws + NX;
  C* bufB = bufA + smem_padded(Sh::NG * NX * W);
  pdl_trigger();
  const C* tw = stage_twiddles<LOGX, Sh::LR, Sh::THREADS, Sh::ONEBUF>(tws, a.twx);
  pdl_wait();
  if (a.st && (a.st->done || (a.cg_only && a.st->branch != 0))) return;
  __syncthreads();
  const int ny = a.ny;
  const int c = threadIdx.x & (W - 1);
  const int tt = (threadIdx.x >> LW) & (P::TPS - 1);
  const int j = threadIdx.x >> (LW + P::LTPS);
  const int units = ny / 2 + 1;
  const int ngroups = (units + W - 1) >> LW;
  const int base = j * NX * W + c;
  const int tlw = a.lw, tW = 1 << tlw;  // the table's column tiles
  for (int g0 = blockIdx.x * Sh::NG; g0 < ngroups; g0 += gridDim.x * Sh::NG) {
    const int k = (g0 + j) * W + c;
    const bool ok = k < units;
    const int km = k == 0 ? 0 : ny - k;  // the mirror column (ny need not be a power of two)
    C v[E];
    col_split_load<C, P::TPS, E>(v, a.spec, ny, k, km, tt, a.in_rows, ok);
    fft_len<C, false, LOGX, Sh::LR, Sh::ONEBUF, Sh::ONESTG>(v, bufA, bufB, base, W, tt, tw);
    if (a.fwd_real) {
      // forward transform only: the real part of the 2D transform, in the
      // natural (nx, ny/2 + 1) layout (a real, even kernel's Green's table)
      if (ok) {
#pragma unroll
        for (int q = 0; q < E; ++q) a.fwd_real[(size_t)kfreq<LOGX, Sh::LR>(tt, q) * units + k] = v[q].x;
      }
      __syncthreads();
      continue;
    }
    // the table's row of register q: its frequency index along x
    const R* __restrict__ tb = a.tab + ((size_t)(k >> tlw) * NX << tlw) + (k & (tW - 1)) +
                               (P::F == 1 ? (size_t)tt << tlw : 0);
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const size_t row = P::F == 1 ? (size_t)(q * P::TPS) : (size_t)kfreq<LOGX, Sh::LR>(tt, q);
      v[q] = cscale(v[q], ok ? __ldg(tb + (row << tlw)) : (R)0);
    }
    __syncthreads();
    fft_len<C, true, LOGX, Sh::LR, Sh::ONEBUF, Sh::ONESTG>(v, bufA, bufB, base, W, tt, tw);
    col_pack_store<C, P::TPS, W, E>(v, a.spec, ny, k, km, tt, a.out_rows, ok);
    __syncthreads();  // buffers free for the next group
  }
}

template <typename R, int LOGN>
__global__ void __launch_bounds__(OpShape<R, LOGN>::THREADS, OpShape<R, LOGN>::MINB)
k_op_row_inv(OpArgs<R> a) {
  typedef typename CT<R>::C C;
  typedef OpShape<R, LOGN> Sh;
  typedef typename Sh::P P;
  constexpr int N = P::N, NP = Sh::NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tws = reinterpret_cast<C*>(smem_raw);
  C* bufA = Sh::ONEBUF ? tws : tws + N;
  C* bufB = bufA + smem_padded(NP * N);
  pdl_trigger();
  const C* tw = stage_twiddles<LOGN, Sh::LR, Sh::THREADS, Sh::ONEBUF>(tws, a.twy);
  pdl_wait();
  __syncthreads();
  const int s = threadIdx.x >> P::LTPS, tt = threadIdx.x & (P::TPS - 1);
  const int npairs = (a.out_rows + 1) >> 1;
  for (int p0 = blockIdx.x * NP; p0 < npairs; p0 += gridDim.x * NP) {
    const int p = p0 + s, xa = 2 * p;
    C v[Sh::E];
    const C* __restrict__ row = a.spec + (size_t)p * N;
#pragma unroll
    for (int q = 0; q < Sh::E; ++q) v[q] = p < npairs ? row[kfreq<LOGN, Sh::LR>(tt, q)] : czero<C>();
    fft_len<C, true, LOGN, Sh::LR, Sh::ONEBUF, Sh::ONESTG>(v, bufA, bufB, s * N, 1, tt, tw);
#pragma unroll
    for (int q = 0; q < Sh::E; ++q) {
      const int y = tt + q * P::TPS;
      if (y >= a.out_cols) continue;
      if (xa < a.out_rows) a.out[(size_t)xa * a.out_ld + y] = v[q].x;
      if (xa + 1 < a.out_rows) a.out[(size_t)(xa + 1) * a.out_ld + y] = v[q].y;
    }
    __syncthreads();  // buffers free for the next pairs
  }
}
