// Register-resident power-of-two FFT (N = 2^LOGN, 64 <= N <= 4096).
//
// Every thread owns the 8 elements {tt + q*N/8 : q = 0..7} of one sequence
// before the first and after the last stage, whatever the radices, so
//  * the first stage takes its inputs from registers (a fused prologue
//    computes them, or they come straight from global memory),
//  * the last stage leaves the transform in registers (a fused epilogue
//    consumes it, or it goes straight to global memory),
//  * a forward transform followed by an inverse one needs no shared-memory
//    pass in between (the column pass multiplies by the Green's table in
//    registers).
// Stages: one radix-2/4/8 stage (LOGN % 3 selects it) followed by radix-8
// stages; each stage but the last writes to one of two ping-pong shared
// buffers (Stockham, self-sorting), so a transform of NST stages makes
// NST-1 shared-memory round trips with one barrier each.  All index
// arithmetic is compile-time shifts and masks.
#pragma once
#include "cm_fft.cuh"

template <int LOGN>
struct P2Plan {
  static constexpr int N = 1 << LOGN;
  static constexpr int TPS = N / 8;              // threads per sequence
  static constexpr int LTPS = LOGN - 3;
  static constexpr int FIRST = (LOGN % 3 == 0) ? 8 : (1 << (LOGN % 3));
  static constexpr int NST = 1 + (LOGN - (LOGN % 3 == 0 ? 3 : LOGN % 3)) / 3;
};

// Shared-memory index with one padding slot per 8 elements: the strided
// Stockham writes (stride 4 or 8 elements across a warp) and the column
// layouts then hit distinct banks.  A buffer of E elements needs
// smem_padded(E) slots.
CM_DEVINL int spad(int e) { return e + (e >> 3); }
__host__ __device__ inline int smem_padded(int e) { return e + (e >> 3) + 1; }

template <bool INV, int R, typename C>
CM_DEVINL void dft_r(C* v) {
  if (R == 8) Dft<INV, 8, C>::run(*reinterpret_cast<C(*)[8]>(v), nullptr, 8);
  else if (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
  else {
    C a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
}

// Transform the thread's 8 elements in place.  Sequence layout in shared
// memory: element i of this thread's sequence at buf[spad(base + i*estride)];
// sA / sB are the two ping-pong buffers; tw: twiddle table exp(-2 pi i m / N)
// in shared memory.  Ends with the result in v and no pending shared-memory
// reads (a barrier is needed before reusing sA/sB).
template <typename C, bool INV, int LOGN>
CM_DEVINL void fft_p2(C (&v)[8], C* sA, C* sB, int base, int estride, int tt, const C* tw) {
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  // ---- first stage (Ns = 1): radix FIRST, 8/FIRST butterflies per thread
  {
    constexpr int R = P::FIRST;
    constexpr int B = 8 / R;
    C o[8];
#pragma unroll
    for (int i = 0; i < B; ++i) {
      C g[R];
#pragma unroll
      for (int q = 0; q < R; ++q) g[q] = v[i + B * q];
      dft_r<INV, R>(g);
#pragma unroll
      for (int q = 0; q < R; ++q) o[i * R + q] = g[q];
    }
    if (P::NST == 1) {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = o[i];
      return;
    }
    // butterfly j = tt + i*N/8 writes element j*R + q
#pragma unroll
    for (int i = 0; i < B; ++i) {
      const int j = tt + i * P::TPS;
#pragma unroll
      for (int q = 0; q < R; ++q) sA[spad(base + (j * R + q) * estride)] = o[i * R + q];
    }
  }
  __syncthreads();
  // ---- radix-8 stages
  C* src = sA;
  C* dst = sB;
  int Ns = P::FIRST;
#pragma unroll
  for (int s = 1; s < P::NST; ++s) {
    const int k = tt & (Ns - 1);
    C g[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) g[q] = src[spad(base + (tt + q * P::TPS) * estride)];
    const int step = N / (Ns * 8);
#pragma unroll
    for (int q = 1; q < 8; ++q) {
      const C w = tw[(q * k * step) & (N - 1)];
      g[q] = INV ? cmulc(g[q], w) : cmul(g[q], w);
    }
    Dft<INV, 8, C>::run(g, nullptr, 8);
    if (s == P::NST - 1) {
      // last stage: output index tt + q*N/8, i.e. the thread's own elements
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = g[q];
    } else {
      const int ob = (tt - k) * 8 + k;
#pragma unroll
      for (int q = 0; q < 8; ++q) dst[spad(base + (ob + q * Ns) * estride)] = g[q];
      __syncthreads();
      C* t = src;
      src = dst;
      dst = t;
    }
    Ns *= 8;
  }
}
