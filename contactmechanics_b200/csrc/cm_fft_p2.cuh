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


// Twiddles of the radix-8 stages in shared memory, one table per stage:
// stage s (Ns = FIRST * 8^(s-1) butterfly groups) holds
// tw[toff(s) + (q-1)*Ns + k] = W^(q k N/(8 Ns)), W = exp(-2 pi i / N), for
// q = 1..7, k < Ns, so the threads of a warp (consecutive k, or a shared k)
// read consecutive words or one broadcast word.  The stage tables sum to at
// most N entries.  Built from the length-N table tw_n[m] = W^m, so every
// value is an entry of that table.
template <int LOGN, typename C>
CM_DEVINL void stage_tw_p2(C* tws, const C* __restrict__ tw_n) {
  typedef P2Plan<LOGN> P;
  constexpr int N = P::N;
  int toff = 0;
#pragma unroll
  for (int s = 1, Ns = P::FIRST; s < P::NST; ++s, Ns *= 8) {
    const int step = N / (Ns * 8);
    for (int i = threadIdx.x; i < 7 * Ns; i += blockDim.x) {
      const int q = 1 + i / Ns, k = i & (Ns - 1);
      tws[toff + i] = __ldg(tw_n + ((q * k * step) & (N - 1)));
    }
    toff += 7 * Ns;
  }
}

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
// sA / sB are the two ping-pong buffers; tw: the stage tables of
// stage_tw_p2 in shared memory.  Ends with the result in v and no pending shared-memory
// reads (a barrier is needed before reusing sA/sB).
template <typename C, bool INV, int LOGN>
CM_DEVINL void fft_p2(C (&v)[8], C* sA, C* sB, int base, int estride, int tt, const C* tw) {
  typedef P2Plan<LOGN> P;
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
  int toff = 0;
#pragma unroll
  for (int s = 1; s < P::NST; ++s) {
    const int k = tt & (Ns - 1);
    C g[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) g[q] = src[spad(base + (tt + q * P::TPS) * estride)];
#pragma unroll
    for (int q = 1; q < 8; ++q) {
      const C w = tw[toff + (q - 1) * Ns + k];
      g[q] = INV ? cmulc(g[q], w) : cmul(g[q], w);
    }
    toff += 7 * Ns;
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
