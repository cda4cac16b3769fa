// Register-resident power-of-two FFT (N = 2^LOGN, 64 <= N <= 8192).
//
// Every thread owns the 2^LR elements {tt + q*N/2^LR} of one sequence
// before the first and after the last stage, whatever the radices, so
//  * the first stage takes its inputs from registers (a fused prologue
//    computes them, or they come straight from global memory),
//  * the last stage leaves the transform in registers (a fused epilogue
//    consumes it, or it goes straight to global memory),
//  * a forward transform followed by an inverse one needs no shared-memory
//    pass in between (the column pass multiplies by the Green's table in
//    registers).
// Stages: one short first stage (LOGN % LR selects its radix) followed by
// radix-2^LR stages; each stage but the last writes to one of two ping-pong
// shared buffers (Stockham, self-sorting; one buffer and an extra barrier
// where two do not fit), so a transform of NST stages makes NST-1
// shared-memory round trips.  All index arithmetic is compile-time shifts
// and masks.
#pragma once
#include "cm_fft.cuh"

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

// ---------------------------------------------------------------------------
// 2^LR elements per thread (LR = 3 or 4): the same scheme with radix-16
// stages for LR = 4, fewer stages and exchanges per transform.
// ---------------------------------------------------------------------------
template <int LOGN, int LR>
struct P2PlanR {
  static constexpr int N = 1 << LOGN;
  static constexpr int RAD = 1 << LR;
  static constexpr int TPS = N / RAD;  // threads per sequence
  static constexpr int LTPS = LOGN - LR;
  static constexpr int FL = (LOGN % LR == 0) ? LR : LOGN % LR;
  static constexpr int FIRST = 1 << FL;
  static constexpr int NST = 1 + (LOGN - FL) / LR;
};

// a * W16^M (W16 = exp(-2 pi i / 16); conjugate for the inverse), M in
// {1, 2, 3, 4, 6, 9}: the internal twiddles of the length-16 DFT
template <bool INV, int M, typename C>
CM_DEVINL C w16(C a) {
  typedef decltype(a.x) R;
  const R c1 = (R)0.92387953251128675613;  // cos(pi/8)
  const R s1 = (R)0.38268343236508977173;  // sin(pi/8)
  const R h = (R)0.70710678118654752440;   // sqrt(1/2)
  if (M == 4) return mul_mi<INV>(a);
  R wr, wi;  // forward W16^M = wr + i wi
  if (M == 1) { wr = c1; wi = -s1; }
  else if (M == 2) { wr = h; wi = -h; }
  else if (M == 3) { wr = s1; wi = -c1; }
  else if (M == 6) { wr = -h; wi = -h; }
  else { wr = -c1; wi = s1; }  // M == 9
  if (INV) wi = -wi;
  return cmake<C>(a.x * wr - a.y * wi, a.x * wi + a.y * wr);
}

// Length-16 DFT in place, as 4 x 4: X[k1 + 4 k2] =
// sum_n2 W4^(n2 k2) W16^(n2 k1) sum_n1 x[4 n1 + n2] W4^(n1 k1).
template <bool INV, typename C>
CM_DEVINL void dft16(C (&v)[16]) {
  C y[4][4];  // y[n2][k1]
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    C a = v[n2], b = v[4 + n2], c = v[8 + n2], d = v[12 + n2];
    dft4<INV>(a, b, c, d);
    y[n2][0] = a; y[n2][1] = b; y[n2][2] = c; y[n2][3] = d;
  }
  y[1][1] = w16<INV, 1>(y[1][1]);
  y[1][2] = w16<INV, 2>(y[1][2]);
  y[1][3] = w16<INV, 3>(y[1][3]);
  y[2][1] = w16<INV, 2>(y[2][1]);
  y[2][2] = w16<INV, 4>(y[2][2]);
  y[2][3] = w16<INV, 6>(y[2][3]);
  y[3][1] = w16<INV, 3>(y[3][1]);
  y[3][2] = w16<INV, 6>(y[3][2]);
  y[3][3] = w16<INV, 9>(y[3][3]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C a = y[0][k1], b = y[1][k1], c = y[2][k1], d = y[3][k1];
    dft4<INV>(a, b, c, d);
    v[k1] = a; v[k1 + 4] = b; v[k1 + 8] = c; v[k1 + 12] = d;
  }
}

template <bool INV, int R, typename C>
CM_DEVINL void dft_rr(C* v) {
  if constexpr (R == 16) dft16<INV>(*reinterpret_cast<C(*)[16]>(v));
  else dft_r<INV, R>(v);
}

// Per-stage twiddle tables for 2^LR elements per thread: stage s (Ns butterfly
// groups) holds tw[toff(s) + (q-1)*Ns + k] = W^(q k N/(RAD Ns)), q = 1..RAD-1,
// k < Ns; N - FIRST entries in all (toff(s) = Ns - FIRST).  Entries of the
// table tw_n[m] = W^m.

// index into tw_n of staged entry i
template <int LOGN, int LR>
CM_DEVINL int tw_stage_index(int i) {
  typedef P2PlanR<LOGN, LR> P;
  constexpr int N = P::N;
  // Ns = FIRST * RAD^j with Ns <= i + FIRST < Ns * RAD
  const int lg = 31 - __clz(i + P::FIRST);  // floor(log2(i + FIRST))
  const int j = (lg - P::FL) / LR;
  const int lns = P::FL + j * LR, Ns = 1 << lns;
  const int r = i - (Ns - P::FIRST);
  const int q = 1 + (r >> lns), k = r & (Ns - 1);
  const int lstep = LOGN - lns - LR;  // step = N / (Ns RAD)
  return (q * k << lstep) & (N - 1);
}

// Stage the tables with NT threads a block: every thread issues all of its
// loads before its first store, so the staging costs one round trip.
template <int LOGN, int LR, int NT, typename C>
CM_DEVINL void stage_tw_p2r(C* tws, const C* __restrict__ tw_n) {
  typedef P2PlanR<LOGN, LR> P;
  constexpr int TOT = P::N - P::FIRST, PER = (TOT + NT - 1) / NT;
  C w[PER];
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int i = threadIdx.x + r * NT;
    if (i < TOT) w[r] = __ldg(tw_n + tw_stage_index<LOGN, LR>(i));
  }
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int i = threadIdx.x + r * NT;
    if (i < TOT) tws[i] = w[r];
  }
}

// Twiddle staging of a pass with NT threads a block; returns the table the
// transforms take (tw_n itself when ONEBUF: those transforms read it directly).
template <int LOGN, int LR, int NT, bool ONEBUF, typename C>
CM_DEVINL const C* stage_twiddles(C* tws, const C* __restrict__ tw_n) {
  if constexpr (ONEBUF) {
    return tw_n;
  } else {
    stage_tw_p2r<LOGN, LR, NT>(tws, tw_n);
    return tws;
  }
}

// Transform the thread's RAD elements {tt + q N/RAD} of one sequence in
// place (tables of stage_tw_p2r; the result is left in v with no pending
// shared-memory reads).
template <typename C, bool INV, int LOGN, int LR>
CM_DEVINL void fft_p2r(C (&v)[1 << LR], C* sA, C* sB, int base, int estride, int tt,
                       const C* tw) {
  typedef P2PlanR<LOGN, LR> P;
  constexpr int RAD = P::RAD;
  {
    constexpr int R = P::FIRST;
    constexpr int B = RAD / R;
    C o[RAD];
#pragma unroll
    for (int i = 0; i < B; ++i) {
      C g[R];
#pragma unroll
      for (int q = 0; q < R; ++q) g[q] = v[i + B * q];
      dft_rr<INV, R>(g);
#pragma unroll
      for (int q = 0; q < R; ++q) o[i * R + q] = g[q];
    }
    if (P::NST == 1) {
#pragma unroll
      for (int i = 0; i < RAD; ++i) v[i] = o[i];
      return;
    }
#pragma unroll
    for (int i = 0; i < B; ++i) {
      const int j = tt + i * P::TPS;
#pragma unroll
      for (int q = 0; q < R; ++q) sA[spad(base + (j * R + q) * estride)] = o[i * R + q];
    }
  }
  __syncthreads();
  C* src = sA;
  C* dst = sB;
  int Ns = P::FIRST;
  int toff = 0;
#pragma unroll
  for (int s = 1; s < P::NST; ++s) {
    const int k = tt & (Ns - 1);
    C g[RAD];
#pragma unroll
    for (int q = 0; q < RAD; ++q) g[q] = src[spad(base + (tt + q * P::TPS) * estride)];
#pragma unroll
    for (int q = 1; q < RAD; ++q) {
      const C w = tw[toff + (q - 1) * Ns + k];
      g[q] = INV ? cmulc(g[q], w) : cmul(g[q], w);
    }
    toff += (RAD - 1) * Ns;
    dft_rr<INV, RAD>(g);
    if (s == P::NST - 1) {
#pragma unroll
      for (int q = 0; q < RAD; ++q) v[q] = g[q];
    } else {
      const int ob = (tt - k) * RAD + k;
#pragma unroll
      for (int q = 0; q < RAD; ++q) dst[spad(base + (ob + q * Ns) * estride)] = g[q];
      __syncthreads();
      C* t = src;
      src = dst;
      dst = t;
    }
    Ns *= RAD;
  }
}

// The same transform for lengths whose ping-pong buffers and staged twiddle
// tables do not fit a block's shared memory (FP64 at 2^13): one shared
// buffer (every exchange writes, waits, reads and waits again before the
// next write) and the twiddles read from the length-N table tw_n[m] = W^m in
// global memory (L1/L2-cached; W^(q k N/(RAD Ns)) is entry q k step mod N,
// the value the staged tables hold).  Same contract as fft_p2r otherwise.
template <typename C, bool INV, int LOGN, int LR>
CM_DEVINL void fft_p2r_1buf(C (&v)[1 << LR], C* buf, int base, int estride, int tt,
                            const C* __restrict__ tw_n) {
  typedef P2PlanR<LOGN, LR> P;
  constexpr int RAD = P::RAD, N = P::N;
  {
    constexpr int R = P::FIRST;
    constexpr int B = RAD / R;
    C o[RAD];
#pragma unroll
    for (int i = 0; i < B; ++i) {
      C g[R];
#pragma unroll
      for (int q = 0; q < R; ++q) g[q] = v[i + B * q];
      dft_rr<INV, R>(g);
#pragma unroll
      for (int q = 0; q < R; ++q) o[i * R + q] = g[q];
    }
    if (P::NST == 1) {
#pragma unroll
      for (int i = 0; i < RAD; ++i) v[i] = o[i];
      return;
    }
#pragma unroll
    for (int i = 0; i < B; ++i) {
      const int j = tt + i * P::TPS;
#pragma unroll
      for (int q = 0; q < R; ++q) buf[spad(base + (j * R + q) * estride)] = o[i * R + q];
    }
  }
  __syncthreads();
  int Ns = P::FIRST;
#pragma unroll
  for (int s = 1; s < P::NST; ++s) {
    const int k = tt & (Ns - 1);
    const int step = N / (Ns * RAD);
    C g[RAD];
#pragma unroll
    for (int q = 0; q < RAD; ++q) g[q] = buf[spad(base + (tt + q * P::TPS) * estride)];
#pragma unroll
    for (int q = 1; q < RAD; ++q) {
      const C w = __ldg(tw_n + ((q * k * step) & (N - 1)));
      g[q] = INV ? cmulc(g[q], w) : cmul(g[q], w);
    }
    dft_rr<INV, RAD>(g);
    if (s == P::NST - 1) {
#pragma unroll
      for (int q = 0; q < RAD; ++q) v[q] = g[q];
    } else {
      __syncthreads();  // every read of this stage is done before the buffer is rewritten
      const int ob = (tt - k) * RAD + k;
#pragma unroll
      for (int q = 0; q < RAD; ++q) buf[spad(base + (ob + q * Ns) * estride)] = g[q];
      __syncthreads();
    }
    Ns *= RAD;
  }
}

// fft_p2r, or fft_p2r_1buf when ONEBUF (bufB and the staged tables unused;
// tw is then the global length-N table)
template <typename C, bool INV, int LOGN, int LR, bool ONEBUF>
CM_DEVINL void fft_p2x(C (&v)[1 << LR], C* bufA, C* bufB, int base, int estride, int tt,
                       const C* tw) {
  if constexpr (ONEBUF) fft_p2r_1buf<C, INV, LOGN, LR>(v, bufA, base, estride, tt, tw);
  else fft_p2r<C, INV, LOGN, LR>(v, bufA, bufB, base, estride, tt, tw);
}
