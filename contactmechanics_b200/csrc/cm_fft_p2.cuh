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

// Transform lengths of the register-resident passes, by code: L < 32 is
// N = 2^L, L = 32 + m is N = 3 * 2^m.
#define CM_T3(m) (32 + (m))
template <int L>
struct LenCode {
  static constexpr int F = L >= 32 ? 3 : 1;
  static constexpr int LOGM = L >= 32 ? L - 32 : L;
  static constexpr int M = 1 << LOGM;
  static constexpr int N = F * M;
};

// Thread layout of a length-N transform with 2^LR elements of each of its F
// power-of-two parts per thread: thread tt of a sequence owns the E elements
// at time index tt + q TPS, q < E.
template <int L, int LR>
struct FftLen {
  static constexpr int F = LenCode<L>::F, LOGM = LenCode<L>::LOGM;
  static constexpr int M = LenCode<L>::M, N = LenCode<L>::N;
  static constexpr int RAD = 1 << LR;
  static constexpr int E = F * RAD;    // elements per thread
  static constexpr int TPS = M / RAD;  // threads per sequence
  static constexpr int LTPS = LOGM - LR;
};

// Frequency index of register q after a forward transform (and of the input
// of an inverse one): tt + q TPS for N = 2^L; for N = 3M the radix-3 split
// leaves X(3k + j) in register j RAD + qq with k = tt + qq TPS.
template <int L, int LR>
CM_DEVINL int kfreq(int tt, int q) {
  typedef FftLen<L, LR> P;
  if constexpr (P::F == 1) return tt + q * P::TPS;
  else return 3 * (tt + (q & (P::RAD - 1)) * P::TPS) + (q >> LR);
}

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

// Tables of a length-3M transform (M = 2^LOGM): the sub-transforms' tables
// of stage_tw_p2r for length M (W_M^m = W_N^(3m) of the length-N table tw_n)
// followed by W_N^m for m < 2M, the twiddles of the radix-3 split.
template <int LOGM, int LR, int NT, typename C>
CM_DEVINL void stage_tw_t3(C* tws, const C* __restrict__ tw_n) {
  typedef P2PlanR<LOGM, LR> P;
  constexpr int M = P::N, SUB = M - P::FIRST, TOT = SUB + 2 * M, PER = (TOT + NT - 1) / NT;
  C w[PER];
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int i = threadIdx.x + r * NT;
    if (i < TOT) w[r] = __ldg(tw_n + (i < SUB ? 3 * tw_stage_index<LOGM, LR>(i) : i - SUB));
  }
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int i = threadIdx.x + r * NT;
    if (i < TOT) tws[i] = w[r];
  }
}

// Twiddle staging of a pass with NT threads a block for length code L;
// returns the table the transforms take (tw_n itself when ONEBUF: those
// transforms read it directly).
template <int L, int LR, int NT, bool ONEBUF, typename C>
CM_DEVINL const C* stage_twiddles(C* tws, const C* __restrict__ tw_n) {
  if constexpr (ONEBUF) {
    static_assert(LenCode<L>::F == 1, "lengths 3 * 2^m keep both transform buffers");
    return tw_n;
  } else if constexpr (LenCode<L>::F == 1) {
    stage_tw_p2r<L, LR, NT>(tws, tw_n);
    return tws;
  } else {
    stage_tw_t3<LenCode<L>::LOGM, LR, NT>(tws, tw_n);
    return tws;
  }
}

// Transform G sequences of the thread's RAD elements {tt + q N/RAD} each in
// place: group g is v[g RAD .. g RAD + RAD - 1] and lives at shared offset
// base + g gstride (tables of stage_tw_p2r; the result is left in v with no
// pending shared-memory reads).  The groups share every barrier.  ONE: sA
// and sB are the same buffer, so every stage reads all of its groups into
// registers, waits, and only then writes (one barrier more per stage).
template <typename C, bool INV, int LOGN, int LR, int G, bool ONE = false>
CM_DEVINL void fft_p2g(C (&v)[G << LR], C* sA, C* sB, int base, int gstride, int estride, int tt,
                       const C* tw) {
  typedef P2PlanR<LOGN, LR> P;
  constexpr int RAD = P::RAD;
#pragma unroll
  for (int g = 0; g < G; ++g) {
    constexpr int R = P::FIRST;
    constexpr int B = RAD / R;
    C* vg = v + g * RAD;
    const int bg = base + g * gstride;
    C o[RAD];
#pragma unroll
    for (int i = 0; i < B; ++i) {
      C e[R];
#pragma unroll
      for (int q = 0; q < R; ++q) e[q] = vg[i + B * q];
      dft_rr<INV, R>(e);
#pragma unroll
      for (int q = 0; q < R; ++q) o[i * R + q] = e[q];
    }
    if (P::NST == 1) {
#pragma unroll
      for (int i = 0; i < RAD; ++i) vg[i] = o[i];
      continue;
    }
#pragma unroll
    for (int i = 0; i < B; ++i) {
      const int j = tt + i * P::TPS;
#pragma unroll
      for (int q = 0; q < R; ++q) sA[spad_t<sizeof(C)>(bg + (j * R + q) * estride)] = o[i * R + q];
    }
  }
  if (P::NST == 1) return;
  __syncthreads();
  C* src = sA;
  C* dst = sB;
  int Ns = P::FIRST;
  int toff = 0;
#pragma unroll
  for (int s = 1; s < P::NST; ++s) {
    const int k = tt & (Ns - 1);
    if constexpr (ONE) {
      // every read of the stage before the buffer is rewritten
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int bg = base + g * gstride;
#pragma unroll
        for (int q = 0; q < RAD; ++q) v[g * RAD + q] = src[spad_t<sizeof(C)>(bg + (tt + q * P::TPS) * estride)];
      }
      if (s < P::NST - 1) __syncthreads();
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int bg = base + g * gstride;
      C e[RAD];
#pragma unroll
      for (int q = 0; q < RAD; ++q)
        e[q] = ONE ? v[g * RAD + q] : src[spad_t<sizeof(C)>(bg + (tt + q * P::TPS) * estride)];
#pragma unroll
      for (int q = 1; q < RAD; ++q) {
        const C w = tw[toff + (q - 1) * Ns + k];
        e[q] = INV ? cmulc(e[q], w) : cmul(e[q], w);
      }
      dft_rr<INV, RAD>(e);
      if (s == P::NST - 1) {
#pragma unroll
        for (int q = 0; q < RAD; ++q) v[g * RAD + q] = e[q];
      } else {
        const int ob = (tt - k) * RAD + k;
#pragma unroll
        for (int q = 0; q < RAD; ++q) dst[spad_t<sizeof(C)>(bg + (ob + q * Ns) * estride)] = e[q];
      }
    }
    toff += (RAD - 1) * Ns;
    if (s < P::NST - 1) {
      __syncthreads();
      C* t = src;
      src = dst;
      dst = t;
    }
    Ns *= RAD;
  }
}

// One sequence: the thread's RAD elements {tt + q N/RAD}.
template <typename C, bool INV, int LOGN, int LR>
CM_DEVINL void fft_p2r(C (&v)[1 << LR], C* sA, C* sB, int base, int estride, int tt,
                       const C* tw) {
  fft_p2g<C, INV, LOGN, LR, 1>(v, sA, sB, base, 0, estride, tt, tw);
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
      for (int q = 0; q < R; ++q) buf[spad_t<sizeof(C)>(base + (j * R + q) * estride)] = o[i * R + q];
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
    for (int q = 0; q < RAD; ++q) g[q] = buf[spad_t<sizeof(C)>(base + (tt + q * P::TPS) * estride)];
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
      for (int q = 0; q < RAD; ++q) buf[spad_t<sizeof(C)>(base + (ob + q * Ns) * estride)] = g[q];
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

// Length N = 3M (M = 2^LOGM).  The thread's elements v[qq + r RAD] (qq < RAD,
// r < 3) sit at time index n + r M with n = tt + qq M/RAD.
// Forward: the radix-3 split by decimation in frequency, in registers,
//   a_j(n) = W_N^(j n) sum_r W_3^(r j) x(n + r M),   j < 3,
// then the three length-M transforms of a_j, which share their barriers:
// X(3k + j) = sum_n W_M^(n k) a_j(n) is left in v[j RAD + qq], k = tt + qq M/RAD
// (kfreq).  Inverse: the mirror image (length-M inverse transforms of
// X(3k + j) over k, the twiddle W_N^(-j n), the radix-3 combination), again
// unnormalised, leaving x(n + r M) in v[qq + r RAD].  Sub-sequence j lives at
// shared offset base + j M estride; tw holds the tables of stage_tw_t3.
template <typename C, bool INV, int LOGM, int LR, bool ONE = false>
CM_DEVINL void fft_t3(C (&v)[3 << LR], C* sA, C* sB, int base, int estride, int tt, const C* tw) {
  typedef P2PlanR<LOGM, LR> P;
  typedef decltype(v[0].x) R;
  constexpr int RAD = P::RAD, M = P::N;
  const C* __restrict__ w3 = tw + (M - P::FIRST);  // W_N^m, m < 2M
  const R s3 = (R)0.86602540378443864676;         // sqrt(3) / 2
  const R half = (R)0.5;
  if (!INV) {
#pragma unroll
    for (int qq = 0; qq < RAD; ++qq) {
      const int n = tt + qq * P::TPS;
      const C x0 = v[qq], x1 = v[qq + RAD], x2 = v[qq + 2 * RAD];
      const C sm = cadd(x1, x2), df = csub(x1, x2);
      const C md = cmake<C>(x0.x - half * sm.x, x0.y - half * sm.y);
      const C rt = cmake<C>(s3 * df.y, -s3 * df.x);  // -i sqrt(3)/2 (x1 - x2)
      v[qq] = cadd(x0, sm);
      v[qq + RAD] = cmul(cadd(md, rt), w3[n]);
      v[qq + 2 * RAD] = cmul(csub(md, rt), w3[2 * n]);
    }
    fft_p2g<C, false, LOGM, LR, 3, ONE>(v, sA, sB, base, M * estride, estride, tt, tw);
  } else {
    fft_p2g<C, true, LOGM, LR, 3, ONE>(v, sA, sB, base, M * estride, estride, tt, tw);
#pragma unroll
    for (int qq = 0; qq < RAD; ++qq) {
      const int n = tt + qq * P::TPS;
      const C y0 = v[qq];
      const C y1 = cmulc(v[qq + RAD], w3[n]), y2 = cmulc(v[qq + 2 * RAD], w3[2 * n]);
      const C sm = cadd(y1, y2), df = csub(y1, y2);
      const C md = cmake<C>(y0.x - half * sm.x, y0.y - half * sm.y);
      const C rt = cmake<C>(-s3 * df.y, s3 * df.x);  // +i sqrt(3)/2 (y1 - y2)
      v[qq] = cadd(y0, sm);
      v[qq + RAD] = cadd(md, rt);
      v[qq + 2 * RAD] = csub(md, rt);
    }
  }
}

// The transform of length code L: fft_p2x for 2^L, fft_t3 for 3 * 2^m.
// ONEBUF: one buffer, twiddles read from the global table (2^L only);
// ONESTG: one buffer (bufA), staged twiddles.
template <typename C, bool INV, int L, int LR, bool ONEBUF, bool ONESTG = false>
CM_DEVINL void fft_len(C (&v)[FftLen<L, LR>::E], C* bufA, C* bufB, int base, int estride, int tt,
                       const C* tw) {
  if constexpr (LenCode<L>::F == 1) {
    if constexpr (ONESTG)
      fft_p2g<C, INV, L, LR, 1, true>(v, bufA, bufA, base, 0, estride, tt, tw);
    else
      fft_p2x<C, INV, L, LR, ONEBUF>(v, bufA, bufB, base, estride, tt, tw);
  } else {
    static_assert(!ONEBUF, "lengths 3 * 2^m stage their twiddles");
    fft_t3<C, INV, LenCode<L>::LOGM, LR, ONESTG>(v, bufA, ONESTG ? bufA : bufB, base, estride, tt,
                                                 tw);
  }
}
