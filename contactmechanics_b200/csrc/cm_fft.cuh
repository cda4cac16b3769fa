// Shared-memory mixed-radix Stockham FFT used by the row and column passes.
//
// A block transforms `nseq` complex sequences of length n held in shared
// memory.  Element i of sequence s lives at buf[s*sstride + i*estride], so
// the same engine serves row tiles (sequences contiguous) and column tiles
// (sequences interleaved).  Stages ping-pong between two shared buffers
// (out-of-place Stockham, self-sorting); radices 2,3,4,5,7,8 have unrolled
// butterflies, any other prime factor runs as an O(r^2) direct DFT stage.
//
// Twiddles come from a per-length table tw[m] = exp(-2 pi i m / n), built on
// the host in long double and rounded once (so FP64 transforms keep full
// accuracy) and staged in shared memory by each kernel.
#pragma once
#include "cm_common.cuh"

#define CM_MAX_STAGES 24

struct FftDesc {
  int n;
  int nst;
  int generic;  // 1 when a stage radix is outside {2,3,4,5,7,8}
  int rad[CM_MAX_STAGES];
};

// twiddle lookup (the table is staged in shared memory by the caller)
template <typename C>
CM_DEVINL C tw_get(const C* tw, int m) { return tw[m]; }

// Length-RR DFT on registers.  Forward uses W = exp(-2 pi i / RR).
template <bool INV, int RR, typename C>
struct Dft {
  // generic small radix (3, 5, 7): direct sum with twiddles from the table
  static CM_DEVINL void run(C (&v)[RR], const C* tw, int n) {
    C w[RR];
    const int ws = n / RR;
    w[0] = cmake<C>(1, 0);
#pragma unroll
    for (int m = 1; m < RR; ++m) {
      C t = tw_get(tw, m * ws);
      w[m] = INV ? cconj(t) : t;
    }
    C y[RR];
#pragma unroll
    for (int q = 0; q < RR; ++q) {
      C acc = v[0];
#pragma unroll
      for (int p = 1; p < RR; ++p) acc = cadd(acc, cmul(v[p], w[(p * q) % RR]));
      y[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < RR; ++q) v[q] = y[q];
  }
};

template <bool INV, typename C>
struct Dft<INV, 2, C> {
  static CM_DEVINL void run(C (&v)[2], const C*, int) {
    C a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
};

template <bool INV, typename C>
CM_DEVINL void dft4(C& x0, C& x1, C& x2, C& x3) {
  C a0 = cadd(x0, x2), a1 = csub(x0, x2), a2 = cadd(x1, x3);
  C a3 = mul_mi<INV>(csub(x1, x3));
  x0 = cadd(a0, a2);
  x1 = cadd(a1, a3);
  x2 = csub(a0, a2);
  x3 = csub(a1, a3);
}

template <bool INV, typename C>
struct Dft<INV, 4, C> {
  static CM_DEVINL void run(C (&v)[4], const C*, int) { dft4<INV>(v[0], v[1], v[2], v[3]); }
};

template <bool INV, typename C>
struct Dft<INV, 8, C> {
  static CM_DEVINL void run(C (&v)[8], const C*, int) {
    typedef decltype(v[0].x) R;
    const R h = (R)0.70710678118654752440;  // sqrt(1/2)
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    C t1, t3;
    if (INV) {
      t1 = cmake<C>((o1.x - o1.y) * h, (o1.x + o1.y) * h);
      t3 = cmake<C>((-o3.x - o3.y) * h, (o3.x - o3.y) * h);
    } else {
      t1 = cmake<C>((o1.x + o1.y) * h, (o1.y - o1.x) * h);
      t3 = cmake<C>((o3.y - o3.x) * h, -(o3.x + o3.y) * h);
    }
    C t2 = mul_mi<INV>(o2);
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1);
    v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2);
    v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3);
    v[7] = csub(e3, t3);
  }
};

// One Stockham stage of radix RR from src to dst (out of place); every
// thread walks its butterflies one at a time, so only RR values are live.
template <typename C, bool INV, int RR>
CM_DEVINL void fft_stage(const C* src, C* dst, int n, int Ns, int nseq, int sstride, int estride,
                         bool seq_fastest, const C* tw) {
  const int m = n / RR;
  const int B = m * nseq;
  const int step = n / (Ns * RR);
  for (int bi = threadIdx.x; bi < B; bi += blockDim.x) {
    int s, j;
    if (seq_fastest) { s = bi % nseq; j = bi / nseq; }
    else { j = bi % m; s = bi / m; }
    const C* in = src + s * sstride;
    const int k = j % Ns;
    C v[RR];
#pragma unroll
    for (int q = 0; q < RR; ++q) v[q] = in[(j + q * m) * estride];
    if (Ns > 1) {
#pragma unroll
      for (int q = 1; q < RR; ++q) {
        const C w = tw_get(tw, q * k * step);
        v[q] = INV ? cmulc(v[q], w) : cmul(v[q], w);
      }
    }
    Dft<INV, RR, C>::run(v, tw, n);
    C* out = dst + s * sstride + ((j - k) * RR + k) * estride;
#pragma unroll
    for (int q = 0; q < RR; ++q) out[q * Ns * estride] = v[q];
  }
  __syncthreads();
}

// Direct DFT stage for an arbitrary radix r (prime factors above 7).
template <typename C, bool INV>
CM_DEVINL void fft_stage_generic(const C* src, C* dst, int n, int r, int Ns, int nseq,
                                 int sstride, int estride, bool seq_fastest,
                                 const C* tw) {
  const int m = n / r;
  const int B = m * nseq;
  const int step = n / (Ns * r);
  const int ws = n / r;
  for (int bi = threadIdx.x; bi < B; bi += blockDim.x) {
    int s, j;
    if (seq_fastest) { s = bi % nseq; j = bi / nseq; }
    else { j = bi % m; s = bi / m; }
    const C* in = src + s * sstride;
    C* out = dst + s * sstride;
    const int k = j % Ns;
    const int ob = (j - k) * r + k;
    for (int q = 0; q < r; ++q) {
      C acc = czero<C>();
      for (int p = 0; p < r; ++p) {
        C x = in[(j + p * m) * estride];
        if (Ns > 1 && p > 0) {
          const C w = tw_get(tw, p * k * step);
          x = INV ? cmulc(x, w) : cmul(x, w);
        }
        const C w = tw_get(tw, ((p * q) % r) * ws);
        acc = cadd(acc, INV ? cmulc(x, w) : cmul(x, w));
      }
      out[(ob + q * Ns) * estride] = acc;
    }
  }
  __syncthreads();
}

// Transform all sequences; data starts in `a`, `b` is a buffer of the same
// size.  Returns the buffer that holds the result.
template <typename C, bool INV>
CM_DEVINL C* fft_smem(C* a, C* b, const FftDesc& d, int nseq, int sstride, int estride,
                      bool seq_fastest, const C* tw) {
  int Ns = 1;
  for (int st = 0; st < d.nst; ++st) {
    const int r = d.rad[st];
    switch (r) {
      case 8: fft_stage<C, INV, 8>(a, b, d.n, Ns, nseq, sstride, estride, seq_fastest, tw); break;
      case 4: fft_stage<C, INV, 4>(a, b, d.n, Ns, nseq, sstride, estride, seq_fastest, tw); break;
      case 2: fft_stage<C, INV, 2>(a, b, d.n, Ns, nseq, sstride, estride, seq_fastest, tw); break;
      case 3: fft_stage<C, INV, 3>(a, b, d.n, Ns, nseq, sstride, estride, seq_fastest, tw); break;
      case 5: fft_stage<C, INV, 5>(a, b, d.n, Ns, nseq, sstride, estride, seq_fastest, tw); break;
      case 7: fft_stage<C, INV, 7>(a, b, d.n, Ns, nseq, sstride, estride, seq_fastest, tw); break;
      default: fft_stage_generic<C, INV>(a, b, d.n, r, Ns, nseq, sstride, estride, seq_fastest, tw); break;
    }
    C* t = a;
    a = b;
    b = t;
    Ns *= r;
  }
  return a;
}
