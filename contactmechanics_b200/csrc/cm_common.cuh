// Common device helpers for the contact-mechanics CUDA library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define CM_DEVINL __device__ __forceinline__

// Shared-memory index of element e of a transform buffer whose elements have
// BYTES bytes: the low bits within each 128-byte row are XORed with the row
// number.  A warp's contiguous accesses then take the fewest wavefronts,
// and the strided Stockham writes (4 to 16 elements apart across a warp)
// spread over all banks.  The alternative, one padding slot per 8 elements,
// makes every contiguous 32-element access span three rows (FP32 operator
// 2048^2: 45.3 us against 41.8 us with the swizzle).  The map is a
// bijection on every aligned row, so a buffer of E elements (E a multiple of
// the row) needs E slots; smem_padded(E) slots are allocated, the sizes the
// passes' occupancy was measured with.
template <int BYTES>
CM_DEVINL int spad_t(int e) {
  constexpr int ROW = 128 / BYTES, LROW = ROW == 16 ? 4 : 3;
  return e ^ ((e >> LROW) & (ROW - 1));
}
__host__ __device__ inline int smem_padded(int e) { return e + (e >> 3) + 1; }

template <typename R> struct CT;
template <> struct CT<float> { typedef float2 C; };
template <> struct CT<double> { typedef double2 C; };

template <typename C> CM_DEVINL C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> CM_DEVINL C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> CM_DEVINL C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a * conj(b)
template <typename C> CM_DEVINL C cmulc(C a, C b) {
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}
template <typename C> CM_DEVINL C cconj(C a) { a.y = -a.y; return a; }
template <typename C, typename R> CM_DEVINL C cscale(C a, R s) { a.x *= s; a.y *= s; return a; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> CM_DEVINL C mul_mi(C a) {
  C r;
  if (INV) { r.x = -a.y; r.y = a.x; }
  else { r.x = a.y; r.y = -a.x; }
  return r;
}
template <typename C> CM_DEVINL C czero() { C r; r.x = 0; r.y = 0; return r; }
template <typename C, typename R> CM_DEVINL C cmake(R x, R y) { C r; r.x = x; r.y = y; return r; }

// Programmatic dependent launch.  pdl_trigger lets the next kernel of the
// stream start launching (its blocks are placed as this grid's blocks leave
// room); pdl_wait blocks until every preceding grid the launch depends on has
// completed and its memory is visible.  A kernel launched without the
// programmatic-serialization attribute was already ordered behind its
// predecessor, and both are no-ops for it.  Kernels read only constant
// inputs (twiddle tables, launch arguments) before pdl_wait.
CM_DEVINL void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
CM_DEVINL void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

#define CM_BARRIER_TIMEOUT_CYCLES 4000000000LL  // about two seconds

// ---------------------------------------------------------------------------
// bulk asynchronous copies global -> shared (TMA engine), completed on an
// mbarrier.  Sources and destinations 16-byte aligned, sizes multiples of 16.
// ---------------------------------------------------------------------------
CM_DEVINL unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

CM_DEVINL void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}

// make initialised mbarriers visible to the async proxy (before first use)
CM_DEVINL void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

CM_DEVINL void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes)
               : "memory");
}

// order this thread's view of global memory (written by the generic proxy of
// any block before the last grid barrier) before its following bulk copies
CM_DEVINL void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// order this thread's earlier shared-memory accesses (generic proxy) before
// its following bulk copies into the same shared memory
CM_DEVINL void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

CM_DEVINL void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(b))
      : "memory");
}

// Hint: start bringing [p, p + bytes) into L2 ahead of the loads that will
// read it.  Nothing is returned and nothing waits on it; L2 is the point of
// coherence, so a range written later by another kernel is still read
// correctly.  Skipped unless p is 16-byte aligned and bytes a multiple of 16.
CM_DEVINL void prefetch_l2(const void* p, size_t bytes) {
  if (bytes == 0 || ((reinterpret_cast<size_t>(p) | bytes) & 15) != 0) return;
  const char* c = static_cast<const char*>(p);
  for (size_t o = 0; o < bytes; o += 32768) {
    const unsigned n = (unsigned)(bytes - o < 32768 ? bytes - o : 32768);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c + o), "r"(n) : "memory");
  }
}

CM_DEVINL bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait for the completion of phase `parity` of mbarrier b; false after about
// two seconds (the copies it tracks read valid device memory and always
// complete, so this only bounds the wait).
CM_DEVINL bool mbar_wait(unsigned long long* b, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(b, parity))
    if (clock64() - t0 > CM_BARRIER_TIMEOUT_CYCLES) return false;
  return true;
}

// Division by a divisor that is fixed for a pass, as a high multiply and a
// shift (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): for d >= 2 with l = ceil(log2 d),
// m = ceil(2^(31+l) / d) < 2^32, and floor(x / d) = (x m) >> (31 + l) for
// every 0 <= x < 2^31.  The multiplier is computed on the host (one 64-bit
// division per divisor); m = 0 encodes d = 1.
struct FastDiv {
  unsigned d, m, s;  // divisor, multiplier, shift applied to the high word
};

inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f;
  f.d = d;
  f.m = 0;
  f.s = 0;
  if (d >= 2) {
    unsigned l = 0;
    while ((1ull << l) < d) ++l;
    f.m = (unsigned)(((1ull << (31 + l)) + d - 1) / d);
    f.s = l - 1;
  }
  return f;
}

// floor(x / f.d) for 0 <= x < 2^31
CM_DEVINL int fdiv(const FastDiv& f, int x) {
  return f.m ? (int)(__umulhi((unsigned)x, f.m) >> f.s) : x;
}

enum { RED_SUM = 0, RED_MAX = 1, RED_MIN = 2 };

CM_DEVINL double red_neutral(int kind) {
  return kind == RED_SUM ? 0.0 : (kind == RED_MAX ? -INFINITY : INFINITY);
}
CM_DEVINL double red_apply(int kind, double a, double b) {
  return kind == RED_SUM ? a + b : (kind == RED_MAX ? fmax(a, b) : fmin(a, b));
}

// Reduce NV doubles across the block with a fixed tree (deterministic).
// kinds[i] selects sum / max / min.  Result valid in thread 0.
// `sm` must hold 32*NV doubles.  All threads must call.
template <int NV>
CM_DEVINL void block_reduce(double (&v)[NV], const int (&kinds)[NV], double* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v[i] = red_apply(kinds[i], v[i], __shfl_xor_sync(0xffffffffu, v[i], o));
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) sm[i * 32 + warp] = v[i];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = lane < nw ? sm[i * 32 + lane] : red_neutral(kinds[i]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
        x = red_apply(kinds[i], x, __shfl_xor_sync(0xffffffffu, x, o));
      v[i] = x;
    }
  }
  __syncthreads();
}

// Loop over e in [0, n) with the block's threads, U indices per thread per
// round: all U loads are issued before any use, so U global loads are in
// flight per thread instead of one.
template <int U, typename LoadF, typename UseF>
CM_DEVINL void batched_loop(int n, LoadF load, UseF use) {
  typedef decltype(load(0)) V;
  const int T = blockDim.x;
  for (int e0 = threadIdx.x; e0 < n; e0 += U * T) {
    V v[U];
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const int e = e0 + i * T;
      if (e < n) v[i] = load(e);
    }
#pragma unroll
    for (int i = 0; i < U; ++i) {
      const int e = e0 + i * T;
      if (e < n) use(e, v[i]);
    }
  }
}
