// Launchers of the register-resident power-of-two FFT passes of the CCG
// iteration (kernels in cm_kernels_p2.cuh), one instantiation per side.
#include "cm_kernels_p2.cuh"
#include "cm_launch.h"

template <typename R, int MODE>
bool p2_row_fwd(int logn, int grid, int threads, size_t smem, cudaStream_t s, const Slot<R>* S,
                const int2* it) {
  switch (logn) {
#define CM_CASE(L) case L: k_row_fwd_p2<R, MODE, L><<<grid, threads, smem, s>>>(S, it); return true;
    CM_P2_CASES(CM_CASE)
#undef CM_CASE
    default: return false;
  }
}

template <typename R, int MODE>
bool p2_col(int logn, int grid, int threads, size_t smem, cudaStream_t s, const Slot<R>* S,
            const int2* it) {
  switch (logn) {
#define CM_CASE(L) case L: k_col_p2<R, MODE, L><<<grid, threads, smem, s>>>(S, it); return true;
    CM_P2_CASES(CM_CASE)
#undef CM_CASE
    default: return false;
  }
}

template <typename R, int MODE>
bool p2_row_inv(int logn, int grid, int threads, size_t smem, cudaStream_t s, const Slot<R>* S,
                const int2* it) {
  switch (logn) {
#define CM_CASE(L) case L: k_row_inv_p2<R, MODE, L><<<grid, threads, smem, s>>>(S, it); return true;
    CM_P2_CASES(CM_CASE)
#undef CM_CASE
    default: return false;
  }
}

template <typename R>
void set_p2_attrs() {
  bool done = false;
  if (done) return;
  done = true;
  const int mx = CM_SMEM_DYN_MAX;
  const int carve = cudaSharedmemCarveoutMaxShared;
#define CM_ATTR(K)                                                                  \
  cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);         \
  cudaFuncSetAttribute(K, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
#define CM_CASE(L)                           \
  CM_ATTR((k_row_fwd_p2<R, MODE_T, L>))      \
  CM_ATTR((k_row_fwd_p2<R, MODE_F, L>))      \
  CM_ATTR((k_col_p2<R, MODE_T, L>))          \
  CM_ATTR((k_col_p2<R, MODE_F, L>))          \
  CM_ATTR((k_row_inv_p2<R, MODE_T, L>))      \
  CM_ATTR((k_row_inv_p2<R, MODE_F, L>))
  CM_P2_CASES(CM_CASE)
#undef CM_CASE
#undef CM_ATTR
}


#define CM_INST(R, MODE)                                                                       \
  template bool p2_row_fwd<R, MODE>(int, int, int, size_t, cudaStream_t, const Slot<R>*,     \
                                    const int2*);                                             \
  template bool p2_col<R, MODE>(int, int, int, size_t, cudaStream_t, const Slot<R>*,         \
                                const int2*);                                                 \
  template bool p2_row_inv<R, MODE>(int, int, int, size_t, cudaStream_t, const Slot<R>*,     \
                                    const int2*);
CM_INST(float, MODE_T)
CM_INST(float, MODE_F)
CM_INST(double, MODE_T)
CM_INST(double, MODE_F)
#undef CM_INST
template void set_p2_attrs<float>();
template void set_p2_attrs<double>();
