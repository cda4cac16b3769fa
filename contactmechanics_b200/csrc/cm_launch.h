// Host-side declarations shared by the translation units of the library:
// launchers of the power-of-two passes (cm_op_p2.cu), of the persistent batch
// kernel (cm_batch.cu) and the types their callers need.
#pragma once
#include <cuda_runtime.h>

#include "cm_slot.cuh"


// Dynamic shared memory a transform kernel may use (of the 227 KB a block can
// hold on sm_100, leaving room for its static shared variables).
#define CM_SMEM_DYN_MAX (220 * 1024)


#define CM_P2_CASES(X) X(6) X(7) X(8) X(9) X(10) X(11) X(12)
// the by-value operator and solver passes also cover 2^13
#define CM_OP_P2_CASES(X) CM_P2_CASES(X) X(13)
// and lengths 3 * 2^m, m = 5..11 (96..6144), by their length codes 32 + m
#define CM_T3_CASES(X) X(37) X(38) X(39) X(40) X(41) X(42) X(43)
#define CM_OP_LEN_CASES(X) CM_OP_P2_CASES(X) CM_T3_CASES(X)

// The plain operator on power-of-two domains (cm_op_p2.cuh): three launches
// on stream s.  op_p2_supported: whether sides 2^logx x 2^logy with column
// tiles of width 2^lw can use it.  op_p2_apply returns 0 when launched, -1
// when not supported, 1 on a CUDA error.
// Arguments of the operator passes, passed by value to every launch.
template <typename R>
struct OpArgs {
  typedef typename CT<R>::C C;
  const R* in;
  R* out;
  int in_rows, in_cols, in_ld;
  int out_rows, out_cols, out_ld;
  int nx, nyh, lw;  // domain rows, half-spectrum columns, log2 of the table's column tiles
  int ny;           // domain columns (row length of the pair-major spectrum)
  R* fwd_real;      // column pass: forward transform only, its real part to this
                    // natural (nx, ny/2 + 1) array (nullptr: the operator)
  int ntile_cols;
  C* spec;
  const R* tab;     // the selected Green's table, tiled like the spectrum
  const C* twx;     // twiddles of length nx
  const C* twy;     // twiddles of length ny
  const CcgState* st;  // column pass of a solve: skip after convergence (else nullptr)
  int cg_only;         // ... and skip unless the iteration takes a CG step
};

// Arguments of the row passes of one CCG iteration (cm_ccg_p2.cuh).
template <typename R>
struct CcgArgs {
  OpArgs<R> op;  // geometry, spectrum, Green's table, twiddles
  R* u;          // (nx, ny)
  const R* h;    // (tx, ty)
  R* f[2];       // (tx, ty)
  R* t;          // (tx, ty)
  const unsigned char* gneg;
  CcgState* st;
  double* partials;
  unsigned int* counter;
  int tx, ty;
  int ny;        // row length of u (domain columns)
  int ew_grid;   // blocks of the vectorised element-wise passes
  int u_rows;    // rows of u the displacement pass updates: nx, or tx in the
                 // FP32 phase of a mixed solve (the padding's displacement
                 // feeds only max |du| and the result, which the FP64 phase
                 // recomputes from the forces)
  int fuse_gsum; // the displacement pass also forms the next iteration's G
                 // (FP32 phase of a mixed solve; the iterations then run
                 // without the gsum pass)
  FastDiv ew_vpr;  // 16-byte vectors per topography row (element-wise passes)
};
// Launch with programmatic stream serialization: the kernel may start while
// its predecessor on the stream finishes, and calls pdl_wait before reading
// anything an earlier kernel wrote.  Off when the environment sets CM_PDL=0.
bool pdl_enabled();
template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(bool chained, void (*kernel)(KArgs...), int grid, int block,
                                  size_t smem, cudaStream_t s, Args... args);
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem,
                              cudaStream_t s, Args... args) {
  return launch_chained(true, kernel, grid, block, smem, s, args...);
}
// launch_pdl when `chained` (a kernel of ours precedes it on the stream),
// else a plain launch
template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(bool chained, void (*kernel)(KArgs...), int grid, int block,
                                  size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = chained && pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename R>
int op_p2_supported(int logx, int logy, int lw);
template <typename R>
int op_p2_apply(const OpArgs<R>& a, int logx, int logy, cudaStream_t s);
// The row pass and a forward-only column pass writing the real part of the
// 2D transform to a.fwd_real (same return codes).
template <typename R>
int op_p2_fwd_real(const OpArgs<R>& a, int logx, int logy, cudaStream_t s);
// The passes of one CCG iteration of a single solve on a power-of-two domain
// (MODE_T: r = G t, MODE_F: u = G f), same return codes.
template <typename R, int MODE>
int ccg_p2_row_fwd(const CcgArgs<R>& a, int logy, cudaStream_t s);
template <typename R>
int ccg_p2_col(const OpArgs<R>& a, int logx, cudaStream_t s);
template <typename R, int MODE>
int ccg_p2_row_inv(const CcgArgs<R>& a, int logy, cudaStream_t s);
// Set the kernels' attributes and occupancy ahead of the first launch (which
// may be inside a stream capture): 0, -1 unsupported, 1 CUDA error.
template <typename R>
int ccg_p2_prepare(const CcgArgs<R>& a, int logx, int logy);
// The vectorised element-wise passes of the single-solve path (gsum, force
// update), chained behind the previous pass; grid a.ew_grid.
template <typename R>
int ccg_p2_gsum(const CcgArgs<R>& a, cudaStream_t s, bool chained);
template <typename R>
int ccg_p2_update(const CcgArgs<R>& a, cudaStream_t s, bool chained);
// Resident blocks per SM of those passes as a's solve launches them (for
// sizing a.ew_grid), or -1.
template <typename R>
int ccg_p2_ew_blocks_per_sm(const CcgArgs<R>& a);

// The persistent batch kernel (cm_batch.cu): one launch over n jobs taken in
// queue order `order` (next: a zeroed device counter), smem bytes of dynamic
// shared memory per block; *clusters receives the clusters launched.
// Returns 0 when launched.
int batch_solve_launch(const BatchJob* jobs, const int* order, int n, int* next, size_t smem,
                       cudaStream_t s, int* clusters);

