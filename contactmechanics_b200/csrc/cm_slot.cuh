// Per-solve descriptors shared by host and device code.
//
// One "slot" is one operator or one contact solve.  Every kernel takes an
// array of slots plus a list of work items (slot, tile) so the same kernels
// run a single solve or a batch of solves of different sizes in one launch.
#pragma once
#include "cm_fft.cuh"

// status codes written by the device and returned through the C ABI
enum {
  CMS_RUNNING = 0,
  CMS_CONVERGED = 1,
  CMS_MAXITER = 2,
  CMS_NAN = 3,
  CMS_BISECT_SIGN = 4,
};

// delta_str of the reference loop
enum { CMM_RESET = 0, CMM_SD = 1, CMM_CG = 2, CMM_MIX = 3 };

#define CM_BIS_CAND 31   // thresholds evaluated per bisection pass (5 levels)
#define CM_BISECT_PASSES 21  // bisection passes per mixing step: 105 levels >= scipy's 100 iterations
#define CMS_TIMEOUT 6  // solve status: a grid-barrier or bulk-copy wait gave up
#define CM_RED_MAX 8     // reduction values per kernel

struct CcgParams {
  double F;          // external force (load control)
  double offset0;    // rigid-body offset (offset control)
  double H;          // hardness in force units
  double pentol, forcetol, thermotol, mixfac, mixdecfac;
  double rel_forcetol;  // FP32 phases: forcetol >= rel_forcetol * max|f|
  double n_surface;  // number of topography points
  double max_surface;
  int load_control;
  int has_h;
  int minmixsteps;
  int maxiter;
};

struct CcgState {
  CcgParams p;
  int it;        // iteration being computed (1-based)
  int done;
  int status;
  int parity;    // which f buffer holds the force at the start of the iteration
  int mode;      // CMM_*
  int delta;
  int mixsteps;
  int branch;    // 0 = Polonsky-Keer (cg/sd) step, 1 = mixing step
  int apply_nc;
  int uniform;
  int have_last_tf, have_last_mh;
  int nfev;
  int bs_active, bs_iter;
  long long A_contact, A_cg, A_fl, n_nc;
  double G_old, G, beta, tau, offset, cur_mixfac, scale;
  double last_tf, last_mh;
  double sum_cg, sum_cgt, gmax, gmin;
  double max_pres, pad_pres, total_force, maxdu, max_pen, rms_pen, fmax;
  // scipy-compatible bisection state (offset of the mixing step)
  double bs_xa, bs_dm, bs_fa;
  double bs_cand[CM_BIS_CAND + 1];
  // the finished iteration's start-of-iteration values, kept by the
  // convergence test for the per-iteration observer (a fused pass may have
  // started the next iteration already)
  long long rep_area, rep_cg_area;
  double rep_offset;
  int rep_mode;
};

// Grid barrier (count of arrivals, generation, abort flag) of the kernels
// whose blocks meet inside a launch: the persistent solver and the
// bisection passes.  Zeroed with the solve's state.
struct GridBarrier {
  unsigned int count;
  unsigned int gen;
  unsigned int abort;
  unsigned int pad;
};

template <typename R>
struct Slot {
  typedef typename CT<R>::C C;
  // geometry: domain (nx, ny), half spectrum (nx, nyh), topography (tx, ty)
  int nx, ny, nyh, tx, ty;
  int row_tile, col_tile, comp_rows;       // tile shapes (col_tile = 2^lw)
  int lw;                                  // log2 of the spectrum column-tile width
  int nt_comp, nt_rowt, nt_rowd, nt_col;   // tiles over comp rows, rows<tx, rows<nx, columns
  FastDiv dv_ny, dv_nyh, dv_ty;            // the element loops' divisors
  FftDesc fx, fy;
  const C* twx;
  const C* twy;
  C* spec;
  const R* tab[2];    // 0: displacement table -G/(a N); 1: force table -K a/N
  // plain operator I/O
  const R* in;
  R* out;
  int in_rows, in_cols, in_ld, out_rows, out_cols, out_ld, table_sel;
  // contact solve fields
  const R* h;         // (tx, ty)
  R* u;               // (nx, ny)
  R* f[2];            // (tx, ty)
  R* t;               // (tx, ty)
  unsigned char* gneg;  // (tx, ty) gap < 0 of the last mixing-capable step (plastic only)
  CcgState* st;
  double* partials;
  unsigned int* counter;
  // lockstep batches: per-solve inputs and results of the batched set-up
  // and result kernels (unused elsewhere)
  const double* h64;        // FP64 heights (tx, ty)
  const double* u0;         // initial displacement (nx, ny) or null
  const float* prev_f[2];   // FP64 phase of a mixed solve: the FP32 phase's forces
  const CcgState* prev_st;  // ... and its state (which buffer holds them)
  double* x_out;            // results, each may be null
  double* jac_out;
  unsigned char* act_out;
  unsigned char* pl_out;
};

// One solve of the persistent batch kernel (cm_batch.cu): its slots of the
// two precisions, the initial state of each phase (the final ones go to the
// slots' st), the FP64 inputs and the result buffers.
struct BatchJob {
  Slot<float> s32;       // FP32 phase (prec CM_FP32 or CM_MIXED)
  Slot<double> s64;      // FP64 phase (prec CM_FP64 or CM_MIXED)
  CcgState init32, init64;
  const double* h64;     // heights (tx, ty)
  const double* u0;      // initial displacement (nx, ny) or null
  double* x;             // results, each may be null: displacement (nx, ny)
  double* jac;           // -force (tx, ty)
  unsigned char* active;   // (tx, ty)
  unsigned char* plastic;  // (tx, ty)
  int prec;              // CM_FP64 / CM_FP32 / CM_MIXED
  int pentol_auto;       // pentol from the heights (the reference's default)
  int maxiter;           // iteration budget of the whole solve
  double rel_pentol32;   // FP32 phase of a mixed solve: pentol >= this * (max h - min h)
};

