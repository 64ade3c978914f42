// Dense complex LU factorisation and solves on the device (no library): the
// FP64 path of the global boundary-integral system and of the per-domain dpv
// systems, replacing the reference's PARDISO (b_mkl_solver_pardiso_d,
// d3qd2_mkl_solver.c:18-148) and LAPACKE_zgesv (solve_dpv_bv,
// bem3_aw_qd2_solve_bieq.c:533-653).  See bem_lu.cu for the algorithm.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "bem_tc.h"

#define BEM_LU_W 32            // panel width (columns factored per panel)
#define BEM_LU_OB 128          // outer block: trailing updates right of it are applied once per block
#define BEM_LU_ST_ZERO 0x20u   // a zero pivot (singular matrix), as BEMGPU_ST_SOLVE
#define BEM_LU_ST_WAIT 0x40u   // a triangular-solve wait gave up (no hang; result invalid)
#define BEM_LU_ST_INTERNAL 0x80u  // a row move out of range (skipped; result invalid)

struct bem_lu {
  int *rowmap = nullptr;    // [n] original row of each position after pivoting
  size_t rowmap_cap = 0;
  int *piv = nullptr;       // panel scratch: selected pivot rows, candidates, permutation list
  void *u11 = nullptr;      // panel scratch: packed L11\U11, inverse of U11, inverse of L11, staged rows
  unsigned *status = nullptr;
  unsigned *flags = nullptr;  // triangular-solve progress counters (lower, upper), 128 bytes apart
  size_t flags_cap = 0;
  void *y = nullptr;          // triangular-solve intermediate (n x nrhs complex)
  size_t y_cap = 0;
  // the factorisation of one (matrix, size) as a CUDA graph, replayed while both stay the same
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  const void *g_A = nullptr;
  int g_n = 0, g_tc = -1, g_obm = 0;
  size_t g_nodes = 0;   // kernels in the captured graph (launch count per replay)
  bem_tc *tc = nullptr;       // complex FP32 only: trailing updates on the tensor cores when set
  cudaStream_t side = nullptr;  // second stream of the captured factorisation (look-ahead updates)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int sms = 0, coop_blocks = 0;  // device facts for the launches
  int one_block_max = 0;      // largest n factored as one outer block (0: the default, 2048)
  char err[200] = {0};
};

extern "C" {
int bem_lu_init(bem_lu *w, int device);
void bem_lu_free(bem_lu *w);
// In-place LU with row pivoting of the row-major n x n complex FP64 matrix A:
// P A = L U (L unit lower, U upper, both in A; w->rowmap holds P).
int bem_lu_factor_z(bem_lu *w, double *A, int n, cudaStream_t st);
// Solve A X = B with the factors of bem_lu_factor_z; B is n x nrhs complex,
// column-major (ld n), overwritten by X; nrhs <= 4.
int bem_lu_solve_z(bem_lu *w, const double *LU, int n, int nrhs, double *B, cudaStream_t st);
// The same in complex FP32 (interleaved re/im floats): the factors of the
// mixed-precision solves.
int bem_lu_factor_c(bem_lu *w, float *A, int n, cudaStream_t st);
int bem_lu_solve_c(bem_lu *w, const float *LU, int n, int nrhs, float *B, cudaStream_t st);
// R = B - A X in FP64 (A row-major n x n, X, B, R column-major n x nrhs,
// nrhs <= 4): the refinement residual.
int bem_lu_resid_z(const double *A, int n, int nrhs, const double *X, const double *B, double *R, cudaStream_t st);
// Largest n factored as one outer block (bem_lu.one_block_max; 0: default).
void bem_lu_set_one_block(bem_lu *w, int nmax);
// Status bits (BEM_LU_ST_*) accumulated since the last call; waits for st.
unsigned bem_lu_status(bem_lu *w, cudaStream_t st);
}
