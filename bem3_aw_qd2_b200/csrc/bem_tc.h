// Tensor-core (tcgen05) trailing update of the complex FP32 LU; see bem_tc.cu.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#define LU_OUTER_W 128           // outer block of the LU (bem_lu.h BEM_LU_OB): the update's depth
#define BEM_TC_ST_WAIT 0x100u     // a tensor-core update wait gave up (no hang; result invalid)

struct bem_tc {
  float *Ap = nullptr, *Bp = nullptr;  // packed K-major operands (A'': L21 rows, B'': output columns)
  alignas(64) CUtensorMap tmA;         // 2D TMA maps of the packed operands
  alignas(64) CUtensorMap tmB;
  int n = 0, nprod = 0;                // largest size prepared; TF32 products per term (1 or 3)
  bool ready = false;
  char err[160] = {0};
};

extern "C" {
// packed-operand buffers and TMA maps for systems up to n (no allocation
// inside a stream capture: call before capturing)
int bem_tc_prepare(bem_tc *t, int n, int nprod);
// pack and launch the update of the outer block starting at column K of the
// row-major complex FP32 matrix M: M[r0:n, r0:n] -= M[r0:n, K:r0] M[K:r0, r0:n],
// r0 = K + LU_OUTER_W
void bem_tc_launch(bem_tc *t, float2 *M, long lda, int n, int K, unsigned *status, cudaStream_t st);
void bem_tc_free(bem_tc *t);
}
