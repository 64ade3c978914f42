// Trailing update of the complex FP32 LU on the fifth-generation tensor cores
// (tcgen05, Blackwell): C -= L21 U12 for one outer block (BEM_LU_OB = 128
// columns, four 32-column panels) of the mixed-precision factorisation
// (bem_lu.cu), in place of the CUDA-core update.  No counterpart in the
// reference, whose solves are FP64 (b_mkl_solver_pardiso_d,
// d3qd2_mkl_solver.c:18-148).
//
// The complex product is one real GEMM: a row of L21 read as 2K reals
// (re, im interleaved) times, for output column c, the 2K reals
// (Re U, -Im U) (real part) or (Im U, Re U) (imaginary part).  Operands are
// TF32 (kind::tf32, FP32 accumulation in TMEM).  With nprod = 3 each operand
// is split x = hi + lo (hi rounded to TF32) and the product is
// hi hi + hi lo + lo hi: close to FP32 accuracy; nprod = 1 is a single TF32
// product.  A pack kernel writes the operands K-major (A'' rows: L21 rows;
// B'' rows: per 64-column sub-tile, 64 real-part then 64 imaginary-part
// columns).  Each CTA computes a 128-row x 128-complex-column tile: one
// thread streams the 128-byte-wide K boxes of both operands with 2D TMA into
// a ring of shared-memory stages (128-byte swizzle), another issues the MMAs
// (M = 128, N = 256) into a 128 x 256 FP32 accumulator in TMEM and frees each
// stage with tcgen05.commit, and the four warps read the accumulator back
// (tcgen05.ld) and subtract it from C a row at a time.  Every wait on an mbarrier is bounded: a wait that
// gives up sets BEM_TC_ST_WAIT, waits (bounded) for the copies and MMAs in
// flight, frees the TMEM and returns.  The TMA loads read this GPU's own
// memory and use no multicast.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include "bem_tc.h"

#define TC_M 128        // rows of a tile (TMEM lanes)
#define TC_NC 64        // complex columns of a packed sub-tile (its 64 real then 64 imaginary B'' rows)
#define TC_NS 2         // sub-tiles of a CTA's tile: 128 complex columns
#define TC_N (2 * TC_NC * TC_NS)  // real accumulator columns of a tile (256: the MMA's N)
#define TC_TH 128       // four warps: one TMEM lane quarter each
#define TC_BOX_K 32     // FP32 elements per 128-byte swizzle row
#define TC_A_BYTES (TC_M * 128)   // an A box: TC_M rows x 128 bytes
#define TC_B_BYTES (TC_N * 128)   // a B box: TC_N rows x 128 bytes
#define TC_STAGE_BYTES (TC_A_BYTES + TC_B_BYTES)
#define TC_STAGES 2     // K boxes in flight (48 KB a stage)
#define TC_KR (2 * LU_OUTER_W)  // reals of one product part of a packed row
#define TC_WAIT_NS 1000000000ull  // one second

// ---------------------------------------------------------------- packing
// A'' [rows][TC_KR nprod]: [hi(a) | hi(a) | lo(a)] of the 2K reals of L21's
// row (nprod 3) or [a] (nprod 1); B'' [tile rows][TC_KR nprod]: [hi(b) |
// lo(b) | hi(b)] or [b] of the 2K reals of an output column (see above).
__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__global__ void k_tc_pack(const float2 *__restrict__ M, long lda, int n, int K, int r0, int nprod,
                          float *__restrict__ Ap, float *__restrict__ Bp, int rows, int ntiles) {
  const int kp = TC_KR * nprod;
  // A'': one thread per (row, k)
  const long na = (long)rows * LU_OUTER_W;
  const long nb = (long)ntiles * TC_NC * LU_OUTER_W;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < na + nb; e += (long)gridDim.x * blockDim.x) {
    if (e < na) {
      const int r = (int)(e / LU_OUTER_W), kk = (int)(e % LU_OUTER_W);
      const int row = r0 + r;
      const float2 a = row < n ? M[(size_t)row * lda + K + kk] : make_float2(0.f, 0.f);
      float *dst = Ap + (size_t)r * kp;
      if (nprod == 1) {
        dst[2 * kk] = a.x;
        dst[2 * kk + 1] = a.y;
      } else {
        const float hx = tf32_hi(a.x), hy = tf32_hi(a.y);
        dst[2 * kk] = hx; dst[2 * kk + 1] = hy;
        dst[TC_KR + 2 * kk] = hx; dst[TC_KR + 2 * kk + 1] = hy;
        dst[2 * TC_KR + 2 * kk] = a.x - hx; dst[2 * TC_KR + 2 * kk + 1] = a.y - hy;
      }
    } else {
      const long f = e - na;
      const int cc = (int)(f / LU_OUTER_W), kk = (int)(f % LU_OUTER_W);
      const int col = r0 + cc;
      const float2 b = col < n ? M[(size_t)(K + kk) * lda + col] : make_float2(0.f, 0.f);
      const int tile = cc / TC_NC, j = cc % TC_NC;
      float *re = Bp + (size_t)(tile * 2 * TC_NC + j) * kp, *im = Bp + (size_t)(tile * 2 * TC_NC + TC_NC + j) * kp;
      // real output: (Re b, -Im b); imaginary output: (Im b, Re b)
      const float v[4] = {b.x, -b.y, b.y, b.x};
      if (nprod == 1) {
        re[2 * kk] = v[0]; re[2 * kk + 1] = v[1];
        im[2 * kk] = v[2]; im[2 * kk + 1] = v[3];
      } else {
        float h[4];
        for (int q = 0; q < 4; ++q) h[q] = tf32_hi(v[q]);
        re[2 * kk] = h[0]; re[2 * kk + 1] = h[1];
        re[TC_KR + 2 * kk] = v[0] - h[0]; re[TC_KR + 2 * kk + 1] = v[1] - h[1];
        re[2 * TC_KR + 2 * kk] = h[0]; re[2 * TC_KR + 2 * kk + 1] = h[1];
        im[2 * kk] = h[2]; im[2 * kk + 1] = h[3];
        im[TC_KR + 2 * kk] = v[2] - h[2]; im[TC_KR + 2 * kk + 1] = v[3] - h[3];
        im[2 * TC_KR + 2 * kk] = h[2]; im[2 * TC_KR + 2 * kk + 1] = h[3];
      }
    }
  }
}

// ---------------------------------------------------------------- tcgen05 / TMA / mbarrier helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(phase)
      : "memory");
  return ok != 0;
}
// bounded wait on phase (one second by the global timer); false when it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t phase) {
  unsigned long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (uint32_t it = 0;; ++it) {
    if (mbar_try_wait(b, phase)) return true;
    if ((it & 63) == 63) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      if (t - t0 > TC_WAIT_NS) return false;
    }
  }
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(tm), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// instruction descriptor: D F32, A and B TF32, both K-major, N = 256, M = 128
#define TC_IDESC ((1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)TC_N >> 3 << 17) | ((uint32_t)TC_M >> 4 << 24))

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------- the update
// grid: (column tiles, row tiles); dynamic smem: TC_STAGES stages of an A box
// and a B box (TC_M rows x 128 bytes each)
__global__ void __launch_bounds__(TC_TH, 2)
    k_tc_update(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, float2 *C, long ldc,
                int n, int r0, int nbox, unsigned *status) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  __shared__ __align__(8) uint64_t bar_full[TC_STAGES], bar_empty[TC_STAGES], bar_done;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  unsigned char *sm = (unsigned char *)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int row_tile = r0 + blockIdx.y * TC_M;   // matrix row of the tile's first row
  const int col_tile = blockIdx.x;               // column tile (TC_NC x TC_NS complex columns)
  if (t == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(&bar_full[s], 1);
      mbar_init(&bar_empty[s], 1);
    }
    mbar_init(&bar_done, 1);
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TC_N)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  if (warp == 0 && lane == 0) {
    // producer: box b into stage b % TC_STAGES once the MMAs of box b - TC_STAGES freed it
    int issued = 0;
    for (int b = 0; b < nbox; ++b) {
      const int s = b % TC_STAGES;
      if (b >= TC_STAGES && !mbar_wait(&bar_empty[s], (uint32_t)((b / TC_STAGES) - 1) & 1u)) {
        atomicOr(status, BEM_TC_ST_WAIT);
        s_fail = 1;
        break;
      }
      unsigned char *sA = sm + (size_t)s * TC_STAGE_BYTES, *sB = sA + TC_A_BYTES;
      mbar_expect_tx(&bar_full[s], (uint32_t)TC_STAGE_BYTES);
      tma_load_2d(sA, &tmA, b * TC_BOX_K, row_tile - r0, &bar_full[s]);
      tma_load_2d(sB, &tmB, b * TC_BOX_K, col_tile * TC_N, &bar_full[s]);
      issued = b + 1;
    }
    // the copies still in flight land before the CTA may end (bounded)
    for (int b = issued > TC_STAGES ? issued - TC_STAGES : 0; b < issued; ++b)
      mbar_wait(&bar_full[b % TC_STAGES], (uint32_t)(b / TC_STAGES) & 1u);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: K steps of 8 TF32 (32 bytes) within each 128-byte swizzle row
    int done_boxes = 0;
    for (int b = 0; b < nbox; ++b) {
      const int s = b % TC_STAGES;
      if (!mbar_wait(&bar_full[s], (uint32_t)(b / TC_STAGES) & 1u)) {
        atomicOr(status, BEM_TC_ST_WAIT);
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(sm + (size_t)s * TC_STAGE_BYTES), b0 = a0 + TC_A_BYTES;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        tc_mma(tmem, umma_desc(a0 + 32u * ks), umma_desc(b0 + 32u * ks), (b | ks) ? 1u : 0u);
      tc_commit(&bar_empty[s]);
      done_boxes = b + 1;
    }
    tc_commit(&bar_done);  // every MMA this thread issued
    // the last stages' releases arrive before the CTA may end (bounded)
    for (int b = done_boxes > TC_STAGES ? done_boxes - TC_STAGES : 0; b < done_boxes; ++b)
      mbar_wait(&bar_empty[b % TC_STAGES], (uint32_t)(b / TC_STAGES) & 1u);
  }
  __syncthreads();
  // one lane per warp waits for the MMAs; the warp reads TMEM only together
  int ok = 1;
  {
    int got = 1;
    if (lane == 0 && !mbar_wait(&bar_done, 0)) {
      atomicOr(status, BEM_TC_ST_WAIT);
      got = 0;
      mbar_wait(&bar_done, 0);
    }
    ok = __shfl_sync(0xffffffffu, got, 0) && !s_fail;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    // warp w reads accumulator lanes 32 w .. 32 w + 31 (rows 32 w + lane of
    // the tile), 32 columns at a time, and turns them through shared memory
    // (the stages are free: every copy and MMA has completed) so that C is
    // read and written a row at a time, 32 consecutive columns per warp access
    float *tre = (float *)sm + warp * (2 * 32 * 33), *tim = tre + 32 * 33;
    const uint32_t tw = tmem + ((uint32_t)(32 * warp) << 16);
    // accumulator columns: per sub-tile u, 64 real-part then 64 imaginary-part columns
#pragma unroll 1
    for (int q = 0; q < 2 * TC_NS; ++q) {
      const int u = q >> 1, half = q & 1;
      const int col0 = r0 + (col_tile * TC_NS + u) * TC_NC + 32 * half;
      float re[32], im[32];
      tmem_ld32(tw + (uint32_t)(2 * TC_NC * u + 32 * half), re);
      tmem_ld32(tw + (uint32_t)(2 * TC_NC * u + TC_NC + 32 * half), im);
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        tre[lane * 33 + j] = re[j];
        tim[lane * 33 + j] = im[j];
      }
      __syncwarp();
      const int col = col0 + lane;
      // all 32 rows' loads in flight at once, then the stores
      float2 x[32];
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        const int row = row_tile + 32 * warp + r;
        x[r] = (row < n && col < n) ? C[(size_t)row * ldc + col] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        const int row = row_tile + 32 * warp + r;
        if (row < n && col < n)
          C[(size_t)row * ldc + col] = make_float2(x[r].x - tre[r * 33 + lane], x[r].y - tim[r * 33 + lane]);
      }
      __syncwarp();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_N) : "memory");
}

// ---------------------------------------------------------------- host side
typedef CUresult (*encode_tiled_t)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode(bem_tc *t, CUtensorMap *tm, float *base, int cols, long rows, int box_rows) {
  static encode_tiled_t fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void **)&fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      snprintf(t->err, sizeof(t->err), "cuTensorMapEncodeTiled not available");
      fn = nullptr;
      return -1;
    }
  }
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * sizeof(float)};
  const cuuint32_t box[2] = {TC_BOX_K, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  const CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    snprintf(t->err, sizeof(t->err), "tensor map encoding failed (%d)", (int)r);
    return -1;
  }
  return 0;
}

static size_t tc_smem() { return (size_t)TC_STAGES * TC_STAGE_BYTES + 1024; }

extern "C" int bem_tc_prepare(bem_tc *t, int n, int nprod) {
  if (nprod != 1 && nprod != 3) nprod = 3;
  if (t->ready && t->n >= n && t->nprod == nprod) return 0;
  cudaFree(t->Ap);
  cudaFree(t->Bp);
  t->Ap = t->Bp = nullptr;
  t->ready = false;
  const int kp = TC_KR * nprod;
  // rows a tile's TMA boxes may reach: A to the last row tile's end, B'' to
  // the last column tile's TC_N rows
  const long arows = n + TC_M, brows = (long)TC_N * ((n + TC_NC * TC_NS - 1) / (TC_NC * TC_NS) + 1);
  if (cudaMalloc(&t->Ap, (size_t)arows * kp * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&t->Bp, (size_t)brows * kp * sizeof(float)) != cudaSuccess) {
    snprintf(t->err, sizeof(t->err), "tensor-core update: out of device memory");
    return -1;
  }
  // rows a partial tile reads past the packed ones: zero until a pack writes
  // them (an accumulator row or column depends only on its own operand row)
  if (cudaMemset(t->Ap, 0, (size_t)arows * kp * sizeof(float)) != cudaSuccess ||
      cudaMemset(t->Bp, 0, (size_t)brows * kp * sizeof(float)) != cudaSuccess)
    return -1;
  if (encode(t, &t->tmA, t->Ap, kp, arows, TC_M) || encode(t, &t->tmB, t->Bp, kp, brows, TC_N)) return -1;
  if (cudaFuncSetAttribute(k_tc_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem()) != cudaSuccess) {
    snprintf(t->err, sizeof(t->err), "tensor-core update: shared memory attribute");
    return -1;
  }
  t->n = n;
  t->nprod = nprod;
  t->ready = true;
  return 0;
}

extern "C" void bem_tc_launch(bem_tc *t, float2 *M, long lda, int n, int K, unsigned *status, cudaStream_t st) {
  const int r0 = K + LU_OUTER_W;
  const int rows = n - r0;
  if (rows <= 0) return;
  const int ctiles = (rows + TC_NC * TC_NS - 1) / (TC_NC * TC_NS), rtiles = (rows + TC_M - 1) / TC_M;
  const int subtiles = ctiles * TC_NS;  // 64-column sub-tiles packed (the last ones may lie past n)
  const long work = (long)rows * LU_OUTER_W + (long)subtiles * TC_NC * LU_OUTER_W;
  const int pb = (int)((work + 255) / 256 < 8192 ? (work + 255) / 256 : 8192);
  k_tc_pack<<<pb, 256, 0, st>>>(M, lda, n, K, r0, t->nprod, t->Ap, t->Bp, rows, subtiles);
  const int nbox = TC_KR * t->nprod / TC_BOX_K;
  k_tc_update<<<dim3(ctiles, rtiles), TC_TH, tc_smem(), st>>>(t->tmA, t->tmB, M, lda, n, r0, nbox, status);
}

extern "C" void bem_tc_free(bem_tc *t) {
  cudaFree(t->Ap);
  cudaFree(t->Bp);
  *t = bem_tc();
}

// Give a complex FP32 LU (bem_lu) tensor-core trailing updates of its own
// (buffers for systems up to n); bem_lu_detach_tc releases them.  The
// mixed-precision solves own theirs (bem_mixed.tc); these serve direct users
// of bem_lu and its tests.
#include "bem_lu.h"
extern "C" int bem_lu_attach_tc(bem_lu *w, int n, int nprod) {
  bem_tc *t = new bem_tc();
  if (bem_tc_prepare(t, n, nprod)) {
    snprintf(w->err, sizeof(w->err), "%s", t->err);
    bem_tc_free(t);
    delete t;
    return -1;
  }
  w->tc = t;
  return 0;
}
extern "C" void bem_lu_detach_tc(bem_lu *w) {
  if (!w->tc) return;
  bem_tc_free(w->tc);
  delete w->tc;
  w->tc = nullptr;
}
