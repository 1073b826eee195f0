// Learned warm start for the block-Davidson exciton solve (no counterpart in the reference).
//
// A per-transition MLP maps gauge-fixed band-edge data of basis state i = (k, c, v) -- the BSE
// diagonal (band-energy difference), the velocity matrix elements, the k position, the band
// indices and the sweep globals (Q, r0, eps) -- to 5 complex coefficients per wanted state s.
// The initial block is X[i, s] = sum_c coef[i, s, c] * carrier[c][i] with carriers
// 1, hx/|h|, hy/|h|, conj(hx)/|h|, conj(hy)/|h|, so the phase structure of the exciton
// envelopes is carried by the velocity matrix elements in the basis' own gauge.
//
// Network: 3 layers, width 512, SiLU; weights in BF16 (FP32 master copy for Adam), every
// GEMM on tcgen05 (bf16 inputs, FP32 accumulation in TMEM) through one stream-K kernel that
// writes C^T with red.add. Loss per sample (targets A = lowest eigenvectors of the plain
// dense FP64 solve, orthonormal): the distance to the nearest orthonormal basis of their span,
//   L = min_R unitary ||X - A R||_F^2 = tr(X^H X) - 2 ||A^H X||_* + 32   (mixing/phase-invariant)
// with R the polar factor of A^H X (Newton-Schulz); dL/dX = 2 (X - A R), backpropagated by
// hand-written kernels.
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

#include <cudaTypedefs.h>

#include "tc_sm100.cuh"

namespace {

using namespace tc;
using bf16 = __nv_bfloat16;

constexpr int NF = 32;      // input features (padded)
constexpr int WD = 512;     // hidden width
constexpr int NS = 32;      // states per block
constexpr int NCAR = 5;     // phase carriers
constexpr int NO = NS * NCAR * 2;   // 320 outputs

// ------------------------------------------------------------------ generic tcgen05 GEMM
// C^T += A B^T: A (M x K) and B (N x K) bf16 row-major (K contiguous), C stored column-major
// C[n * ldc + m] in FP32, accumulated with red.add (C must be cleared by the caller). Units are
// (128-row tile, BN-column tile, 32-wide K block); a persistent grid splits them stream-K.
constexpr int G_BM = 128, G_BK = 32, G_STAGES = 6, G_THREADS = 192;

struct GemmArgs {
  int M, N, BN, KB, NT;
  long long W;
  float* C;
  long long ldc;
  int* err;
};

__host__ __device__ inline uint32_t tmem_cols_for(int BN) {
  uint32_t n = 32;
  while (n < 2u * (uint32_t)BN) n <<= 1;
  return n;
}

__global__ void __launch_bounds__(G_THREADS, 1)
    k_gemm_bf16(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs a) {
  extern __shared__ unsigned char g_smem[];
  __shared__ __align__(8) uint64_t bars[2 * G_STAGES + 5];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t raw = smem_u32(g_smem);
  const uint32_t base = (raw + 1023u) & ~1023u;
  const int BN = a.BN;
  const uint32_t A_BYTES = G_BM * G_BK * 2u;
  const uint32_t STAGE = A_BYTES + (uint32_t)BN * G_BK * 2u;
  const uint32_t ncols = tmem_cols_for(BN);
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[G_STAGES]);
  const uint32_t accf0 = smem_u32(&bars[2 * G_STAGES]), acce0 = smem_u32(&bars[2 * G_STAGES + 2]);
  const uint32_t done = smem_u32(&bars[2 * G_STAGES + 4]);
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int i = 0; i < G_STAGES; ++i) {
      mbar_init(full0 + 8 * i, 1);
      mbar_init(empty0 + 8 * i, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, 4);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  volatile int* abort_flag = &s_abort;
  const long long W = a.W;
  const long long u0 = W * blockIdx.x / gridDim.x, u1 = W * (blockIdx.x + 1) / gridDim.x;
  const int KB = a.KB, NT = a.NT;

  if (warp == 0 && lane == 0) {
    long long it = 0;
    for (long long u = u0; u < u1; ++u, ++it) {
      const int s = (int)(it % G_STAGES);
      const long long r = it / G_STAGES;
      if (r > 0 && !mbar_wait(empty0 + 8 * s, (uint32_t)((r - 1) & 1), abort_flag)) break;
      const long long tile = u / KB;
      const int kb = (int)(u % KB), mt = (int)(tile / NT), nt = (int)(tile % NT);
      const uint32_t sa = base + (uint32_t)s * STAGE;
      mbar_expect_tx(full0 + 8 * s, STAGE);
      tma_load_2d(sa, &tmA, kb * G_BK, mt * G_BM, full0 + 8 * s);
      tma_load_2d(sa + A_BYTES, &tmB, kb * G_BK, nt * BN, full0 + 8 * s);
    }
    for (int s = 0; s < G_STAGES && s < it; ++s) {
      const long long last = (it - 1 - s) / G_STAGES;
      mbar_wait(full0 + 8 * s, (uint32_t)(last & 1), abort_flag, false);
    }
  } else if (warp == 1 && lane == 0) {
    const uint32_t idesc = idesc_bf16(G_BM, BN, false);
    long long it = 0, u = u0;
    int seg = 0;
    bool ok = true;
    while (u < u1 && ok) {
      const long long tile = u / KB;
      const long long uend = min(u1, (tile + 1) * KB);
      const int b = seg & 1;
      if (seg >= 2 && !mbar_wait(acce0 + 8 * b, (uint32_t)(((seg - 2) >> 1) & 1), abort_flag)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t dt = tmem + (uint32_t)b * (ncols / 2);
      uint32_t acc = 0;
      for (; u < uend; ++u, ++it) {
        const int s = (int)(it % G_STAGES);
        const long long r = it / G_STAGES;
        if (!mbar_wait(full0 + 8 * s, (uint32_t)(r & 1), abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = base + (uint32_t)s * STAGE, sb = sa + A_BYTES;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
          tc_mma(dt, sdesc(sa + kk * 32u), sdesc(sb + kk * 32u), idesc, acc);
          acc = 1;
        }
        tc_commit(empty0 + 8 * s);
      }
      if (!ok) break;
      tc_commit(accf0 + 8 * b);
      ++seg;
    }
    tc_commit(done);
    mbar_wait(done, 0, abort_flag, false);
  } else if (warp >= 2) {
    const int q = warp & 3;
    long long u = u0;
    int seg = 0;
    while (u < u1) {
      const long long tile = u / KB;
      const long long uend = min(u1, (tile + 1) * KB);
      const int mt = (int)(tile / NT), nt = (int)(tile % NT);
      const int b = seg & 1;
      if (!mbar_wait(accf0 + 8 * b, (uint32_t)((seg >> 1) & 1), abort_flag)) break;
      tc_fence_after();
      const int row = mt * G_BM + q * 32 + lane;
      const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)b * (ncols / 2);
      for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t v[32];
        tc_ld16(ta + (uint32_t)c0, v);
        if (c0 + 16 < BN) tc_ld16(ta + (uint32_t)c0 + 16u, v + 16);
        tc_wait_ld();
        if (row < a.M) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = nt * BN + c0 + j;
            if (c0 + j < BN && col < a.N) atomicAdd(a.C + (long long)col * a.ldc + row, __uint_as_float(v[j]));
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce0 + 8 * b);
      u = uend;
      ++seg;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
  if (threadIdx.x == 0 && s_abort) atomicExch(a.err, 1);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

int encode_2d(wtbg_ctx* ctx, CUtensorMap* map, const void* ptr, unsigned long long inner, unsigned long long rows,
              unsigned long long pitch_bytes, unsigned box_rows) {
  auto fn = encode_fn();
  if (!fn) return set_err(ctx, WTBG_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t dims[2] = {inner, rows};
  cuuint64_t strides[1] = {pitch_bytes};
  cuuint32_t box[2] = {(cuuint32_t)G_BK, box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_err(ctx, WTBG_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return WTBG_OK;
}

}  // namespace

// C^T (N x M, ldc) (+)= A (M x K, lda) B (N x K, ldb)^T; K a multiple of 8, pitches multiples of 8.
int gemm_bf16(wtbg_ctx* ctx, int* err, const bf16* A, long long lda, int M, int K, const bf16* B, long long ldb, int N,
              float* C, long long ldc, bool clear) {
  if (M <= 0 || N <= 0 || K <= 0) return WTBG_OK;
  if ((K % 8) || (lda % 8) || (ldb % 8)) return set_err(ctx, WTBG_ERR_ARG, "gemm_bf16: K and pitches must be multiples of 8");
  const int ntile = (N + 255) / 256;
  const int BN = std::max(32, ((N + ntile - 1) / ntile + 15) / 16 * 16);
  alignas(64) CUtensorMap ma, mb;
  if (int r = encode_2d(ctx, &ma, A, (unsigned long long)K, (unsigned long long)M, (unsigned long long)lda * 2, G_BM))
    return r;
  if (int r = encode_2d(ctx, &mb, B, (unsigned long long)K, (unsigned long long)N, (unsigned long long)ldb * 2,
                        (unsigned)BN))
    return r;
  if (clear) CK(cudaMemsetAsync(C, 0, (size_t)N * ldc * sizeof(float), ctx->stream));
  GemmArgs g;
  g.M = M;
  g.N = N;
  g.BN = BN;
  g.KB = (K + G_BK - 1) / G_BK;
  g.NT = (N + BN - 1) / BN;
  const long long MT = (M + G_BM - 1) / G_BM;
  g.W = MT * g.NT * g.KB;
  g.C = C;
  g.ldc = ldc;
  g.err = err;
  int dev = 0, nsm = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const size_t smem = (size_t)G_STAGES * (G_BM * G_BK * 2 + (size_t)BN * G_BK * 2) + 1024;
  CK(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(G_STAGES * (G_BM * G_BK * 2 + 256 * G_BK * 2) + 1024)));
  const int grid = (int)std::min<long long>(nsm, g.W);
  k_gemm_bf16<<<grid, G_THREADS, smem, ctx->stream>>>(ma, mb, g);
  WTBG_COUNT(ctx, 1);
  CKL("k_gemm_bf16");
  return WTBG_OK;
}

namespace {

// ------------------------------------------------------------------ elementwise kernels
__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float sg = 1.0f / (1.0f + __expf(-z));
  return sg * (1.0f + z * (1.0f - sg));
}

// ZT [Wd][M] (+= bias in place); H [M][Wd] and HT [Wd][M] = silu(Z) in bf16. Block (32, 8),
// 32 x 32 tiles (w, m).
__global__ void k_bias_silu(float* ZT, const float* bias, int Wd, long long M, bf16* H, bf16* HT) {
  __shared__ float t[32][33];
  const long long m0 = (long long)blockIdx.x * 32;
  const int w0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int r = ty; r < 32; r += 8) {
    const int w = w0 + r;
    const long long m = m0 + tx;
    float h = 0.0f;
    if (w < Wd && m < M) {
      const float z = ZT[(long long)w * M + m] + bias[w];
      ZT[(long long)w * M + m] = z;
      h = silu(z);
      HT[(long long)w * M + m] = __float2bfloat16(h);
    }
    t[r][tx] = h;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const long long m = m0 + r;
    const int w = w0 + tx;
    if (w < Wd && m < M) H[m * Wd + w] = __float2bfloat16(t[tx][r]);
  }
}

// OT [NO][M] += bias
__global__ void k_bias(float* OT, const float* bias, int No, long long M) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int o = blockIdx.y;
  if (m < M) OT[(long long)o * M + m] += bias[o];
}

// X [ns][M] complex (column-major per sample row block) from OT and the carriers CAR [NCAR][M]
__global__ void k_combine(const float* OT, const float2* CAR, long long M, float2* X) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (m >= M) return;
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll
  for (int c = 0; c < NCAR; ++c) {
    const float re = OT[(long long)((s * NCAR + c) * 2) * M + m];
    const float im = OT[(long long)((s * NCAR + c) * 2 + 1) * M + m];
    const float2 z = CAR[(long long)c * M + m];
    acc.x += re * z.x - im * z.y;
    acc.y += re * z.y + im * z.x;
  }
  X[(long long)s * M + m] = acc;
}

// per-sample 32 x 32 complex grams P = A^H X and G = X^H X over the rows of sample `smp`:
// grid (chunks, nsamp), partials part[smp][chunk][2][32][32]
constexpr int CG_ROWS = 16;
__global__ void __launch_bounds__(256) k_cgram2(const float2* A, const float2* X, long long M, int rows, int nchunk,
                                                float2* part) {
  __shared__ float2 as[CG_ROWS][NS + 1], xs[CG_ROWS][NS + 1];
  const int smp = blockIdx.y, ch = blockIdx.x;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const long long r0 = (long long)smp * rows;
  const int per = (rows + nchunk - 1) / nchunk;
  const int c0 = ch * per, c1 = min(rows, c0 + per);
  float2 pa[2][2], pg[2][2];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) pa[i][j] = pg[i][j] = make_float2(0.f, 0.f);
  for (int b = c0; b < c1; b += CG_ROWS) {
    __syncthreads();
    for (int it = tid; it < CG_ROWS * NS; it += 256) {
      const int rr = it % CG_ROWS, s = it / CG_ROWS;
      const bool ok = b + rr < c1;
      as[rr][s] = ok ? A[(long long)s * M + r0 + b + rr] : make_float2(0.f, 0.f);
      xs[rr][s] = ok ? X[(long long)s * M + r0 + b + rr] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int rr = 0; rr < CG_ROWS; ++rr) {
      for (int i = 0; i < 2; ++i) {
        const float2 a_ = as[rr][tx + 16 * i], x_ = xs[rr][tx + 16 * i];
        for (int j = 0; j < 2; ++j) {
          const float2 y = xs[rr][ty + 16 * j];
          // conj(a) y, conj(x) y
          pa[i][j].x += a_.x * y.x + a_.y * y.y;
          pa[i][j].y += a_.x * y.y - a_.y * y.x;
          pg[i][j].x += x_.x * y.x + x_.y * y.y;
          pg[i][j].y += x_.x * y.y - x_.y * y.x;
        }
      }
    }
  }
  float2* out = part + ((long long)smp * nchunk + ch) * 2 * NS * NS;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      const int a = tx + 16 * i, b = ty + 16 * j;
      out[a + b * NS] = pa[i][j];
      out[NS * NS + a + b * NS] = pg[i][j];
    }
}

__global__ void k_cgram2_sum(const float2* part, int nchunk, float2* PG) {
  const int smp = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * NS * NS) return;
  double sx = 0, sy = 0;
  for (int c = 0; c < nchunk; ++c) {
    const float2 v = part[((long long)smp * nchunk + c) * 2 * NS * NS + i];
    sx += v.x;
    sy += v.y;
  }
  PG[(long long)smp * 3 * NS * NS + i] = make_float2((float)sx, (float)sy);
}

// R = polar factor of P (P = R H, R unitary) by Newton-Schulz, Y <- Y (3I - Y^H Y) / 2 from
// Y0 = P / ||P||_F; one 1024-thread block per sample, R stored after P and G.
__global__ void __launch_bounds__(1024) k_polar(float2* PG, int iters) {
  __shared__ float2 Y[NS][NS + 1], T[NS][NS + 1];
  __shared__ float red[32];
  const int smp = blockIdx.x;
  float2* P = PG + (long long)smp * 3 * NS * NS;
  float2* R = P + 2 * NS * NS;
  const int a = threadIdx.x % NS, b = threadIdx.x / NS;
  const float2 p = P[a + b * NS];
  float n2 = p.x * p.x + p.y * p.y;
  for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = n2;
  __syncthreads();
  float fro = 0.f;
  for (int k = 0; k < 32; ++k) fro += red[k];
  fro = sqrtf(fro);
  Y[a][b] = fro > 0.f ? make_float2(p.x / fro, p.y / fro) : make_float2(a == b ? 1.f : 0.f, 0.f);
  __syncthreads();
  for (int it = 0; it < iters; ++it) {
    float2 g = make_float2(0.f, 0.f);
    for (int k = 0; k < NS; ++k) {
      const float2 u = Y[k][a], v = Y[k][b];
      g.x += u.x * v.x + u.y * v.y;
      g.y += u.x * v.y - u.y * v.x;
    }
    T[a][b] = make_float2((a == b ? 3.f : 0.f) - g.x, -g.y);
    __syncthreads();
    float2 y = make_float2(0.f, 0.f);
    for (int k = 0; k < NS; ++k) {
      const float2 u = Y[a][k], v = T[k][b];
      y.x += u.x * v.x - u.y * v.y;
      y.y += u.x * v.y + u.y * v.x;
    }
    __syncthreads();
    Y[a][b] = make_float2(0.5f * y.x, 0.5f * y.y);
    __syncthreads();
  }
  R[a + b * NS] = Y[a][b];
}

// loss per sample = ||X - A R||^2 = tr(G) - 2 Re tr(R^H P) + NS (scaled); one block per sample
__global__ void k_loss(const float2* PG, int nsamp, float scale, float* loss) {
  __shared__ float red[256];
  const int smp = blockIdx.x;
  const float2* P = PG + (long long)smp * 3 * NS * NS;
  const float2* G = P + NS * NS;
  const float2* R = P + 2 * NS * NS;
  float acc = 0.f;
  for (int i = threadIdx.x; i < NS * NS; i += blockDim.x) {
    const int a = i % NS, b = i / NS;
    const float2 p = P[i], r = R[i];
    acc -= 2.f * (r.x * p.x + r.y * p.y);
    if (a == b) acc += G[i].x + 1.f;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] * scale);
}

// dL/dX -> dO (bf16, [M][NO] and [NO][M]) and db3 (atomics): G_X = 2 (X - A R),
// dO[(s,c) re] = Re(conj(GX) car_c), dO[(s,c) im] = -Im(conj(GX) car_c); all scaled by `scale`.
__global__ void __launch_bounds__(128) k_dout(const float2* A, const float2* X, const float2* PG, const float2* CAR,
                                              long long M, int rows, float scale, bf16* dO, bf16* dOT, float* db3) {
  __shared__ float2 Rs[NS * NS];
  __shared__ float dbs[NO];
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long mfirst = (long long)blockIdx.x * blockDim.x;
  const int smp = (int)(mfirst / rows);
  const float2* R = PG + (long long)smp * 3 * NS * NS + 2 * NS * NS;
  for (int i = threadIdx.x; i < NS * NS; i += blockDim.x) Rs[i] = R[i];
  for (int i = threadIdx.x; i < NO; i += blockDim.x) dbs[i] = 0.f;
  __syncthreads();
  // a block covers rows of at most two samples (rows >= blockDim): pass 1 handles the second
  for (int pass = 0; pass < 2; ++pass) {
    const int sm = smp + pass;
    const bool act = m < M && (m / rows) == sm;
    if (pass == 1) {
      __syncthreads();
      const long long mlast = min(M, mfirst + (long long)blockDim.x) - 1;
      if (mlast / rows == smp) break;
      const float2* R2 = PG + (long long)sm * 3 * NS * NS + 2 * NS * NS;
      for (int i = threadIdx.x; i < NS * NS; i += blockDim.x) Rs[i] = R2[i];
      __syncthreads();
    }
    if (act) {
      float2 a[NS];
      for (int s = 0; s < NS; ++s) a[s] = A[(long long)s * M + m];
      float2 car[NCAR];
      for (int c = 0; c < NCAR; ++c) car[c] = CAR[(long long)c * M + m];
      for (int s = 0; s < NS; ++s) {
        float2 ar = make_float2(0.f, 0.f);
        for (int t = 0; t < NS; ++t) {
          const float2 r = Rs[t + s * NS];
          ar.x += a[t].x * r.x - a[t].y * r.y;
          ar.y += a[t].x * r.y + a[t].y * r.x;
        }
        const float2 x = X[(long long)s * M + m];
        const float gx = scale * 2.f * (x.x - ar.x);
        const float gy = scale * 2.f * (x.y - ar.y);
        for (int c = 0; c < NCAR; ++c) {
          const float re = gx * car[c].x + gy * car[c].y;
          const float im = gx * car[c].y - gy * car[c].x;
          const int o = (s * NCAR + c) * 2;
          const bf16 bre = __float2bfloat16(re), bim = __float2bfloat16(-im);
          dO[m * NO + o] = bre;
          dO[m * NO + o + 1] = bim;
          dOT[(long long)o * M + m] = bre;
          dOT[(long long)(o + 1) * M + m] = bim;
          atomicAdd(&dbs[o], re);
          atomicAdd(&dbs[o + 1], -im);
        }
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NO; i += blockDim.x)
    if (dbs[i] != 0.f) atomicAdd(&db3[i], dbs[i]);
}

// dZ = dH * silu'(Z): dHT, ZT [Wd][M] fp32 -> dZ [M][Wd] and dZT [Wd][M] bf16, db += sum_m dZ
__global__ void k_silu_back(const float* dHT, const float* ZT, int Wd, long long M, bf16* dZ, bf16* dZT, float* db) {
  __shared__ float t[32][33];
  __shared__ float cs[32];
  const long long m0 = (long long)blockIdx.x * 32;
  const int w0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  if (ty == 0) cs[tx] = 0.f;
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int w = w0 + r;
    const long long m = m0 + tx;
    float g = 0.f;
    if (w < Wd && m < M) {
      const long long o = (long long)w * M + m;
      g = dHT[o] * dsilu(ZT[o]);
      if (dZT) dZT[o] = __float2bfloat16(g);
    }
    t[r][tx] = g;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const long long m = m0 + r;
    const int w = w0 + tx;
    const float g = t[tx][r];
    if (w < Wd && m < M && dZ) dZ[m * Wd + w] = __float2bfloat16(g);
    atomicAdd(&cs[tx], g);
  }
  __syncthreads();
  if (ty == 0 && w0 + tx < Wd) atomicAdd(&db[w0 + tx], cs[tx]);
}

// bf16 transpose: in [M][C] -> out [C][M]
__global__ void k_transpose_bf16(const bf16* in, int Cn, long long M, bf16* out) {
  __shared__ bf16 t[32][34];
  const long long m0 = (long long)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int r = ty; r < 32; r += 8) {
    const long long m = m0 + r;
    const int c = c0 + tx;
    t[r][tx] = (m < M && c < Cn) ? in[m * Cn + c] : __float2bfloat16(0.f);
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int c = c0 + r;
    const long long m = m0 + tx;
    if (m < M && c < Cn) out[(long long)c * M + m] = t[tx][r];
  }
}

// Adam on a weight W [out][in] (fp32 master) with its gradient given transposed gT [in][out];
// writes W (bf16 [out][in]) and Wt (bf16 [in][out]).
__global__ void k_adam_w(float* W, float* m1, float* m2, const float* gT, int out, int in, float lr, float b1, float b2,
                         float c1, float c2, float eps, bf16* Wb, bf16* Wtb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= out * in) return;
  const int o = i / in, k = i % in;
  const float g = gT[(long long)k * out + o];
  const float a = b1 * m1[i] + (1.f - b1) * g;
  const float v = b2 * m2[i] + (1.f - b2) * g * g;
  m1[i] = a;
  m2[i] = v;
  const float w = W[i] - lr * (a / c1) / (sqrtf(v / c2) + eps);
  W[i] = w;
  const bf16 wb = __float2bfloat16(w);
  Wb[i] = wb;
  Wtb[(long long)k * out + o] = wb;
}

__global__ void k_adam_b(float* B, float* m1, float* m2, const float* g, int n, float lr, float b1, float b2, float c1,
                         float c2, float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float a = b1 * m1[i] + (1.f - b1) * g[i];
  const float v = b2 * m2[i] + (1.f - b2) * g[i] * g[i];
  m1[i] = a;
  m2[i] = v;
  B[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

__global__ void k_to_bf16_pair(const float* W, int out, int in, bf16* Wb, bf16* Wtb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= out * in) return;
  const int o = i / in, k = i % in;
  const bf16 wb = __float2bfloat16(W[i]);
  Wb[i] = wb;
  Wtb[(long long)k * out + o] = wb;
}

// ------------------------------------------------------------------ features of the basis
// glob: qx, qy, qz (1/Angstrom), r0 (Angstrom), eps_env
__global__ void k_dmin(const double2* H, long long N, double* out) {
  __shared__ double red[1024];
  double mn = 1e300;
  for (long long i = threadIdx.x; i < N; i += blockDim.x) mn = fmin(mn, H[i + i * N].x);
  red[threadIdx.x] = mn;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

struct FeatArgs {
  const double2* H;
  const double2* h;   // [5][N]
  const double* kpt;  // [nk][3]
  const double* dmin;
  long long N;
  int nc, nv;
  double a1[3], a2[3];
  double q[3], r0, eps;
  bf16* F;            // [rowoff + i][NF]
  float2* CAR;        // [NCAR][M] at column offset rowoff
  long long M, rowoff;
};

__global__ void k_features(FeatArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const int ncv = a.nc * a.nv;
  const long long k = i / ncv;
  const int c = (int)((i % ncv) / a.nv), v = (int)(i % a.nv);
  const double d = a.H[i + i * a.N].x - *a.dmin;
  const double2 hx = a.h[i], hy = a.h[a.N + i];
  const double hx2 = hx.x * hx.x + hx.y * hx.y, hy2 = hy.x * hy.x + hy.y * hy.y;
  const double h2 = hx2 + hy2;
  const double inv2 = h2 > 1e-60 ? 1.0 / h2 : 0.0;
  const double rxy = (hx.x * hy.x + hx.y * hy.y) * inv2, ixy = (hx.y * hy.x - hx.x * hy.y) * inv2;
  const double* kp = a.kpt + 3 * k;
  const double f1 = (kp[0] * a.a1[0] + kp[1] * a.a1[1] + kp[2] * a.a1[2]);
  const double f2 = (kp[0] * a.a2[0] + kp[1] * a.a2[1] + kp[2] * a.a2[2]);
  const double qm = sqrt(a.q[0] * a.q[0] + a.q[1] * a.q[1] + a.q[2] * a.q[2]);
  float f[NF];
  for (int j = 0; j < NF; ++j) f[j] = 0.f;
  f[0] = (float)d;
  f[1] = (float)exp(-d / 0.05);
  f[2] = (float)exp(-d / 0.2);
  f[3] = (float)exp(-d / 1.0);
  f[4] = (float)(hx2 * inv2);
  f[5] = (float)rxy;
  f[6] = (float)ixy;
  f[7] = (float)(log10(h2 + 1e-12) / 10.0);
  f[8] = (float)cos(f1);
  f[9] = (float)sin(f1);
  f[10] = (float)cos(f2);
  f[11] = (float)sin(f2);
  if (c < 4) f[12 + c] = 1.f;
  if (v < 4) f[16 + v] = 1.f;
  f[20] = (float)qm;
  f[21] = (float)(a.r0 / 60.0);
  f[22] = (float)(a.eps / 5.0);
  f[23] = (float)(1.0 / a.eps);
  f[24] = 1.f;
  bf16* out = a.F + (a.rowoff + i) * NF;
  for (int j = 0; j < NF; ++j) out[j] = __float2bfloat16(f[j]);
  const double inv = h2 > 1e-60 ? 1.0 / sqrt(h2) : 0.0;
  const long long col = a.rowoff + i;
  a.CAR[col] = make_float2(1.f, 0.f);
  a.CAR[a.M + col] = make_float2((float)(hx.x * inv), (float)(hx.y * inv));
  a.CAR[2 * a.M + col] = make_float2((float)(hy.x * inv), (float)(hy.y * inv));
  a.CAR[3 * a.M + col] = make_float2((float)(hx.x * inv), (float)(-hx.y * inv));
  a.CAR[4 * a.M + col] = make_float2((float)(hy.x * inv), (float)(-hy.y * inv));
}

// targets: host N x NS complex128 -> [NS][M] float2 at row offset
__global__ void k_targets(const double2* A, long long N, long long M, long long rowoff, float2* T) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (i >= N) return;
  const double2 z = A[i + (long long)s * N];
  T[(long long)s * M + rowoff + i] = make_float2((float)z.x, (float)z.y);
}

}  // namespace

// ------------------------------------------------------------------ network object
struct wtbg_net {
  wtbg_ctx* ctx = nullptr;
  unsigned long long seed = 0;
  long long rows = 0;          // rows per sample (N of the basis)
  int nsamp = 0, cap = 0;      // stored samples, capacity
  // parameters (fp32 master), Adam moments, bf16 copies
  DevBuf P, M1, M2, G;         // flat fp32: W1, b1, W2, b2, W3, b3
  DevBuf Wb;                   // bf16: W1b, W1tb, W2b, W2tb, W3b, W3tb
  long long step = 0;
  // training store
  DevBuf F, CAR, T;            // [cap*rows][NF] bf16, [NCAR][cap*rows] float2, [NS][cap*rows] float2
  // batch work
  DevBuf work;
  long long work_rows = 0;
  DevBuf err, loss, small;
};

namespace {

constexpr long long OFF_W1 = 0, OFF_B1 = OFF_W1 + (long long)WD * NF, OFF_W2 = OFF_B1 + WD,
                    OFF_B2 = OFF_W2 + (long long)WD * WD, OFF_W3 = OFF_B2 + WD, OFF_B3 = OFF_W3 + (long long)NO * WD,
                    NPARAM = OFF_B3 + NO;
constexpr long long BOFF_W1 = 0, BOFF_W1T = BOFF_W1 + (long long)WD * NF, BOFF_W2 = BOFF_W1T + (long long)WD * NF,
                    BOFF_W2T = BOFF_W2 + (long long)WD * WD, BOFF_W3 = BOFF_W2T + (long long)WD * WD,
                    BOFF_W3T = BOFF_W3 + (long long)NO * WD, NBF = BOFF_W3T + (long long)NO * WD;

struct Work {
  bf16 *Fin, *FinT, *H1, *H1T, *H2, *H2T, *dO, *dOT, *dZ2, *dZ2T, *dZ1T;
  float *Z1T, *Z2T, *OT, *dH2T, *dH1T;
  float2 *X, *Tt, *CARb, *part, *PG;
};

size_t work_bytes(long long M) {
  size_t b = 0;
  b += (size_t)M * NF * 2 * 2;          // Fin, FinT
  b += (size_t)M * WD * 2 * 4;          // H1, H1T, H2, H2T
  b += (size_t)M * NO * 2 * 2;          // dO, dOT
  b += (size_t)M * WD * 2 * 3;          // dZ2, dZ2T, dZ1T
  b += (size_t)M * WD * 4 * 4;          // Z1T, Z2T, dH2T, dH1T
  b += (size_t)M * NO * 4;              // OT
  b += (size_t)M * NS * 8 * 2;          // X, Tt
  b += (size_t)M * NCAR * 8;            // CARb
  b += 64 * 64 * 2 * NS * NS * 8 + 64 * 3 * NS * NS * 8 + 64 * 256;
  return b;
}

Work carve(char* p, long long M) {
  Work w;
  auto take = [&](size_t bytes) {
    char* r = p;
    p += (bytes + 255) / 256 * 256;
    return r;
  };
  w.Fin = (bf16*)take((size_t)M * NF * 2);
  w.FinT = (bf16*)take((size_t)M * NF * 2);
  w.H1 = (bf16*)take((size_t)M * WD * 2);
  w.H1T = (bf16*)take((size_t)M * WD * 2);
  w.H2 = (bf16*)take((size_t)M * WD * 2);
  w.H2T = (bf16*)take((size_t)M * WD * 2);
  w.dO = (bf16*)take((size_t)M * NO * 2);
  w.dOT = (bf16*)take((size_t)M * NO * 2);
  w.dZ2 = (bf16*)take((size_t)M * WD * 2);
  w.dZ2T = (bf16*)take((size_t)M * WD * 2);
  w.dZ1T = (bf16*)take((size_t)M * WD * 2);
  w.Z1T = (float*)take((size_t)M * WD * 4);
  w.Z2T = (float*)take((size_t)M * WD * 4);
  w.dH2T = (float*)take((size_t)M * WD * 4);
  w.dH1T = (float*)take((size_t)M * WD * 4);
  w.OT = (float*)take((size_t)M * NO * 4);
  w.X = (float2*)take((size_t)M * NS * 8);
  w.Tt = (float2*)take((size_t)M * NS * 8);
  w.CARb = (float2*)take((size_t)M * NCAR * 8);
  w.part = (float2*)take((size_t)64 * 64 * 2 * NS * NS * 8);
  w.PG = (float2*)take((size_t)64 * 3 * NS * NS * 8);
  return w;
}

int ensure_work(wtbg_net* net, long long M) {
  wtbg_ctx* ctx = net->ctx;
  if (int r = ensure(ctx, net->work, work_bytes(M) + 64 * 256)) return r;
  net->work_rows = M;
  return WTBG_OK;
}

const float* pf(const wtbg_net* n, long long off) { return n->P.as<float>() + off; }
float* gf(wtbg_net* n, long long off) { return n->G.as<float>() + off; }
const bf16* bfp(const wtbg_net* n, long long off) { return n->Wb.as<bf16>() + off; }

// forward over M rows: Fin (+FinT when training) filled; leaves X
int forward(wtbg_net* net, Work& w, long long M, const float2* CAR) {
  wtbg_ctx* ctx = net->ctx;
  cudaStream_t s = ctx->stream;
  int* err = net->err.as<int>();
  const dim3 tb(32, 8);
  if (int r = gemm_bf16(ctx, err, w.Fin, NF, (int)M, NF, bfp(net, BOFF_W1), NF, WD, w.Z1T, M, true)) return r;
  k_bias_silu<<<dim3((unsigned)((M + 31) / 32), WD / 32), tb, 0, s>>>(w.Z1T, pf(net, OFF_B1), WD, M, w.H1, w.H1T);
  WTBG_COUNT(ctx, 1);
  if (int r = gemm_bf16(ctx, err, w.H1, WD, (int)M, WD, bfp(net, BOFF_W2), WD, WD, w.Z2T, M, true)) return r;
  k_bias_silu<<<dim3((unsigned)((M + 31) / 32), WD / 32), tb, 0, s>>>(w.Z2T, pf(net, OFF_B2), WD, M, w.H2, w.H2T);
  WTBG_COUNT(ctx, 1);
  if (int r = gemm_bf16(ctx, err, w.H2, WD, (int)M, WD, bfp(net, BOFF_W3), WD, NO, w.OT, M, true)) return r;
  k_bias<<<dim3((unsigned)((M + 255) / 256), NO), 256, 0, s>>>(w.OT, pf(net, OFF_B3), NO, M);
  WTBG_COUNT(ctx, 1);
  k_combine<<<dim3((unsigned)((M + 255) / 256), NS), 256, 0, s>>>(w.OT, CAR, M, w.X);
  WTBG_COUNT(ctx, 1);
  CKL("mlp forward");
  return WTBG_OK;
}

// loss and gradients for nsamp samples of `rows` rows in the work buffers (Fin, FinT, CARb, Tt);
// gradients accumulate into net->G (cleared here), loss into net->loss[0].
int loss_backward(wtbg_net* net, Work& w, int nsamp, long long rows, float* loss_out) {
  wtbg_ctx* ctx = net->ctx;
  cudaStream_t s = ctx->stream;
  int* err = net->err.as<int>();
  const long long M = (long long)nsamp * rows;
  if (int r = forward(net, w, M, w.CARb)) return r;
  const float scale = 1.0f / ((float)NS * (float)nsamp);
  const int nchunk = (int)std::min<long long>(64, (rows + 255) / 256);
  k_cgram2<<<dim3(nchunk, nsamp), 256, 0, s>>>(w.Tt, w.X, M, (int)rows, nchunk, w.part);
  WTBG_COUNT(ctx, 1);
  k_cgram2_sum<<<dim3((2 * NS * NS + 255) / 256, nsamp), 256, 0, s>>>(w.part, nchunk, w.PG);
  WTBG_COUNT(ctx, 1);
  k_polar<<<nsamp, 1024, 0, s>>>(w.PG, 40);
  WTBG_COUNT(ctx, 1);
  float* dloss = net->loss.as<float>();
  CK(cudaMemsetAsync(dloss, 0, 4, s));
  k_loss<<<nsamp, 256, 0, s>>>(w.PG, nsamp, scale, dloss);
  WTBG_COUNT(ctx, 1);
  CK(cudaMemsetAsync(net->G.p, 0, (size_t)NPARAM * 4, s));
  k_dout<<<(unsigned)((M + 127) / 128), 128, 0, s>>>(w.Tt, w.X, w.PG, w.CARb, M, (int)rows, scale, w.dO, w.dOT,
                                                    gf(net, OFF_B3));
  WTBG_COUNT(ctx, 1);
  CKL("mlp loss");
  const dim3 tb(32, 8);
  // layer 3: dW3^T [WD][NO] = (dO^T H2)^T ; dH2 = dO W3
  if (int r = gemm_bf16(ctx, err, w.dOT, M, NO, (int)M, w.H2T, M, WD, gf(net, OFF_W3), NO, false)) return r;
  if (int r = gemm_bf16(ctx, err, w.dO, NO, (int)M, NO, bfp(net, BOFF_W3T), NO, WD, w.dH2T, M, true)) return r;
  k_silu_back<<<dim3((unsigned)((M + 31) / 32), WD / 32), tb, 0, s>>>(w.dH2T, w.Z2T, WD, M, w.dZ2, w.dZ2T,
                                                                      gf(net, OFF_B2));
  WTBG_COUNT(ctx, 1);
  // layer 2: dW2^T = (dZ2^T H1)^T ; dH1 = dZ2 W2
  if (int r = gemm_bf16(ctx, err, w.dZ2T, M, WD, (int)M, w.H1T, M, WD, gf(net, OFF_W2), WD, false)) return r;
  if (int r = gemm_bf16(ctx, err, w.dZ2, WD, (int)M, WD, bfp(net, BOFF_W2T), WD, WD, w.dH1T, M, true)) return r;
  k_silu_back<<<dim3((unsigned)((M + 31) / 32), WD / 32), tb, 0, s>>>(w.dH1T, w.Z1T, WD, M, nullptr, w.dZ1T,
                                                                      gf(net, OFF_B1));
  WTBG_COUNT(ctx, 1);
  // layer 1: dW1^T [NF][WD] = (dZ1^T Fin)^T
  if (int r = gemm_bf16(ctx, err, w.dZ1T, M, WD, (int)M, w.FinT, M, NF, gf(net, OFF_W1), WD, false)) return r;
  CKL("mlp backward");
  if (loss_out) {
    CK(cudaMemcpyAsync(loss_out, dloss, 4, cudaMemcpyDeviceToHost, s));
  }
  return WTBG_OK;
}

int refresh_bf16(wtbg_net* net) {
  wtbg_ctx* ctx = net->ctx;
  cudaStream_t s = ctx->stream;
  bf16* b = net->Wb.as<bf16>();
  const float* P = net->P.as<float>();
  k_to_bf16_pair<<<(WD * NF + 255) / 256, 256, 0, s>>>(P + OFF_W1, WD, NF, b + BOFF_W1, b + BOFF_W1T);
  k_to_bf16_pair<<<(WD * WD + 255) / 256, 256, 0, s>>>(P + OFF_W2, WD, WD, b + BOFF_W2, b + BOFF_W2T);
  k_to_bf16_pair<<<(NO * WD + 255) / 256, 256, 0, s>>>(P + OFF_W3, NO, WD, b + BOFF_W3, b + BOFF_W3T);
  WTBG_COUNT(ctx, 3);
  CKL("mlp bf16 weights");
  return WTBG_OK;
}

int adam_step(wtbg_net* net, float lr) {
  wtbg_ctx* ctx = net->ctx;
  cudaStream_t s = ctx->stream;
  net->step++;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, (float)net->step), c2 = 1.f - powf(b2, (float)net->step);
  float* P = net->P.as<float>();
  float* m1 = net->M1.as<float>();
  float* m2 = net->M2.as<float>();
  float* G = net->G.as<float>();
  bf16* b = net->Wb.as<bf16>();
  k_adam_w<<<(WD * NF + 255) / 256, 256, 0, s>>>(P + OFF_W1, m1 + OFF_W1, m2 + OFF_W1, G + OFF_W1, WD, NF, lr, b1, b2,
                                                 c1, c2, eps, b + BOFF_W1, b + BOFF_W1T);
  k_adam_w<<<(WD * WD + 255) / 256, 256, 0, s>>>(P + OFF_W2, m1 + OFF_W2, m2 + OFF_W2, G + OFF_W2, WD, WD, lr, b1, b2,
                                                 c1, c2, eps, b + BOFF_W2, b + BOFF_W2T);
  k_adam_w<<<(NO * WD + 255) / 256, 256, 0, s>>>(P + OFF_W3, m1 + OFF_W3, m2 + OFF_W3, G + OFF_W3, NO, WD, lr, b1, b2,
                                                 c1, c2, eps, b + BOFF_W3, b + BOFF_W3T);
  k_adam_b<<<(WD + 255) / 256, 256, 0, s>>>(P + OFF_B1, m1 + OFF_B1, m2 + OFF_B1, G + OFF_B1, WD, lr, b1, b2, c1, c2, eps);
  k_adam_b<<<(WD + 255) / 256, 256, 0, s>>>(P + OFF_B2, m1 + OFF_B2, m2 + OFF_B2, G + OFF_B2, WD, lr, b1, b2, c1, c2, eps);
  k_adam_b<<<(NO + 255) / 256, 256, 0, s>>>(P + OFF_B3, m1 + OFF_B3, m2 + OFF_B3, G + OFF_B3, NO, lr, b1, b2, c1, c2, eps);
  WTBG_COUNT(ctx, 6);
  CKL("mlp adam");
  return WTBG_OK;
}

int net_check(wtbg_net* net) {
  wtbg_ctx* ctx = net->ctx;
  int e = 0;
  CK(cudaMemcpyAsync(&e, net->err.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (e) {
    CK(cudaMemsetAsync(net->err.p, 0, 4, ctx->stream));
    return set_err(ctx, WTBG_ERR_CUDA, "tensor-core GEMM: a pipeline wait timed out");
  }
  return WTBG_OK;
}

// features + carriers of the current basis into F [rowoff..][NF] and CAR [c][M] columns rowoff..
int features_into(wtbg_ctx* ctx, const double* glob, bf16* F, float2* CAR, long long M, long long rowoff,
                  double* dmin_scratch) {
  if (!ctx->have_matrix) return set_err(ctx, WTBG_ERR_STATE, "learned warm start: call wtbg_bse_build first");
  if (!ctx->have_velocity) return set_err(ctx, WTBG_ERR_STATE, "learned warm start: call wtbg_velocity first");
  const long long N = ctx->N;
  k_dmin<<<1, 1024, 0, ctx->stream>>>(ctx->H.as<double2>(), N, dmin_scratch);
  WTBG_COUNT(ctx, 1);
  FeatArgs a;
  a.H = ctx->H.as<double2>();
  a.h = ctx->h.as<double2>();
  a.kpt = ctx->kpt.as<double>();
  a.dmin = dmin_scratch;
  a.N = N;
  a.nc = ctx->nc;
  a.nv = ctx->nv;
  for (int c = 0; c < 3; ++c) {
    a.a1[c] = ctx->rlat[c];
    a.a2[c] = ctx->rlat[3 + c];
    a.q[c] = glob[c];
  }
  a.r0 = glob[3];
  a.eps = glob[4];
  a.F = F;
  a.CAR = CAR;
  a.M = M;
  a.rowoff = rowoff;
  k_features<<<(unsigned)((N + 255) / 256), 256, 0, ctx->stream>>>(a);
  WTBG_COUNT(ctx, 1);
  CKL("k_features");
  return WTBG_OK;
}

}  // namespace

extern "C" {

int wtbg_net_create(wtbg_ctx* ctx, wtbg_net** out, unsigned long long seed) {
  if (!ctx || !out) return WTBG_ERR_ARG;
  if (int r = set_device(ctx)) return r;
  wtbg_net* net = new wtbg_net();
  net->ctx = ctx;
  net->seed = seed;
  auto fail = [&](int r) {
    wtbg_net_destroy(net);
    return r;
  };
  if (int r = ensure(ctx, net->P, (size_t)NPARAM * 4)) return fail(r);
  if (int r = ensure(ctx, net->M1, (size_t)NPARAM * 4)) return fail(r);
  if (int r = ensure(ctx, net->M2, (size_t)NPARAM * 4)) return fail(r);
  if (int r = ensure(ctx, net->G, (size_t)NPARAM * 4)) return fail(r);
  if (int r = ensure(ctx, net->Wb, (size_t)NBF * 2)) return fail(r);
  if (int r = ensure(ctx, net->err, 16)) return fail(r);
  if (int r = ensure(ctx, net->loss, 16)) return fail(r);
  if (int r = ensure(ctx, net->small, 4096)) return fail(r);
  // He-style init: W ~ N(0, 1/fan_in) (last layer scaled down), biases 0
  std::vector<float> p((size_t)NPARAM, 0.0f);
  std::mt19937_64 g(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (long long i = 0; i < (long long)WD * NF; ++i) p[OFF_W1 + i] = nd(g) * std::sqrt(2.0f / NF);
  for (long long i = 0; i < (long long)WD * WD; ++i) p[OFF_W2 + i] = nd(g) * std::sqrt(2.0f / WD);
  for (long long i = 0; i < (long long)NO * WD; ++i) p[OFF_W3 + i] = nd(g) * 0.1f * std::sqrt(1.0f / WD);
  cudaError_t e = cudaMemcpyAsync(net->P.p, p.data(), (size_t)NPARAM * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "net init"));
  cudaMemsetAsync(net->M1.p, 0, (size_t)NPARAM * 4, ctx->stream);
  cudaMemsetAsync(net->M2.p, 0, (size_t)NPARAM * 4, ctx->stream);
  cudaMemsetAsync(net->err.p, 0, 16, ctx->stream);
  if (int r = refresh_bf16(net)) return fail(r);
  *out = net;
  return WTBG_OK;
}

int wtbg_net_destroy(wtbg_net* net) {
  if (!net) return WTBG_OK;
  for (DevBuf* b : {&net->P, &net->M1, &net->M2, &net->G, &net->Wb, &net->F, &net->CAR, &net->T, &net->work, &net->err,
                    &net->loss, &net->small})
    if (b->p) cudaFree(b->p);
  delete net;
  return WTBG_OK;
}

long long wtbg_net_num_params(void) { return NPARAM; }

int wtbg_net_get_params(wtbg_net* net, float* p) {
  if (!net || !p) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = net->ctx;
  CK(cudaMemcpyAsync(p, net->P.p, (size_t)NPARAM * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return WTBG_OK;
}

int wtbg_net_set_params(wtbg_net* net, const float* p) {
  if (!net || !p) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = net->ctx;
  CK(cudaMemcpyAsync(net->P.p, p, (size_t)NPARAM * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(net->M1.p, 0, (size_t)NPARAM * 4, ctx->stream));
  CK(cudaMemsetAsync(net->M2.p, 0, (size_t)NPARAM * 4, ctx->stream));
  net->step = 0;
  if (int r = refresh_bf16(net)) return r;
  CK(cudaStreamSynchronize(ctx->stream));
  return WTBG_OK;
}

int wtbg_net_features(wtbg_net* net, const double* glob, float* F, float* CAR) {
  if (!net || !glob) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = net->ctx;
  const long long N = ctx->N;
  if (int r = ensure_work(net, N)) return r;
  Work w = carve(net->work.as<char>(), N);
  if (int r = features_into(ctx, glob, w.Fin, w.CARb, N, 0, net->small.as<double>())) return r;
  if (F) {
    std::vector<uint16_t> tmp((size_t)N * NF);
    CK(cudaMemcpyAsync(tmp.data(), w.Fin, tmp.size() * 2, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < tmp.size(); ++i) {
      const uint32_t u = (uint32_t)tmp[i] << 16;
      memcpy(&F[i], &u, 4);
    }
  }
  if (CAR) CK(cudaMemcpy(CAR, w.CARb, (size_t)N * NCAR * 8, cudaMemcpyDeviceToHost));
  return WTBG_OK;
}

int wtbg_net_add_sample(wtbg_net* net, const double* glob, const double* A) {
  if (!net || !glob || !A) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = net->ctx;
  const long long N = ctx->N;
  if (net->nsamp == 0) net->rows = N;
  if (N != net->rows) return set_err(ctx, WTBG_ERR_ARG, "net_add_sample: every sample must have the same basis size");
  if (net->nsamp == net->cap) {
    const int ncap = std::max(8, net->cap * 2);
    DevBuf F2, C2, T2;
    if (int r = ensure(ctx, F2, (size_t)ncap * N * NF * 2)) return r;
    if (int r = ensure(ctx, C2, (size_t)ncap * N * NCAR * 8)) return r;
    if (int r = ensure(ctx, T2, (size_t)ncap * N * NS * 8)) return r;
    if (net->nsamp) {
      const long long Mo = (long long)net->cap * N, Mn = (long long)ncap * N, used = (long long)net->nsamp * N;
      CK(cudaMemcpyAsync(F2.p, net->F.p, (size_t)used * NF * 2, cudaMemcpyDeviceToDevice, ctx->stream));
      for (int c = 0; c < NCAR; ++c)
        CK(cudaMemcpyAsync(C2.as<float2>() + c * Mn, net->CAR.as<float2>() + c * Mo, (size_t)used * 8,
                           cudaMemcpyDeviceToDevice, ctx->stream));
      for (int s = 0; s < NS; ++s)
        CK(cudaMemcpyAsync(T2.as<float2>() + s * Mn, net->T.as<float2>() + s * Mo, (size_t)used * 8,
                           cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
    }
    for (DevBuf* b : {&net->F, &net->CAR, &net->T})
      if (b->p) cudaFree(b->p);
    net->F = F2;
    net->CAR = C2;
    net->T = T2;
    net->cap = ncap;
  }
  const long long Mc = (long long)net->cap * N, off = (long long)net->nsamp * N;
  if (int r = features_into(ctx, glob, net->F.as<bf16>(), net->CAR.as<float2>(), Mc, off, net->small.as<double>()))
    return r;
  if (int r = ensure(ctx, ctx->tmp2, (size_t)N * NS * 16)) return r;
  CK(cudaMemcpyAsync(ctx->tmp2.p, A, (size_t)N * NS * 16, cudaMemcpyHostToDevice, ctx->stream));
  k_targets<<<dim3((unsigned)((N + 255) / 256), NS), 256, 0, ctx->stream>>>(ctx->tmp2.as<double2>(), N, Mc, off,
                                                                           net->T.as<float2>());
  WTBG_COUNT(ctx, 1);
  CKL("k_targets");
  CK(cudaStreamSynchronize(ctx->stream));
  net->nsamp++;
  return WTBG_OK;
}

// Stage samples [s0, s0+ns) of the store into the work buffers.
static int stage_batch(wtbg_net* net, Work& w, const int* idx, int ns) {
  wtbg_ctx* ctx = net->ctx;
  cudaStream_t s = ctx->stream;
  const long long N = net->rows, Mc = (long long)net->cap * N, M = (long long)ns * N;
  for (int j = 0; j < ns; ++j) {
    const long long src = (long long)idx[j] * N, dst = (long long)j * N;
    CK(cudaMemcpyAsync(w.Fin + dst * NF, net->F.as<bf16>() + src * NF, (size_t)N * NF * 2, cudaMemcpyDeviceToDevice, s));
    for (int c = 0; c < NCAR; ++c)
      CK(cudaMemcpyAsync(w.CARb + c * M + dst, net->CAR.as<float2>() + c * Mc + src, (size_t)N * 8,
                         cudaMemcpyDeviceToDevice, s));
    for (int t = 0; t < NS; ++t)
      CK(cudaMemcpyAsync(w.Tt + t * M + dst, net->T.as<float2>() + t * Mc + src, (size_t)N * 8,
                         cudaMemcpyDeviceToDevice, s));
  }
  k_transpose_bf16<<<dim3((unsigned)((M + 31) / 32), NF / 32), dim3(32, 8), 0, s>>>(w.Fin, NF, M, w.FinT);
  WTBG_COUNT(ctx, 1);
  CKL("stage batch");
  return WTBG_OK;
}

int wtbg_net_train(wtbg_net* net, int epochs, int batch, float lr, int first, int count, float* loss_hist) {
  if (!net || epochs < 1 || batch < 1 || !(lr > 0)) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = net->ctx;
  if (count <= 0) count = net->nsamp - first;
  if (first < 0 || first + count > net->nsamp || count < 1)
    return set_err(ctx, WTBG_ERR_ARG, "net_train: sample range outside the stored samples");
  batch = std::min(batch, count);
  const long long N = net->rows;
  if (int r = ensure_work(net, (long long)batch * N)) return r;
  Work w = carve(net->work.as<char>(), (long long)batch * N);
  std::mt19937_64 g(net->seed + 7919ull * (unsigned long long)net->step);
  std::vector<int> order(count);
  Timer t(ctx);
  for (int ep = 0; ep < epochs; ++ep) {
    for (int i = 0; i < count; ++i) order[i] = first + i;
    std::shuffle(order.begin(), order.end(), g);
    double ls = 0.0;
    int nb = 0;
    for (int b0 = 0; b0 + batch <= count; b0 += batch) {
      if (int r = stage_batch(net, w, order.data() + b0, batch)) return r;
      float lossv = 0.f;
      if (int r = loss_backward(net, w, batch, N, &lossv)) return r;
      if (int r = adam_step(net, lr)) return r;
      CK(cudaStreamSynchronize(ctx->stream));
      ls += lossv;
      ++nb;
    }
    if (loss_hist) loss_hist[ep] = (float)(ls / std::max(1, nb));
  }
  if (int r = t.stop()) return r;
  return net_check(net);
}

int wtbg_net_eval_loss(wtbg_net* net, int first, int count, float* loss) {
  if (!net || !loss) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = net->ctx;
  if (first < 0 || count < 1 || first + count > net->nsamp) return set_err(ctx, WTBG_ERR_ARG, "net_eval_loss: bad range");
  const long long N = net->rows;
  if (int r = ensure_work(net, N)) return r;
  Work w = carve(net->work.as<char>(), N);
  double ls = 0.0;
  for (int i = first; i < first + count; ++i) {
    if (int r = stage_batch(net, w, &i, 1)) return r;
    float lv = 0.f;
    if (int r = loss_backward(net, w, 1, N, &lv)) return r;
    CK(cudaStreamSynchronize(ctx->stream));
    ls += lv;
  }
  *loss = (float)(ls / count);
  return net_check(net);
}

int wtbg_net_predict(wtbg_net* net, const double* glob, double* X0) {
  if (!net || !glob || !X0) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = net->ctx;
  const long long N = ctx->N;
  if (int r = ensure_work(net, N)) return r;
  Work w = carve(net->work.as<char>(), N);
  Timer t(ctx);
  if (int r = features_into(ctx, glob, w.Fin, w.CARb, N, 0, net->small.as<double>())) return r;
  if (int r = forward(net, w, N, w.CARb)) return r;
  std::vector<float2> x((size_t)N * NS);
  CK(cudaMemcpyAsync(x.data(), w.X, x.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (int r = t.stop()) return r;
  if (int r = net_check(net)) return r;
  for (long long s = 0; s < NS; ++s)
    for (long long i = 0; i < N; ++i) {
      X0[2 * (i + s * N)] = x[s * N + i].x;
      X0[2 * (i + s * N) + 1] = x[s * N + i].y;
    }
  return WTBG_OK;
}

// One forward + backward on explicit inputs (gradient check): F (nsamp*rows x NF, fp32, rounded
// to bf16 here), CAR (NCAR x M complex float), A (NS x M complex float, per sample orthonormal).
int wtbg_net_loss_grad(wtbg_net* net, int nsamp, long long rows, const float* F, const float* CAR, const float* A,
                       float* loss, float* grad) {
  if (!net || nsamp < 1 || rows < 1 || !F || !CAR || !A || !loss || !grad) return WTBG_ERR_ARG;
  wtbg_ctx* ctx = net->ctx;
  const long long M = (long long)nsamp * rows;
  if (int r = ensure_work(net, M)) return r;
  Work w = carve(net->work.as<char>(), M);
  std::vector<bf16> fb((size_t)M * NF);
  for (size_t i = 0; i < fb.size(); ++i) fb[i] = __float2bfloat16(F[i]);
  CK(cudaMemcpyAsync(w.Fin, fb.data(), fb.size() * 2, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(w.CARb, CAR, (size_t)M * NCAR * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(w.Tt, A, (size_t)M * NS * 8, cudaMemcpyHostToDevice, ctx->stream));
  k_transpose_bf16<<<dim3((unsigned)((M + 31) / 32), NF / 32), dim3(32, 8), 0, ctx->stream>>>(w.Fin, NF, M, w.FinT);
  WTBG_COUNT(ctx, 1);
  if (int r = loss_backward(net, w, nsamp, rows, loss)) return r;
  std::vector<float> g((size_t)NPARAM);
  CK(cudaMemcpyAsync(g.data(), net->G.p, (size_t)NPARAM * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  // weight gradients are accumulated transposed ([in][out]); return them as [out][in]
  memcpy(grad, g.data(), (size_t)NPARAM * 4);
  const long long offs[3] = {OFF_W1, OFF_W2, OFF_W3};
  const int outs[3] = {WD, WD, NO}, ins[3] = {NF, WD, WD};
  for (int l = 0; l < 3; ++l)
    for (int o = 0; o < outs[l]; ++o)
      for (int k = 0; k < ins[l]; ++k) grad[offs[l] + (long long)o * ins[l] + k] = g[offs[l] + (long long)k * outs[l] + o];
  return net_check(net);
}

int wtbg_net_num_samples(wtbg_net* net) { return net ? net->nsamp : 0; }

int wtbg_gemm_bf16(wtbg_ctx* ctx, int M, int N, int K, const float* A, const float* B, float* C) {
  if (!ctx || !A || !B || !C || M < 1 || N < 1 || K < 1) return WTBG_ERR_ARG;
  if (K % 8) return set_err(ctx, WTBG_ERR_ARG, "gemm_bf16: K must be a multiple of 8");
  if (int r = set_device(ctx)) return r;
  std::vector<bf16> ab((size_t)M * K), bb((size_t)N * K);
  for (size_t i = 0; i < ab.size(); ++i) ab[i] = __float2bfloat16(A[i]);
  for (size_t i = 0; i < bb.size(); ++i) bb[i] = __float2bfloat16(B[i]);
  const size_t need = ab.size() * 2 + bb.size() * 2 + (size_t)M * N * 4 + 4096;
  ENSURE(ctx->tmp2, need);
  char* p = ctx->tmp2.as<char>();
  bf16* dA = reinterpret_cast<bf16*>(p);
  bf16* dB = reinterpret_cast<bf16*>(p + (ab.size() * 2 + 255) / 256 * 256);
  float* dC = reinterpret_cast<float*>(p + (ab.size() * 2 + 255) / 256 * 256 + (bb.size() * 2 + 255) / 256 * 256);
  ENSURE(ctx->istat, 64);
  int* err = ctx->istat.as<int>();
  CK(cudaMemsetAsync(err, 0, 4, ctx->stream));
  CK(cudaMemcpyAsync(dA, ab.data(), ab.size() * 2, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dB, bb.data(), bb.size() * 2, cudaMemcpyHostToDevice, ctx->stream));
  Timer t(ctx);
  if (int r = gemm_bf16(ctx, err, dA, K, M, K, dB, K, N, dC, M, true)) return r;
  if (int r = t.stop()) return r;
  std::vector<float> ct((size_t)M * N);
  int e = 0;
  CK(cudaMemcpy(ct.data(), dC, ct.size() * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&e, err, 4, cudaMemcpyDeviceToHost));
  if (e) return set_err(ctx, WTBG_ERR_CUDA, "tensor-core GEMM: a pipeline wait timed out");
  for (int m = 0; m < M; ++m)
    for (int n = 0; n < N; ++n) C[(size_t)m * N + n] = ct[(size_t)n * M + m];
  return WTBG_OK;
}

}  // extern "C"
