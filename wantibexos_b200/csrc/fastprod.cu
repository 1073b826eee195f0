// Split-BF16 tensor-core product Y = H X with the exciton Hamiltonian (fast form).
//
// The off-diagonal part of H (diagonal removed) is stored once per kernel build as four
// row-major bf16 planes: Re H hi, Re H lo, Im H hi, Im H lo, with hi = bf16(x) and
// lo = bf16(x - hi), so hi + lo carries ~16 mantissa bits. X (complex, m columns) is split
// the same way into B planes [hi|lo][Re X (mp rows) | Im X (mp rows)][N], mp = m rounded up to
// 16. The real form of the complex product,
//     [Yr | Yi] = Re H [Xr | Xi] + Im H [-Xi | Xr],
// runs on tcgen05 (kind::f16, bf16 inputs, FP32 accumulation in TMEM) with three products
// per pair (hi*hi + hi*lo + lo*hi). The diagonal D (the band-energy differences, which
// dominate |H|) is applied in FP64 in the epilogue kernel, so the split error only scales
// with the much smaller interaction part.
//
// Kernel shape: persistent stream-K grid over (128-row tile, 32-wide K block) units; warp 0
// issues TMA loads (64-byte swizzle) into a 4-stage mbarrier ring, warp 1 issues the MMAs
// into one of two TMEM accumulators in chunks of FP_CHUNK K blocks, warps 2..5 drain each
// finished chunk (tcgen05.ld) into FP64 registers and, at the end of a row tile's K range, add
// the FP64 sums to global memory with red.add.f64 (short FP32 chains keep the product's
// rounding near the bf16-split level). Every mbarrier wait is bounded in time; on
// expiry the CTA raises an error flag, drains its copies and MMAs, frees TMEM and returns.
#include "common.cuh"

#include <algorithm>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include "tc_sm100.cuh"

namespace {

using namespace tc;

constexpr int FP_BM = 128;          // rows per tile = TMEM lanes
constexpr int FP_BK = 32;           // K per stage: 64-byte bf16 rows
constexpr int FP_STAGES = 4;
constexpr int FP_MAXMP = 48;        // padded vectors per half (2*mp FP64 sums per epilogue thread)
constexpr int FP_CHUNK = 8;         // K blocks per FP32 TMEM accumulation before the FP64 drain
constexpr int FP_THREADS = 192;
constexpr uint32_t FP_TMEM_COLS = 256;   // two accumulators of 128 columns
constexpr uint32_t FP_A_BYTES = 4u * FP_BM * FP_BK * 2u;

struct FastArgs {
  int N, m, mp, KB;
  long long W;       // units = tiles * KB
  double* Yacc;      // [2*mp][N]
  int* err;
};

template <int MP>
__global__ void __launch_bounds__(FP_THREADS, 1)
    k_fastprod(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, FastArgs a) {
  extern __shared__ unsigned char fp_smem[];
  __shared__ __align__(8) uint64_t bars[2 * FP_STAGES + 5];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t raw = smem_u32(fp_smem);
  const uint32_t base = (raw + 1023u) & ~1023u;
  constexpr int mp = MP;
  const uint32_t B_BYTES = 2u * 2u * (uint32_t)mp * FP_BK * 2u;
  const uint32_t STAGE = FP_A_BYTES + B_BYTES;
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[FP_STAGES]);
  const uint32_t accf0 = smem_u32(&bars[2 * FP_STAGES]), acce0 = smem_u32(&bars[2 * FP_STAGES + 2]);
  const uint32_t done = smem_u32(&bars[2 * FP_STAGES + 4]);
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int i = 0; i < FP_STAGES; ++i) {
      mbar_init(full0 + 8 * i, 1);
      mbar_init(empty0 + 8 * i, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, 4);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(FP_TMEM_COLS)
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
  const int KB = a.KB;

  if (warp == 0 && lane == 0) {
    // TMA producer
    long long it = 0;
    for (long long u = u0; u < u1; ++u, ++it) {
      const int s = (int)(it % FP_STAGES);
      const long long r = it / FP_STAGES;
      if (r > 0 && !mbar_wait(empty0 + 8 * s, (uint32_t)((r - 1) & 1), abort_flag)) break;
      const int mt = (int)(u / KB), kb = (int)(u % KB);
      const uint32_t sa = base + (uint32_t)s * STAGE;
      mbar_expect_tx(full0 + 8 * s, STAGE);
      tma_load_3d(sa, &tmA, kb * FP_BK, mt * FP_BM, 0, full0 + 8 * s);
      tma_load_3d(sa + FP_A_BYTES, &tmB, kb * FP_BK, 0, 0, full0 + 8 * s);
    }
    // copies in flight: wait (bounded) for the last fill of each stage that was used
    for (int s = 0; s < FP_STAGES && s < it; ++s) {
      const long long last = (it - 1 - s) / FP_STAGES;   // fills of stage s: indices s, s+S, ...
      mbar_wait(full0 + 8 * s, (uint32_t)(last & 1), abort_flag, false);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: each segment (one row tile) is accumulated in chunks of at most FP_CHUNK
    // K blocks, alternating between the two TMEM accumulators
    const uint32_t idf = idesc_bf16(FP_BM, 2 * mp, false), idh = idesc_bf16(FP_BM, mp, false),
                   idn = idesc_bf16(FP_BM, mp, true);
    long long it = 0, u = u0;
    int chunk = 0;
    bool ok = true;
    while (u < u1 && ok) {
      const long long seg_end = min(u1, (u / KB + 1) * KB);
      while (u < seg_end && ok) {
        const long long cend = min(seg_end, u + FP_CHUNK);
        const int b = chunk & 1;
        if (chunk >= 2 && !mbar_wait(acce0 + 8 * b, (uint32_t)(((chunk - 2) >> 1) & 1), abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t dt = tmem + (uint32_t)b * 128u;
        uint32_t acc = 0;
        for (; u < cend; ++u, ++it) {
          const int s = (int)(it % FP_STAGES);
          const long long r = it / FP_STAGES;
          if (!mbar_wait(full0 + 8 * s, (uint32_t)(r & 1), abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = base + (uint32_t)s * STAGE, sb = sa + FP_A_BYTES;
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) {
            const uint32_t ko = (uint32_t)kk * 32u;
            const uint64_t arh = sdesc(sa + ko), arl = sdesc(sa + 8192u + ko);
            const uint64_t aih = sdesc(sa + 16384u + ko), ail = sdesc(sa + 24576u + ko);
            const uint32_t bh = sb + ko, bl = sb + (uint32_t)(2 * mp) * 64u + ko;
            const uint64_t bhf = sdesc(bh), blf = sdesc(bl);
            const uint64_t bhi = sdesc(bh + (uint32_t)mp * 64u), bli = sdesc(bl + (uint32_t)mp * 64u);
            tc_mma(dt, arh, bhf, idf, acc);
            acc = 1;
            tc_mma(dt, arh, blf, idf, 1);
            tc_mma(dt, arl, bhf, idf, 1);
            tc_mma(dt, aih, bhi, idn, 1);              // Yr -= Im H Xi
            tc_mma(dt, aih, bli, idn, 1);
            tc_mma(dt, ail, bhi, idn, 1);
            tc_mma(dt + (uint32_t)mp, aih, bhf, idh, 1);   // Yi += Im H Xr
            tc_mma(dt + (uint32_t)mp, aih, blf, idh, 1);
            tc_mma(dt + (uint32_t)mp, ail, bhf, idh, 1);
          }
          tc_commit(empty0 + 8 * s);
        }
        if (!ok) break;
        tc_commit(accf0 + 8 * b);
        ++chunk;
      }
    }
    // all MMAs issued by this thread complete before TMEM is released
    tc_commit(done);
    mbar_wait(done, 0, abort_flag, false);
  } else if (warp >= 2) {
    // epilogue: TMEM lane quarter q belongs to warps with warp % 4 == q. Every chunk's FP32
    // partial is added into FP64 registers (one row, 2*mp columns per thread); at the end of
    // a segment the FP64 sums go to global memory with red.add.f64.
    const int q = warp & 3;
    long long u = u0;
    int chunk = 0;
    const int N = a.N, m = a.m;
    double accd[2 * MP];
#pragma unroll
    for (int j = 0; j < 2 * MP; ++j) accd[j] = 0.0;
    bool ok = true;
    while (u < u1 && ok) {
      const long long seg_end = min(u1, (u / KB + 1) * KB);
      const int mt = (int)(u / KB);
      const int row = mt * FP_BM + q * 32 + lane;
      while (u < seg_end) {
        const long long cend = min(seg_end, u + FP_CHUNK);
        const int b = chunk & 1;
        if (!mbar_wait(accf0 + 8 * b, (uint32_t)((chunk >> 1) & 1), abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)b * 128u;
#pragma unroll
        for (int c0 = 0; c0 < 2 * MP; c0 += 32) {
          uint32_t v[32];
          tc_ld16(ta + (uint32_t)c0, v);
          if (c0 + 16 < 2 * MP) tc_ld16(ta + (uint32_t)c0 + 16u, v + 16);
          tc_wait_ld();
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (c0 + j < 2 * MP) accd[c0 + j] += (double)__uint_as_float(v[j]);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acce0 + 8 * b);
        u = cend;
        ++chunk;
      }
      if (!ok) break;
      if (row < N) {
#pragma unroll
        for (int j = 0; j < 2 * MP; ++j)
          if ((j % MP) < m) atomicAdd(a.Yacc + (long long)j * N + row, accd[j]);
      }
#pragma unroll
      for (int j = 0; j < 2 * MP; ++j) accd[j] = 0.0;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(FP_TMEM_COLS) : "memory");
  }
  if (threadIdx.x == 0 && s_abort) atomicExch(a.err, 1);
}

__device__ __forceinline__ void split2(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __double2bfloat16(x);
  lo = __double2bfloat16(x - (double)__bfloat162float(hi));
}

// Row-major split planes of the off-diagonal part of H from its lower column-major FP64
// storage, and the FP64 diagonal. 32x32 tile pairs (ti >= tj), block (32, 8).
__global__ void k_split_h(const double2* __restrict__ H, long long N, long long ld, __nv_bfloat16* __restrict__ P,
                          double* __restrict__ D) {
  const int ti = blockIdx.x, tj = blockIdx.y;
  if (tj > ti) return;
  __shared__ double2 t[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const long long r0 = (long long)ti * 32, c0 = (long long)tj * 32;
  for (int c = ty; c < 32; c += 8) {
    const long long row = r0 + tx, col = c0 + c;
    double2 v = make_double2(0.0, 0.0);
    if (row < N && col < N && (ti > tj || tx >= c)) v = H[row + col * N];
    if (ti == tj && tx == c) {
      if (row < N) D[row] = v.x;
      v = make_double2(0.0, 0.0);
    }
    t[c][tx] = v;
  }
  __syncthreads();
  const long long plane = N * ld;
  // the tile itself: (row, col) = H[row][col], coalesced along col
  for (int r = ty; r < 32; r += 8) {
    const long long row = r0 + r, col = c0 + tx;
    if (row >= N || col >= N) continue;
    if (ti == tj && tx > r) continue;   // upper part of a diagonal tile comes from the mirror
    const double2 v = t[tx][r];
    __nv_bfloat16 h, l;
    const long long o = row * ld + col;
    split2(v.x, h, l);
    P[o] = h;
    P[plane + o] = l;
    split2(v.y, h, l);
    P[2 * plane + o] = h;
    P[3 * plane + o] = l;
  }
  if (ti == tj) {
    // mirror within the diagonal tile: (c, r) for r > c
    for (int c = ty; c < 32; c += 8) {
      const long long row = c0 + c, col = r0 + tx;   // H[c][r] = conj(H[r][c]) for r = tx > c
      if (row >= N || col >= N || tx <= c) continue;
      const double2 v = t[c][tx];
      __nv_bfloat16 h, l;
      const long long o = row * ld + col;
      split2(v.x, h, l);
      P[o] = h;
      P[plane + o] = l;
      split2(-v.y, h, l);
      P[2 * plane + o] = h;
      P[3 * plane + o] = l;
    }
    return;
  }
  // mirror tile: (col, row) = conj(H[row][col]), coalesced along row
  for (int c = ty; c < 32; c += 8) {
    const long long row = c0 + c, col = r0 + tx;
    if (row >= N || col >= N) continue;
    const double2 v = t[c][tx];
    __nv_bfloat16 h, l;
    const long long o = row * ld + col;
    split2(v.x, h, l);
    P[o] = h;
    P[plane + o] = l;
    split2(-v.y, h, l);
    P[2 * plane + o] = h;
    P[3 * plane + o] = l;
  }
}

// B planes [hi|lo][2*mp][ld] from X (N x m complex, leading dimension ldx)
__global__ void k_split_x(const double2* __restrict__ X, int ldx, int m, int mp, long long N, long long ld,
                          __nv_bfloat16* __restrict__ B) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;   // 0 .. 2*mp-1
  if (k >= N) return;
  const int v = j % mp;
  double x = 0.0;
  if (v < m) {
    const double2 z = X[k + (long long)v * ldx];
    x = (j < mp) ? z.x : z.y;
  }
  __nv_bfloat16 h, l;
  split2(x, h, l);
  B[(long long)j * ld + k] = h;
  B[(long long)(2 * mp + j) * ld + k] = l;
}

// Y = Yacc + D X (FP64), and clear Yacc for the next product
__global__ void k_fast_finish(double* __restrict__ Yacc, const double* __restrict__ D, const double2* __restrict__ X,
                              int ldx, int m, int mp, long long N, double2* __restrict__ Y, int ldy) {
  const long long row = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (row >= N || j >= m) return;
  double* pr = Yacc + (long long)j * N + row;
  double* pi = Yacc + (long long)(mp + j) * N + row;
  const double2 x = X[row + (long long)j * ldx];
  const double d = D[row];
  Y[row + (long long)j * ldy] = make_double2(*pr + d * x.x, *pi + d * x.y);
  *pr = 0.0;
  *pi = 0.0;
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

int encode_3d(wtbg_ctx* ctx, CUtensorMap* map, void* ptr, unsigned long long d0, unsigned long long d1,
              unsigned long long d2, unsigned long long s1_bytes, unsigned long long s2_bytes, unsigned b0, unsigned b1,
              unsigned b2) {
  auto fn = encode_fn();
  if (!fn) return set_err(ctx, WTBG_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {s1_bytes, s2_bytes};
  cuuint32_t box[3] = {b0, b1, b2};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, ptr, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_err(ctx, WTBG_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return WTBG_OK;
}

}  // namespace

// Build the split planes of the current kernel matrix (once per build).
int run_fast_setup(wtbg_ctx* ctx) {
  if (ctx->fast_ready) return WTBG_OK;
  if (!ctx->have_matrix) return set_err(ctx, WTBG_ERR_STATE, "no BSE matrix: call wtbg_bse_build first");
  const long long N = ctx->N;
  const long long ld = (N + 63) / 64 * 64;
  if (int r = ensure(ctx, ctx->fA, (size_t)4 * N * ld * 2)) return r;
  if (int r = ensure(ctx, ctx->fB, (size_t)4 * FP_MAXMP * ld * 2)) return r;
  if (int r = ensure(ctx, ctx->fY, (size_t)2 * FP_MAXMP * N * 8)) return r;
  if (int r = ensure(ctx, ctx->fD, (size_t)N * 8)) return r;
  if (int r = ensure(ctx, ctx->fErr, 16)) return r;
  CK(cudaMemsetAsync(ctx->fY.p, 0, (size_t)2 * FP_MAXMP * N * 8, ctx->stream));
  CK(cudaMemsetAsync(ctx->fErr.p, 0, 16, ctx->stream));
  const int nt = (int)((N + 31) / 32);
  k_split_h<<<dim3(nt, nt), dim3(32, 8), 0, ctx->stream>>>(ctx->H.as<double2>(), N, ld, ctx->fA.as<__nv_bfloat16>(),
                                                           ctx->fD.as<double>());
  WTBG_COUNT(ctx, 1);
  CKL("k_split_h");
  if (int r = encode_3d(ctx, reinterpret_cast<CUtensorMap*>(ctx->tmA), ctx->fA.p, N, N, 4, ld * 2, ld * N * 2, FP_BK,
                        FP_BM, 4))
    return r;
  ctx->fast_ld = ld;
  ctx->fast_mp = 0;
  ctx->fast_ready = true;
  return WTBG_OK;
}

// Y (N x m, ldy) = H X (N x m, ldx) through the split-BF16 tensor-core product, m <= 64 per pass.
int run_fastprod(wtbg_ctx* ctx, const double2* X, int ldx, int m, double2* Y, int ldy) {
  if (int r = run_fast_setup(ctx)) return r;
  const long long N = ctx->N, ld = ctx->fast_ld;
  cudaStream_t s = ctx->stream;
  static bool attr_done[64] = {false};
  for (int j0 = 0; j0 < m; j0 += FP_MAXMP) {
    const int mm = std::min(FP_MAXMP, m - j0);
    const int mp = (mm + 15) / 16 * 16;
    if (ctx->fast_mp != mp) {
      if (int r = encode_3d(ctx, reinterpret_cast<CUtensorMap*>(ctx->tmB), ctx->fB.p, N, 2 * mp, 2, ld * 2,
                            (unsigned long long)ld * 2 * mp * 2, FP_BK, 2 * mp, 2))
        return r;
      ctx->fast_mp = mp;
    }
    k_split_x<<<dim3((unsigned)((N + 255) / 256), 2 * mp), 256, 0, s>>>(X + (long long)j0 * ldx, ldx, mm, mp, N, ld,
                                                                       ctx->fB.as<__nv_bfloat16>());
    WTBG_COUNT(ctx, 1);
    CKL("k_split_x");
    FastArgs a;
    a.N = (int)N;
    a.m = mm;
    a.mp = mp;
    a.KB = (int)((N + FP_BK - 1) / FP_BK);
    const long long tiles = (N + FP_BM - 1) / FP_BM;
    a.W = tiles * a.KB;
    a.Yacc = ctx->fY.as<double>();
    a.err = ctx->fErr.as<int>();
    const size_t smem = (size_t)FP_STAGES * (FP_A_BYTES + 2u * 2u * mp * FP_BK * 2u) + 1024;
    int dev = 0, nsm = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int maxsm = (int)(FP_STAGES * (FP_A_BYTES + 2u * 2u * FP_MAXMP * FP_BK * 2u) + 1024);
    if (!attr_done[dev & 63]) {
      CK(cudaFuncSetAttribute(k_fastprod<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
      CK(cudaFuncSetAttribute(k_fastprod<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
      CK(cudaFuncSetAttribute(k_fastprod<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm));
      attr_done[dev & 63] = true;
    }
    const int grid = (int)std::min<long long>(nsm, a.W);
    const bool prof = ctx->profiling != 0;
    if (prof) {
      if (int r = ensure_events(ctx, 2)) return r;
      cudaEventRecord(ctx->evpool[0], s);
    }
    const CUtensorMap& ma = *reinterpret_cast<const CUtensorMap*>(ctx->tmA);
    const CUtensorMap& mb = *reinterpret_cast<const CUtensorMap*>(ctx->tmB);
    if (mp == 16)
      k_fastprod<16><<<grid, FP_THREADS, smem, s>>>(ma, mb, a);
    else if (mp == 32)
      k_fastprod<32><<<grid, FP_THREADS, smem, s>>>(ma, mb, a);
    else
      k_fastprod<48><<<grid, FP_THREADS, smem, s>>>(ma, mb, a);
    WTBG_COUNT(ctx, 1);
    CKL("k_fastprod");
    if (prof) {
      cudaEventRecord(ctx->evpool[1], s);
      CK(cudaEventSynchronize(ctx->evpool[1]));
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ctx->evpool[0], ctx->evpool[1]));
      ctx->stats.fast_ms += t;
      ctx->stats.fast_bytes += 8.0 * (double)N * (double)N;
      ctx->stats.fast_launches += 1;
    }
    k_fast_finish<<<dim3((unsigned)((N + 255) / 256), mm), 256, 0, s>>>(ctx->fY.as<double>(), ctx->fD.as<double>(),
                                                                       X + (long long)j0 * ldx, ldx, mm, mp, N,
                                                                       Y + (long long)j0 * ldy, ldy);
    WTBG_COUNT(ctx, 1);
    CKL("k_fast_finish");
  }
  return WTBG_OK;
}

// Error flag of the product kernel (a bounded wait expired); clears it.
int fast_check(wtbg_ctx* ctx) {
  if (!ctx->fast_ready) return WTBG_OK;
  int e = 0;
  CK(cudaMemcpyAsync(&e, ctx->fErr.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (e) {
    CK(cudaMemsetAsync(ctx->fErr.p, 0, 16, ctx->stream));
    return set_err(ctx, WTBG_ERR_CUDA, "tensor-core product: a pipeline wait timed out");
  }
  return WTBG_OK;
}
