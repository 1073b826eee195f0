// Kernel (c), stage 1: blocked Householder reduction of the Hermitian BSE matrix to real
// symmetric tridiagonal form, T = Q^H H Q, in FP64.
//
// Reference: the dense ZHEEV('V','U') call of bsesolver (subprograms/bse_solver-tool-diel.f90:
// 485-492) and ZHEEV('N','U') of bsebnds (bse_kpath-tool.f90:384-387).  The reference links
// MKL's ZHEEV; this file is our own GPU formulation of the standard LAPACK algorithm
// (ZHETRD lower with the ZLATRD panel and ZLARFG reflectors):
//   for each panel of WTBG_PANEL columns, each column i is
//     (1) updated with the panel's pending rank-2 terms      A(i:n,i) -= V W(i,:)^H + W V(i,:)^H
//     (2) reduced by a reflector H_i = I - tau v v^H          (beta real, v(i+1) = 1)
//     (3) used in the Hermitian matrix-vector product y = A22 v (tiled over the lower triangle)
//     (4) w = tau (y - V (W^H v) - W (V^H v)),  w += -tau/2 (w^H v) v
//   and after the panel the trailing matrix gets A22 -= V W^H + W V^H on FP64 tensor cores
//   (mma.sync m16n8k4 f64; Blackwell has no tcgen05 kind for f64).
// The oscillator sums need only A^T h = Z^T (Q^T h) (Z = eigenvectors of T), so the
// reflectors are also applied to the five h vectors as they are generated,
// g <- g - tau conj(v) (v^T g) -- the full O(N^3) eigenvector back-transform is never formed.
// All reductions are deterministic two-pass (no atomics).
#include <cfloat>

#include "common.cuh"

namespace {

constexpr int TB = WTBG_HEMV_TILE;   // 64
constexpr int NB = WTBG_PANEL;       // 32
constexpr int RB = 256;              // rows per block of the column kernels
constexpr int NG = 5;                // h vectors carried through (x, y, z, sp, sm)

struct ColScal {
  double2 tau;
  double2 scal;
  double2 alpha2;
  double beta;
  int trivial;
};

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// (1) column update + partial |x|^2 for rows >= i+2
__global__ void __launch_bounds__(RB) k_colupd(double2* A, long long N, const double2* Wp, int j0, int p, int i,
                                               double* part) {
  __shared__ double2 wrow[NB], vrow[NB];
  __shared__ double red[RB / 32];
  const int tid = threadIdx.x;
  if (tid < p) {
    wrow[tid] = Wp[i + (long long)tid * N];
    vrow[tid] = A[i + (long long)(j0 + tid) * N];
  }
  __syncthreads();
  const long long r = (long long)i + (long long)blockIdx.x * RB + tid;
  double nrm = 0.0;
  if (r < N) {
    double2 a = A[r + (long long)i * N];
    if (p > 0) {
      double2 s1 = make_double2(0, 0), s2 = make_double2(0, 0);
      for (int q = 0; q < p; ++q) {
        const double2 vq = A[r + (long long)(j0 + q) * N];
        const double2 wq = Wp[r + (long long)q * N];
        s1 = cadd(s1, cmul(vq, cconj(wrow[q])));
        s2 = cadd(s2, cmul(wq, cconj(vrow[q])));
      }
      a = csub(csub(a, s1), s2);
    }
    if (r == i) a.y = 0.0;
    A[r + (long long)i * N] = a;
    if (r >= (long long)i + 2) nrm = a.x * a.x + a.y * a.y;
  }
  nrm = warp_sum(nrm);
  if ((tid & 31) == 0) red[tid >> 5] = nrm;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int k = 0; k < RB / 32; ++k) s += red[k];
    part[blockIdx.x] = s;
  }
}

// (2) reflector scalars (ZLARFG)
__global__ void k_reflector(const double2* A, long long N, int i, const double* part, int nparts, double* d,
                            double* e, double2* tau_out, ColScal* sc) {
  __shared__ double red[32];
  const int tid = threadIdx.x;
  double s = 0.0;
  for (int k = tid; k < nparts; k += blockDim.x) s += part[k];
  s = warp_sum(s);
  if ((tid & 31) == 0) red[tid >> 5] = s;
  __syncthreads();
  if (tid == 0) {
    double xn2 = 0.0;
    for (int k = 0; k < (int)(blockDim.x / 32); ++k) xn2 += red[k];
    const double2 alpha = A[(i + 1) + (long long)i * N];
    ColScal c;
    c.alpha2 = make_double2(0, 0);
    if (xn2 == 0.0 && alpha.y == 0.0) {
      c.tau = make_double2(0, 0);
      c.scal = make_double2(0, 0);
      c.beta = alpha.x;
      c.trivial = 1;
    } else {
      const double beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x);
      c.tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
      // scal = 1 / (alpha - beta)
      const double2 den = make_double2(alpha.x - beta, alpha.y);
      const double dd = den.x * den.x + den.y * den.y;
      c.scal = make_double2(den.x / dd, -den.y / dd);
      c.beta = beta;
      c.trivial = 0;
    }
    *sc = c;
    e[i] = c.beta;
    d[i] = A[i + (long long)i * N].x;
    tau_out[i] = c.tau;
  }
}

// (2b) scale v in place, v(i+1)=1; partial dots z1 = W^H v, z2 = V^H v, s = v^T g
__global__ void __launch_bounds__(RB) k_scale_dots(double2* A, long long N, const double2* Wp, int j0, int p, int i,
                                                   const ColScal* sc, const double2* g, double2* part) {
  __shared__ double2 red[RB / 32][2 * NB + NG];
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const long long r = (long long)i + 1 + (long long)blockIdx.x * RB + tid;
  const ColScal c = *sc;
  double2 v = make_double2(0, 0);
  if (r < N) {
    if (r == i + 1) v = make_double2(1.0, 0.0);
    else v = c.trivial ? make_double2(0, 0) : cmul(A[r + (long long)i * N], c.scal);
    A[r + (long long)i * N] = v;
  }
  const int nval = 2 * p + NG;
  for (int q = 0; q < nval; ++q) {
    double2 t = make_double2(0, 0);
    if (r < N) {
      if (q < p) t = cmulc(Wp[r + (long long)q * N], v);
      else if (q < 2 * p) t = cmulc(A[r + (long long)(j0 + q - p) * N], v);
      else t = cmul(v, g[(long long)(q - 2 * p) * N + r]);
    }
    t = warp_sum2(t);
    if (lane == 0) red[wp][q] = t;
  }
  __syncthreads();
  for (int q = tid; q < nval; q += RB) {
    double2 s = make_double2(0, 0);
    for (int k = 0; k < RB / 32; ++k) s = cadd(s, red[k][q]);
    part[(long long)blockIdx.x * (2 * NB + NG) + q] = s;
  }
}

// (3) y = A22 v over the lower-triangular 64x64 tiles of rows/cols [i+1, N).
// Tile (I, J), I >= J: slot[I][J] += A_IJ x_J (for y_I); slot[J][I] = A_IJ^H x_I (for y_J).
__global__ void __launch_bounds__(256) k_hemv(const double2* __restrict__ A, long long N, int i, int nblk,
                                              double2* __restrict__ slots) {
  __shared__ double2 xI[TB], xJ[TB];
  __shared__ double2 rowp[8][TB];
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const int b0 = (i + 1) / TB;
  const int nt = nblk - b0;
  const long long ntiles = (long long)nt * (nt + 1) / 2;
  const long long lo = (long long)i + 1;
  const double2* xcol = A + (long long)i * N;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int bi = (int)floor((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((long long)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
    while ((long long)bi * (bi + 1) / 2 > t) --bi;
    const int bj = (int)(t - (long long)bi * (bi + 1) / 2);
    const int I = b0 + bi, J = b0 + bj;
    const long long R0 = (long long)I * TB, C0 = (long long)J * TB;
    __syncthreads();
    if (tid < TB) {
      const long long r = R0 + tid;
      xI[tid] = (r >= lo && r < N) ? xcol[r] : make_double2(0, 0);
    } else if (tid < 2 * TB) {
      const long long cc = C0 + tid - TB;
      xJ[tid - TB] = (cc >= lo && cc < N) ? xcol[cc] : make_double2(0, 0);
    }
    __syncthreads();
    const bool diag = (I == J);
    double2 rp0 = make_double2(0, 0), rp1 = make_double2(0, 0);
    double2 cp[8];
    const long long ra = R0 + lane, rb = R0 + lane + 32;
    const bool va = (ra >= lo && ra < N), vb = (rb >= lo && rb < N);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int cl = wp + 8 * m;
      const long long cc = C0 + cl;
      cp[m] = make_double2(0, 0);
      const bool vc = (cc >= lo && cc < N);
      if (!vc) continue;
      const double2* colp = A + cc * N;
      const double2 xj = xJ[cl];
      if (va && (!diag || lane >= cl)) {
        double2 a = colp[ra];
        if (diag && lane == cl) a.y = 0.0;
        rp0 = cadd(rp0, cmul(a, xj));
        if (!(diag && lane == cl)) cp[m] = cadd(cp[m], cmulc(a, xI[lane]));
      }
      if (vb && (!diag || lane + 32 >= cl)) {
        double2 a = colp[rb];
        if (diag && lane + 32 == cl) a.y = 0.0;
        rp1 = cadd(rp1, cmul(a, xj));
        if (!(diag && lane + 32 == cl)) cp[m] = cadd(cp[m], cmulc(a, xI[lane + 32]));
      }
    }
    rowp[wp][lane] = rp0;
    rowp[wp][lane + 32] = rp1;
    // column partials: reduce over the 32 lanes for each of this warp's 8 columns
    double2 mycol = make_double2(0, 0);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      double2 s = warp_sum2(cp[m]);
      if (lane == m) mycol = s;
    }
    __syncthreads();
    double2* sIJ = slots + ((long long)I * nblk + J) * TB;
    double2* sJI = slots + ((long long)J * nblk + I) * TB;
    if (tid < TB) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < 8; ++k) s = cadd(s, rowp[k][tid]);
      if (!diag) sIJ[tid] = s;
      else rowp[0][tid] = s;   // combined below
    }
    __syncthreads();
    if (lane < 8) {
      const int cl = wp + 8 * lane;   // column owned by (warp wp, m = lane)
      if (!diag) sJI[cl] = mycol;
      else rowp[1][cl] = mycol;
    }
    __syncthreads();
    if (diag && tid < TB) sIJ[tid] = cadd(rowp[0][tid], rowp[1][tid]);
  }
}

// (4) y rows from slots; w = tau*(y - V z1 - W z2); g update; partial w^H v
__global__ void __launch_bounds__(256) k_hemv_finish(double2* A, long long N, double2* Wp, int j0, int p, int i, int nblk,
                                                     const double2* slots, const double2* partC, int nC,
                                                     const ColScal* sc, double2* g, double2* partE) {
  __shared__ double2 zz[2 * NB + NG];
  __shared__ double2 acc4[4][TB];
  __shared__ double2 red[8];
  const int tid = threadIdx.x;
  const int nval = 2 * p + NG;
  for (int q = tid; q < nval; q += blockDim.x) {
    double2 s = make_double2(0, 0);
    for (int k = 0; k < nC; ++k) s = cadd(s, partC[(long long)k * (2 * NB + NG) + q]);
    zz[q] = s;
  }
  const int b0 = (i + 1) / TB;
  const int a = b0 + blockIdx.x;   // block-row
  const int e = tid & (TB - 1), part = tid >> 6;
  double2 s = make_double2(0, 0);
  for (int b = b0 + part; b < nblk; b += 4) s = cadd(s, slots[((long long)a * nblk + b) * TB + e]);
  acc4[part][e] = s;
  __syncthreads();
  const ColScal c = *sc;
  double2 dot = make_double2(0, 0);
  if (tid < TB) {
    const long long r = (long long)a * TB + tid;
    if (r >= (long long)i + 1 && r < N) {
      double2 y = cadd(cadd(acc4[0][tid], acc4[1][tid]), cadd(acc4[2][tid], acc4[3][tid]));
      double2 t1 = make_double2(0, 0), t2 = make_double2(0, 0);
      for (int q = 0; q < p; ++q) {
        t1 = cadd(t1, cmul(A[r + (long long)(j0 + q) * N], zz[q]));
        t2 = cadd(t2, cmul(Wp[r + (long long)q * N], zz[p + q]));
      }
      const double2 w = cmul(c.tau, csub(csub(y, t1), t2));
      Wp[r + (long long)p * N] = w;
      const double2 v = A[r + (long long)i * N];
      dot = cmulc(w, v);
      // g <- g - tau conj(v) (v^T g)
      const double2 tv = cmul(c.tau, cconj(v));
#pragma unroll
      for (int al = 0; al < NG; ++al) {
        const double2 sa = zz[2 * p + al];
        g[(long long)al * N + r] = csub(g[(long long)al * N + r], cmul(tv, sa));
      }
    }
  }
  if (tid < 64) {
    dot = warp_sum2(dot);
    if ((tid & 31) == 0) red[tid >> 5] = dot;
  }
  __syncthreads();
  if (tid == 0) partE[blockIdx.x] = cadd(red[0], red[1]);
}

// (4b) w += alpha2 v with alpha2 = -tau/2 (w^H v)
__global__ void __launch_bounds__(RB) k_wfix(const double2* A, long long N, double2* Wp, int p, int i,
                                             const double2* partE, int nE, const ColScal* sc) {
  __shared__ double2 s_alpha;
  const int tid = threadIdx.x;
  if (tid == 0) {
    double2 s = make_double2(0, 0);
    for (int k = 0; k < nE; ++k) s = cadd(s, partE[k]);
    const ColScal c = *sc;
    s_alpha = cscale(cmul(c.tau, s), -0.5);
  }
  __syncthreads();
  const long long r = (long long)i + 1 + (long long)blockIdx.x * RB + tid;
  if (r < N) {
    const double2 v = A[r + (long long)i * N];
    Wp[r + (long long)p * N] = cadd(Wp[r + (long long)p * N], cmul(s_alpha, v));
  }
}

// Trailing update A22 -= V W^H + W V^H on the lower triangle with FP64 mma.sync.
// Real form: C_re -= Vr Wr^T + Vi Wi^T + Wr Vr^T + Wi Vi^T
//            C_im -= Vi Wr^T - Vr Wi^T + Wi Vr^T - Wr Vi^T
constexpr int HK = 8;         // q-chunk staged per step
constexpr int HKP = HK + 4;   // padded row stride (bank-conflict free 16-byte loads)

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a0), "d"(a1), "d"(b0));
}

__global__ void __launch_bounds__(256) k_her2k(double2* A, long long N, const double2* Wp, int j0, int jb, int k0) {
  __shared__ __align__(16) double2 sVr[TB][HKP], sWr[TB][HKP], sVc[TB][HKP], sWc[TB][HKP];
  const long long t = blockIdx.x;
  int bi = (int)floor((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((long long)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((long long)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (long long)bi * (bi + 1) / 2);
  const long long r0 = (long long)k0 + (long long)bi * TB, c0 = (long long)k0 + (long long)bj * TB;
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const int wr = wp & 3, wc = wp >> 2;
  const int gq = lane >> 2, tq = lane & 3;
  double accr[4][4], acci[4][4];
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int k = 0; k < 4; ++k) accr[n][k] = acci[n][k] = 0.0;

  for (int qc = 0; qc < jb; qc += HK) {
    __syncthreads();
    for (int it = tid; it < TB * HK; it += 256) {
      const int rr = it % TB, q = it / TB;
      const long long rg = r0 + rr, cg = c0 + rr;
      const bool qv = (qc + q) < jb;
      const long long qcol = (long long)(j0 + qc + q);
      sVr[rr][q] = (qv && rg < N) ? A[rg + qcol * N] : make_double2(0, 0);
      sWr[rr][q] = (qv && rg < N) ? Wp[rg + (long long)(qc + q) * N] : make_double2(0, 0);
      sVc[rr][q] = (qv && cg < N) ? A[cg + qcol * N] : make_double2(0, 0);
      sWc[rr][q] = (qv && cg < N) ? Wp[cg + (long long)(qc + q) * N] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < HK; kk += 4) {
      const int row = wr * 16 + gq;
      const double2 v0 = sVr[row][kk + tq], v1 = sVr[row + 8][kk + tq];
      const double2 w0 = sWr[row][kk + tq], w1 = sWr[row + 8][kk + tq];
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const int col = wc * 32 + n * 8 + gq;
        const double2 bw = sWc[col][kk + tq], bv = sVc[col][kk + tq];
        dmma(accr[n], v0.x, v1.x, bw.x);
        dmma(accr[n], v0.y, v1.y, bw.y);
        dmma(accr[n], w0.x, w1.x, bv.x);
        dmma(accr[n], w0.y, w1.y, bv.y);
        dmma(acci[n], v0.y, v1.y, bw.x);
        dmma(acci[n], -v0.x, -v1.x, bw.y);
        dmma(acci[n], w0.y, w1.y, bv.x);
        dmma(acci[n], -w0.x, -w1.x, bv.y);
      }
    }
  }
#pragma unroll
  for (int n = 0; n < 4; ++n) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const long long row = r0 + wr * 16 + gq + ((k >> 1) ? 8 : 0);
      const long long col = c0 + wc * 32 + n * 8 + 2 * tq + (k & 1);
      if (row < N && col < N && row >= col) {
        double2* pa = A + row + col * N;
        double2 a = *pa;
        a.x -= accr[n][k];
        a.y = (row == col) ? 0.0 : a.y - acci[n][k];
        *pa = a;
      }
    }
  }
}

__global__ void k_last_diag(const double2* A, long long N, double* d) {
  d[N - 1] = A[(N - 1) + (N - 1) * N].x;
}

__global__ void k_copy_g(const double2* h, double2* g, long long n) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) g[i] = h[i];
}

}  // namespace

int run_tridiagonalise(wtbg_ctx* ctx) {
  const long long N = ctx->N;
  if (N < 2) return set_err(ctx, WTBG_ERR_ARG, "tridiagonalise: N < 2");
  const int nblk = (int)((N + TB - 1) / TB);
  const int maxRB = (int)((N + RB - 1) / RB) + 1;
  ENSURE(ctx->d, (size_t)N * 8);
  ENSURE(ctx->e, (size_t)N * 8);
  ENSURE(ctx->tau, (size_t)N * 16);
  ENSURE(ctx->g, (size_t)N * 16 * NG);
  ENSURE(ctx->Wp, (size_t)N * 16 * NB);
  ENSURE(ctx->slots, (size_t)nblk * nblk * TB * 16);
  ENSURE(ctx->part, (size_t)maxRB * (2 * NB + NG) * 16 + (size_t)maxRB * 16 + (size_t)(nblk + 1) * 16 + 4096);
  ENSURE(ctx->scal, sizeof(ColScal) + 64);
  double2* A = ctx->H.as<double2>();
  double2* Wp = ctx->Wp.as<double2>();
  double* d = ctx->d.as<double>();
  double* e = ctx->e.as<double>();
  double2* tau = ctx->tau.as<double2>();
  double2* g = ctx->g.as<double2>();
  double2* slots = ctx->slots.as<double2>();
  char* pb = ctx->part.as<char>();
  double* partA = reinterpret_cast<double*>(pb);
  double2* partC = reinterpret_cast<double2*>(pb + (size_t)maxRB * 16);
  double2* partE = partC + (size_t)maxRB * (2 * NB + NG);
  ColScal* sc = ctx->scal.as<ColScal>();
  cudaStream_t s = ctx->stream;

  if (ctx->have_velocity) {
    k_copy_g<<<(int)((N * NG + 255) / 256), 256, 0, s>>>(ctx->h.as<double2>(), g, N * NG);
  } else {
    CK(cudaMemsetAsync(g, 0, (size_t)N * 16 * NG, s));
  }
  CKL("k_copy_g");
  int num_sms = 148;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, ctx->device);

  for (long long j0 = 0; j0 < N - 1; j0 += NB) {
    const int jb = (int)((N - 1 - j0) < NB ? (N - 1 - j0) : NB);
    for (int p = 0; p < jb; ++p) {
      const int i = (int)(j0 + p);
      const int nA = (int)((N - i + RB - 1) / RB);
      k_colupd<<<nA, RB, 0, s>>>(A, N, Wp, (int)j0, p, i, partA);
      k_reflector<<<1, 256, 0, s>>>(A, N, i, partA, nA, d, e, tau, sc);
      const int nC = (int)((N - i - 1 + RB - 1) / RB);
      k_scale_dots<<<nC, RB, 0, s>>>(A, N, Wp, (int)j0, p, i, sc, g, partC);
      const int b0 = (i + 1) / TB;
      const long long nt = nblk - b0;
      const long long ntiles = nt * (nt + 1) / 2;
      const int grid = (int)(ntiles < (long long)num_sms * 8 ? ntiles : (long long)num_sms * 8);
      k_hemv<<<grid, 256, 0, s>>>(A, N, i, nblk, slots);
      const int nE = nblk - b0;
      k_hemv_finish<<<nE, 256, 0, s>>>(A, N, Wp, (int)j0, p, i, nblk, slots, partC, nC, sc, g, partE);
      k_wfix<<<nC, RB, 0, s>>>(A, N, Wp, p, i, partE, nE, sc);
    }
    CKL("tridiagonal panel");
    const long long k0 = j0 + jb;
    if (k0 < N) {
      const long long T = (N - k0 + TB - 1) / TB;
      const long long ntile = T * (T + 1) / 2;
      k_her2k<<<(unsigned)ntile, 256, 0, s>>>(A, N, Wp, (int)j0, jb, (int)k0);
      CKL("k_her2k");
    }
  }
  k_last_diag<<<1, 1, 0, s>>>(A, N, d);
  CKL("k_last_diag");
  return 0;
}
