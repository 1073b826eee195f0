// Block Davidson on the built BSE matrix: the lowest (or highest) exciton states without a
// dense solve.  This is the fast form of the path (no reference counterpart; its oracle is
// the dense FP64 solve).  All arithmetic is FP64; the matrix is the lower-stored Hermitian
// N x N array written by k_bse_build and is not modified.
//
// Iteration (basis V = [X T], nb + nb columns):
//   R = H X - X diag(theta),  T = R / (diag(H) - theta)   (Davidson preconditioner)
//   T <- T - X (X^H T) (twice), T <- T chol(T^H T)^-1 (twice: CholQR2)
//   M = V^H (H V)  (2nb x 2nb),  (theta, Y) = eig(M) by a one-CTA tridiagonal eigensolver,  X = V Y, HX = HV Y
// Oscillator strengths of the converged states: f_n = |sum_j X_jn h_j|^2 (dielbsev,
// bse_subs.f90:336-378, no conjugate on the eigenvector).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

#include "common.cuh"

namespace {

constexpr int TB = 64;        // tile edge
constexpr int JCH = 8;        // column chunks of the Hermitian product (partials)
constexpr int NG = 5;
constexpr int kMaxRR = 80;    // largest Rayleigh-Ritz size (two 80x80 complex matrices fit in one CTA)

// Y[part][N][m] partial of H X over the block-columns of chunk blockIdx.y; H lower-stored.
// The 64x64 tile H(I,J) (Hermitian-completed from the lower triangle) and the 64 rows of X
// are staged in shared memory; the product runs on the FP64 tensor cores as
// mma.sync m16n8k16 with the complex arithmetic concatenated along k:
//   Yr += [Hr | -Hi] [Xr ; Xi],   Yi += [Hr | Hi] [Xi ; Xr]     (8 complex columns per MMA).
// 8 warps = 4 row groups of 16 rows x 2 halves of the tile's 64 columns; the halves are
// added through shared memory at the end. Fragment layout of m16n8k16 f64: a_i holds row
// gq + 8 (i % 2), k = tq + 4 (i / 2); b_j holds k = tq + 4 j, column gq; c holds rows gq, gq + 8
// and columns 2 tq, 2 tq + 1.
constexpr int HT = TB + 2;   // tile column stride (conflict-free fragment loads)

__device__ __forceinline__ void mma16(double (&c)[4], const double (&a)[8], double b0, double b1, double b2,
                                      double b3) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b0), "d"(b1),
        "d"(b2), "d"(b3));
}

template <int MV>
__global__ void __launch_bounds__(256) k_hemm(const double2* __restrict__ A, long long N, const double2* __restrict__ X,
                                              int ldx, double2* __restrict__ Yp) {
  constexpr int M = 8 * MV;
  constexpr int XS = M + 2;   // xs row stride
  extern __shared__ __align__(16) unsigned char hsm[];
  double2* tile = reinterpret_cast<double2*>(hsm);                                   // tile[c * HT + r]
  double2* xs = reinterpret_cast<double2*>(hsm + sizeof(double2) * TB * HT);         // xs[c * XS + v]
  const int I = blockIdx.x;
  const int nblk = (int)((N + TB - 1) / TB);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int rg = warp & 3, kh = warp >> 2;   // row group, column half
  double accr[MV][4], acci[MV][4];
#pragma unroll
  for (int v = 0; v < MV; ++v)
#pragma unroll
    for (int k = 0; k < 4; ++k) accr[v][k] = acci[v][k] = 0.0;
  const int jper = (nblk + JCH - 1) / JCH;
  const int J0 = blockIdx.y * jper, J1 = min(nblk, J0 + jper);
  const long long R0 = (long long)I * TB;
  for (int J = J0; J < J1; ++J) {
    const long long C0 = (long long)J * TB;
    __syncthreads();
    // H(I,J): J < I from the lower tile (rows I, cols J); J > I from the conj transpose of
    // the lower tile (rows J, cols I); J == I from the lower part of the diagonal tile, mirrored
    for (int it = tid; it < TB * TB; it += 256) {
      const int a = it & (TB - 1), b = it >> 6;   // a fastest: coalesced global reads
      double2 v = make_double2(0, 0);
      if (J < I) {
        const long long rr = R0 + a, cc = C0 + b;
        if (rr < N && cc < N) v = A[rr + cc * N];
        tile[b * HT + a] = v;                 // H(R0+a, C0+b)
      } else if (J > I) {
        const long long rr = C0 + a, cc = R0 + b;   // lower element (C0+a, R0+b)
        if (rr < N && cc < N) v = cconj(A[rr + cc * N]);
        tile[a * HT + b] = v;                 // H(R0+b, C0+a) = conj(L(C0+a, R0+b))
      } else {
        const long long rr = R0 + a, cc = C0 + b;
        if (rr < N && cc < N) {
          if (a > b) {
            v = A[rr + cc * N];
            tile[b * HT + a] = v;
            tile[a * HT + b] = cconj(v);
          } else if (a == b) {
            v = A[rr + cc * N];
            tile[a * HT + a] = make_double2(v.x, 0.0);
          }
        } else {
          tile[b * HT + a] = make_double2(0, 0);
          tile[a * HT + b] = make_double2(0, 0);
        }
      }
    }
    for (int it = tid; it < TB * M; it += 256) {
      const int c = it % TB, v = it / TB;
      const long long rr = C0 + c;
      xs[c * XS + v] = (rr < N) ? X[rr + (long long)v * ldx] : make_double2(0, 0);
    }
    __syncthreads();
    const int row = rg * 16 + gq;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const int c0 = kh * 32 + ks * 8;
      const double2 h00 = tile[(c0 + tq) * HT + row], h10 = tile[(c0 + tq) * HT + row + 8];
      const double2 h01 = tile[(c0 + tq + 4) * HT + row], h11 = tile[(c0 + tq + 4) * HT + row + 8];
      const double are[8] = {h00.x, h10.x, h01.x, h11.x, -h00.y, -h10.y, -h01.y, -h11.y};
      const double aim[8] = {h00.x, h10.x, h01.x, h11.x, h00.y, h10.y, h01.y, h11.y};
#pragma unroll
      for (int v = 0; v < MV; ++v) {
        const double2 x0 = xs[(c0 + tq) * XS + v * 8 + gq], x1 = xs[(c0 + tq + 4) * XS + v * 8 + gq];
        mma16(accr[v], are, x0.x, x1.x, x0.y, x1.y);
        mma16(acci[v], aim, x0.y, x1.y, x0.x, x1.x);
      }
    }
  }
  // add the two column halves through shared memory, then store the partial
  __syncthreads();
  double2* red = tile;   // [64 rows][M] of the kh = 1 warps
  if (kh == 1) {
#pragma unroll
    for (int v = 0; v < MV; ++v)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int rr = rg * 16 + gq + ((k >> 1) ? 8 : 0), cc = v * 8 + 2 * tq + (k & 1);
        red[rr * M + cc] = make_double2(accr[v][k], acci[v][k]);
      }
  }
  __syncthreads();
  if (kh == 0) {
#pragma unroll
    for (int v = 0; v < MV; ++v)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int rr = rg * 16 + gq + ((k >> 1) ? 8 : 0), cc = v * 8 + 2 * tq + (k & 1);
        const long long gr = R0 + rr;
        if (gr < N) {
          const double2 o = red[rr * M + cc];
          Yp[((long long)blockIdx.y * M + cc) * N + gr] = make_double2(accr[v][k] + o.x, acci[v][k] + o.y);
        }
      }
  }
}

// Y = H X reading every lower tile once (for narrow blocks, M = 8*MV <= 16): a CTA streams a
// chunk of up to LHS tiles down block-column J.  Row products L_IJ X_J go to slot[I][J];
// column products L_IJ^H X_I accumulate in registers over the chunk and go to slot[J][I0]
// (zeros for the other tiles of the chunk; added into slot[J][J] for the chunk holding the
// diagonal tile), so that Y_a = sum_b slot[a][b].  Slot layout [a][b][v][64].
constexpr int LHS = 8;
template <int MV>
__global__ void __launch_bounds__(256) k_hemm_lower(const double2* __restrict__ A, long long N, const double2* __restrict__ X,
                                                    int ldx, int nblk, double2* __restrict__ slots) {
  constexpr int M = 8 * MV;
  extern __shared__ __align__(16) unsigned char hsm[];
  double2 (*tile)[TB + 1] = reinterpret_cast<double2 (*)[TB + 1]>(hsm);   // tile[c][r] = H(R0+r, C0+c)
  double2 (*xJ)[M + 1] = reinterpret_cast<double2 (*)[M + 1]>(hsm + sizeof(double2) * TB * (TB + 1));
  double2 (*xI)[M + 1] = xJ + TB;
  const int J = blockIdx.x;
  const int I0 = J + blockIdx.y * LHS;
  if (I0 >= nblk) return;
  const int I1 = min(I0 + LHS, nblk);
  const int tid = threadIdx.x, r = tid & 31, vg = tid >> 5;
  const long long C0 = (long long)J * TB;
  for (int it = tid; it < TB * M; it += 256) {
    const int c = it % TB, v = it / TB;
    xJ[c][v] = (C0 + c < N) ? X[C0 + c + (long long)v * ldx] : make_double2(0, 0);
  }
  double2 cacc[2][MV];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int v = 0; v < MV; ++v) cacc[a][v] = make_double2(0, 0);
  for (int I = I0; I < I1; ++I) {
    const long long R0 = (long long)I * TB;
    const bool diag = (I == J);
    __syncthreads();
    for (int it = tid; it < TB * TB; it += 256) {
      const int a = it & (TB - 1), b = it >> 6;
      const long long rr = R0 + a, cc = C0 + b;
      if (!diag) {
        tile[b][a] = (rr < N && cc < N) ? A[rr + cc * N] : make_double2(0, 0);
      } else if (rr < N && cc < N) {
        if (a > b) {
          const double2 v = A[rr + cc * N];
          tile[b][a] = v;
          tile[a][b] = cconj(v);
        } else if (a == b) {
          tile[a][a] = make_double2(A[rr + cc * N].x, 0.0);
        }
      } else {
        tile[b][a] = make_double2(0, 0);
        tile[a][b] = make_double2(0, 0);
      }
    }
    for (int it = tid; it < TB * M; it += 256) {
      const int c = it % TB, v = it / TB;
      xI[c][v] = (R0 + c < N) ? X[R0 + c + (long long)v * ldx] : make_double2(0, 0);
    }
    __syncthreads();
    // row products
    double2 acc[2][MV];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int v = 0; v < MV; ++v) acc[a][v] = make_double2(0, 0);
#pragma unroll 4
    for (int c = 0; c < TB; ++c) {
      const double2 h0 = tile[c][r], h1 = tile[c][r + 32];
#pragma unroll
      for (int v = 0; v < MV; ++v) {
        const double2 x = xJ[c][vg * MV + v];
        acc[0][v] = cadd(acc[0][v], cmul(h0, x));
        acc[1][v] = cadd(acc[1][v], cmul(h1, x));
      }
    }
    double2* sl = slots + ((long long)I * nblk + J) * M * TB;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int v = 0; v < MV; ++v) sl[(long long)(vg * MV + v) * TB + r + 32 * a] = acc[a][v];
    // column products (the diagonal tile is complete in its row products)
    if (!diag) {
#pragma unroll 4
      for (int rr = 0; rr < TB; ++rr) {
        const double2 h0 = tile[r][rr], h1 = tile[r + 32][rr];   // L(R0+rr, C0+c), c = r, r+32
#pragma unroll
        for (int v = 0; v < MV; ++v) {
          const double2 x = xI[rr][vg * MV + v];
          cacc[0][v] = cadd(cacc[0][v], cmulc(h0, x));
          cacc[1][v] = cadd(cacc[1][v], cmulc(h1, x));
        }
      }
    }
  }
  double2* sl = slots + ((long long)J * nblk + I0) * M * TB;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int v = 0; v < MV; ++v) {
      double2* p = sl + (long long)(vg * MV + v) * TB + r + 32 * a;
      *p = (I0 == J) ? cadd(*p, cacc[a][v]) : cacc[a][v];
    }
  for (int I = I0 + 1; I < I1; ++I) {
    double2* z = slots + ((long long)J * nblk + I) * M * TB;
    for (int it = tid; it < M * TB; it += 256) z[it] = make_double2(0, 0);
  }
}

__global__ void k_sum_slots(const double2* slots, long long N, int nblk, int m, double2* Y, int ldy) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nblk * TB * m) return;
  const int row = (int)(i % TB);
  const int v = (int)((i / TB) % m);
  const int a = (int)(i / ((long long)TB * m));
  const long long gr = (long long)a * TB + row;
  if (gr >= N) return;
  double2 s = make_double2(0, 0);
  for (int b = 0; b < nblk; ++b) s = cadd(s, slots[(((long long)a * nblk + b) * m + v) * TB + row]);
  Y[gr + (long long)v * ldy] = s;
}

// Y(:, v) = sum over chunks of the partials
__global__ void k_sum_parts(const double2* Yp, long long N, int m, double2* Y, int ldy) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N * m) return;
  const long long row = i % N, v = i / N;
  double2 s = make_double2(0, 0);
  for (int p = 0; p < JCH; ++p) s = cadd(s, Yp[((long long)p * m + v) * N + row]);
  Y[row + v * ldy] = s;
}

// C (p x q) = A^H B, A (N x p, lda), B (N x q, ldb): per-block partials [blk][p*q]. Rows are
// staged GR at a time in shared memory; the 16 x 16 threads each own a register tile of
// outputs (a = tx + 16 i, b = ty + 16 j), so every staged value feeds up to 5 products.
constexpr int GR = 16;
constexpr int GT = 5;   // largest register tile: p, q <= 16 * GT = 80
template <int T>
__global__ void __launch_bounds__(256) k_gram(const double2* A, int lda, int p, const double2* B, int ldb, int q,
                                              long long N, double2* part) {
  __shared__ double2 as[GR][kMaxRR + 1], bsm[GR][kMaxRR + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const long long rows_per = (N + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * rows_per, r1 = min(N, r0 + rows_per);
  double2 acc[T][T];
#pragma unroll
  for (int i = 0; i < T; ++i)
#pragma unroll
    for (int j = 0; j < T; ++j) acc[i][j] = make_double2(0, 0);
  for (long long c0 = r0; c0 < r1; c0 += GR) {
    __syncthreads();
    for (int it = tid; it < GR * p; it += 256) {
      const int rr = it % GR, a = it / GR;
      as[rr][a] = (c0 + rr < r1) ? A[c0 + rr + (long long)a * lda] : make_double2(0, 0);
    }
    for (int it = tid; it < GR * q; it += 256) {
      const int rr = it % GR, b = it / GR;
      bsm[rr][b] = (c0 + rr < r1) ? B[c0 + rr + (long long)b * ldb] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < GR; ++rr) {
      double2 av[T], bv[T];
#pragma unroll
      for (int i = 0; i < T; ++i) av[i] = as[rr][min(tx + 16 * i, kMaxRR)];
#pragma unroll
      for (int j = 0; j < T; ++j) bv[j] = bsm[rr][min(ty + 16 * j, kMaxRR)];
#pragma unroll
      for (int i = 0; i < T; ++i)
#pragma unroll
        for (int j = 0; j < T; ++j) {   // conj(a) b as four FMAs
          acc[i][j].x = fma(av[i].x, bv[j].x, acc[i][j].x);
          acc[i][j].x = fma(av[i].y, bv[j].y, acc[i][j].x);
          acc[i][j].y = fma(av[i].x, bv[j].y, acc[i][j].y);
          acc[i][j].y = fma(-av[i].y, bv[j].x, acc[i][j].y);
        }
    }
  }
  const int pq = p * q;
#pragma unroll
  for (int i = 0; i < T; ++i)
#pragma unroll
    for (int j = 0; j < T; ++j) {
      const int a = tx + 16 * i, b = ty + 16 * j;
      if (a < p && b < q) part[(long long)blockIdx.x * pq + a + b * p] = acc[i][j];
    }
}

// C[i] = sum over blocks of part[blk][i]: 32 outputs x 8 block groups per CTA
__global__ void k_gram_sum(const double2* part, int nparts, int pq, double2* C) {
  __shared__ double2 red[8][33];
  const int x = threadIdx.x & 31, y = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + x;
  double2 s = make_double2(0, 0);
  if (i < pq)
    for (int k = y; k < nparts; k += 8) s = cadd(s, part[(long long)k * pq + i]);
  red[y][x] = s;
  __syncthreads();
  if (y == 0 && i < pq) {
    for (int k = 1; k < 8; ++k) s = cadd(s, red[k][x]);
    C[i] = s;
  }
}

// C (N x q, ldc) = A (N x p, lda) * B (p x q, column-major, ldb = p), or C -= A * B.
// Grid (rows / 256, q / 8): every thread owns one row and eight output columns.
template <bool SUB>
__global__ void __launch_bounds__(256) k_tall_gemm(const double2* A, int lda, int p, const double2* B, int q,
                                                   long long N, double2* Cm, int ldc) {
  __shared__ double2 bs[kMaxRR * 8];
  const int b0 = blockIdx.y * 8;
  const int nb = min(8, q - b0);
  for (int i = threadIdx.x; i < p * 8; i += blockDim.x) {
    const int a = i % p, k = i / p;
    bs[a * 8 + k] = (k < nb) ? B[a + (b0 + k) * p] : make_double2(0, 0);
  }
  __syncthreads();
  const long long rr = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (rr >= N) return;
  double2 s[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) s[k] = make_double2(0, 0);
#pragma unroll 4
  for (int a = 0; a < p; ++a) {
    const double2 x = A[rr + (long long)a * lda];
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] = cadd(s[k], cmul(x, bs[a * 8 + k]));
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (k >= nb) break;
    double2* cp = Cm + rr + (long long)(b0 + k) * ldc;
    *cp = SUB ? csub(*cp, s[k]) : s[k];
  }
}

// G (q x q Hermitian PD, q <= 64) -> Rinv (upper triangular, column-major) with G = R^H R,
// R = L^H from a right-looking Cholesky G = L L^H in shared memory; L^-1 by row-wise forward
// substitution with all columns in parallel, Rinv = (L^-1)^H. A non-positive pivot gets a zero
// row in Rinv (its vector is dropped). One CTA.
__global__ void __launch_bounds__(512) k_chol_inv(const double2* G, int q, double2* Rinv, int* bad) {
  extern __shared__ double2 csm[];
  const int ld = q + 1;
  double2* Lm = csm;             // L(i, k) at Lm[i + k * ld] (lower)
  double2* Xm = csm + q * ld;    // X = L^-1 (lower), X(i, j) at Xm[i + j * ld]
  __shared__ double s_piv[64];
  const int tid = threadIdx.x, bs = blockDim.x;
  for (int it = tid; it < q * q; it += bs) {
    const int i = it % q, k = it / q;
    Lm[i + k * ld] = (i >= k) ? G[i + k * q] : make_double2(0, 0);
    Xm[i + k * ld] = make_double2(0, 0);
  }
  __syncthreads();
  for (int j = 0; j < q; ++j) {
    const double gjj = Lm[j + j * ld].x;
    const double scale = fabs(G[j + j * q].x) + 1e-300;
    const double rjj = (gjj > 1e-28 * scale) ? sqrt(gjj) : 0.0;
    __syncthreads();
    if (tid == 0) {
      s_piv[j] = rjj;
      Lm[j + j * ld] = make_double2(rjj, 0.0);
    }
    const double inv = rjj > 0.0 ? 1.0 / rjj : 0.0;
    for (int i = j + 1 + tid; i < q; i += bs) Lm[i + j * ld] = cscale(Lm[i + j * ld], inv);
    __syncthreads();
    // trailing update of the lower part: L(i, k) -= L(i, j) conj(L(k, j)), i >= k > j
    const int m = q - j - 1;
    for (int it = tid; it < m * m; it += bs) {
      const int i = j + 1 + it % m, k = j + 1 + it / m;
      if (i >= k) Lm[i + k * ld] = csub(Lm[i + k * ld], cmul(Lm[i + j * ld], cconj(Lm[k + j * ld])));
    }
    __syncthreads();
  }
  // X = L^-1: row i from rows < i, all columns j <= i in parallel
  for (int i = 0; i < q; ++i) {
    const double lii = s_piv[i];
    for (int j = tid; j <= i; j += bs) {
      double2 sacc = (i == j) ? make_double2(1.0, 0.0) : make_double2(0, 0);
      for (int k = j; k < i; ++k) sacc = csub(sacc, cmul(Lm[i + k * ld], Xm[k + j * ld]));
      Xm[i + j * ld] = (lii > 0.0) ? cscale(sacc, 1.0 / lii) : make_double2(0, 0);
    }
    __syncthreads();
  }
  // Rinv = X^H: Rinv(a, b) = conj(X(b, a)), upper triangular
  for (int it = tid; it < q * q; it += bs) {
    const int a = it % q, b = it / q;
    Rinv[it] = (a <= b) ? cconj(Xm[b + a * ld]) : make_double2(0, 0);
  }
  if (tid == 0) {
    int nbad = 0;
    for (int j = 0; j < q; ++j) nbad += (s_piv[j] == 0.0);
    *bad = nbad;
  }
}

// One-CTA Hermitian eigensolver for the Rayleigh-Ritz matrix (n <= kMaxRR, nb wanted pairs):
//  1. Householder reduction to real tridiagonal form in shared memory (lower reflectors as in
//     ZHETRD: H = I - tau v v^H, v(1) = 1, beta real), the A22 v product with four threads a row;
//  2. multisection Sturm bisection: blockDim/nb threads per wanted eigenvalue each evaluate one
//     point of the current interval, shrinking it (G+1)-fold per round, a fixed number of rounds
//     down to ~eps |T|;
//  3. inverse iteration with partial pivoting (3 steps) for the eigenvectors of T, eigenvalues
//     closer than 1e-7 |T| handled in order by one thread with Gram-Schmidt;
//  4. back-transform y = H_0 H_1 ... H_{n-2} z, one warp per vector in shared memory.
constexpr int RR_THREADS = 512;

__host__ __device__ constexpr size_t rr_smem_bytes(int n, int nb) {
  return (size_t)16 * ((size_t)n * n + 3 * n + (size_t)n * nb) + (size_t)8 * (2 * n + 3 * kMaxRR + (size_t)n * nb) +
         (size_t)4 * RR_THREADS + 64;
}

// Number of eigenvalues of the symmetric tridiagonal (d, e) below x from the sign changes of
// the leading principal minors p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2} (two FMAs a step,
// no division), rescaled by exact powers of two; a zero minor counts as a sign change.
__device__ __forceinline__ int sturm_count(const double* dd, const double* ee, int n, double x) {
  double pm = 0.0, p = 1.0, sgn = 1.0;
  int cnt = 0;
  for (int i = 0; i < n; ++i) {
    const double e2 = (i > 0) ? ee[i - 1] * ee[i - 1] : 0.0;
    const double pn = fma(dd[i] - x, p, -e2 * pm);
    pm = p;
    p = pn;
    const double ap = fabs(p);
    if (ap > 0x1p+500) {
      p *= 0x1p-500;
      pm *= 0x1p-500;
    } else if (ap < 0x1p-500 && ap > 0.0) {
      p *= 0x1p+500;
      pm *= 0x1p+500;
    }
    const double s = (p == 0.0) ? -sgn : (p < 0.0 ? -1.0 : 1.0);
    cnt += (s != sgn);
    sgn = s;
    if (p == 0.0) p = sgn * (fabs(pm) * 0x1p-60 + 0x1p-1000);   // a zero minor: pivot -> sign change
  }
  return cnt;
}

__device__ __forceinline__ double2 warp_sum2(double2 t) {
  for (int o = 16; o > 0; o >>= 1) {
    t.x += __shfl_xor_sync(0xffffffffu, t.x, o);
    t.y += __shfl_xor_sync(0xffffffffu, t.y, o);
  }
  return t;
}

__global__ void __launch_bounds__(RR_THREADS) k_rr_tridiag(const double2* Min, int n, int nb, int descending,
                                                           double* theta, double2* Yout, int* status) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* A = reinterpret_cast<double2*>(smem);   // n x n, column-major; reflectors kept below the diagonal
  double2* vv = A + n * n;
  double2* pp = vv + n;
  double2* taus = pp + n;
  double2* Ys = taus + n;                           // n x nb back-transformed vectors
  double* dd = reinterpret_cast<double*>(Ys + n * nb);
  double* ee = dd + n;
  double* lam = ee + n;                             // kMaxRR
  double* blo = lam + kMaxRR;                       // kMaxRR
  double* bhi = blo + kMaxRR;                       // kMaxRR
  double* Z = bhi + kMaxRR;                         // n x nb eigenvectors of T
  int* cnt = reinterpret_cast<int*>(Z + n * nb);    // RR_THREADS
  __shared__ double red[RR_THREADS / 32];
  __shared__ double2 redc[RR_THREADS / 32];
  __shared__ double2 s_tau, s_scal, s_a2;
  __shared__ int s_triv;
  __shared__ double s_lo, s_hi, s_tn;
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  constexpr int bs = RR_THREADS, NW = RR_THREADS / 32;
  for (int it = tid; it < n * n; it += bs) {
    const int a = it % n, b = it / n;
    double2 v = Min[it];
    if (a == b) v.y = 0.0;
    if (a < b) v = cconj(Min[b + a * n]);
    A[it] = v;
  }
  __syncthreads();
  // ---- 1. tridiagonal reduction
  for (int j = 0; j < n - 1; ++j) {
    const int m = n - j - 1;
    double s = 0.0;
    for (int i = 1 + tid; i < m; i += bs) {
      const double2 x = A[(j + 1 + i) + j * n];
      s += x.x * x.x + x.y * x.y;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[wp] = s;
    __syncthreads();
    if (wp == 0) {
      double xn2 = (lane < NW) ? red[lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) xn2 += __shfl_xor_sync(0xffffffffu, xn2, o);
      if (lane == 0) {
        const double2 al = A[(j + 1) + j * n];
        if (xn2 == 0.0 && al.y == 0.0) {
          s_triv = 1;
          s_tau = make_double2(0, 0);
          ee[j] = al.x;
        } else {
          s_triv = 0;
          const double beta = -copysign(sqrt(al.x * al.x + al.y * al.y + xn2), al.x);
          const double ib = 1.0 / beta;
          s_tau = make_double2((beta - al.x) * ib, -al.y * ib);
          const double2 den = make_double2(al.x - beta, al.y);
          const double idn = 1.0 / (den.x * den.x + den.y * den.y);
          s_scal = make_double2(den.x * idn, -den.y * idn);
          ee[j] = beta;
        }
        dd[j] = A[j + j * n].x;
        taus[j] = s_tau;
      }
    }
    __syncthreads();
    const int triv = s_triv;
    const double2 tau = s_tau;
    for (int i = tid; i < m; i += bs) {
      const double2 v = (i == 0) ? make_double2(1, 0) : (triv ? make_double2(0, 0) : cmul(A[(j + 1 + i) + j * n], s_scal));
      vv[i] = v;
      A[(j + 1 + i) + j * n] = v;
    }
    __syncthreads();
    if (triv) continue;
    // p = tau A22 v: four threads per row; the partial p^H v of each row group on the fly
    double2 t = make_double2(0, 0);
    {
      const int part = tid & 3;
      const unsigned gmask = 0xFu << (lane & ~3);
      for (int i = tid >> 2; i < m; i += bs / 4) {
        double2 acc = make_double2(0, 0);
        for (int k = part; k < m; k += 4) acc = cadd(acc, cmul(A[(j + 1 + i) + (j + 1 + k) * n], vv[k]));
        acc.x += __shfl_xor_sync(gmask, acc.x, 1);
        acc.y += __shfl_xor_sync(gmask, acc.y, 1);
        acc.x += __shfl_xor_sync(gmask, acc.x, 2);
        acc.y += __shfl_xor_sync(gmask, acc.y, 2);
        const double2 pi = cmul(tau, acc);
        if (part == 0) {
          pp[i] = pi;
          t = cadd(t, cmulc(pi, vv[i]));
        }
      }
    }
    t = warp_sum2(t);
    if (lane == 0) redc[wp] = t;
    __syncthreads();
    if (wp == 0) {
      double2 sum = (lane < NW) ? redc[lane] : make_double2(0, 0);
      sum = warp_sum2(sum);
      if (lane == 0) s_a2 = cscale(cmul(tau, sum), -0.5);
    }
    __syncthreads();
    const double2 a2 = s_a2;
    for (int i = tid; i < m; i += bs) pp[i] = cadd(pp[i], cmul(a2, vv[i]));   // w
    __syncthreads();
    for (int it = tid; it < m * m; it += bs) {
      const int r = it % m, c = it / m;
      double2 x = A[(j + 1 + r) + (j + 1 + c) * n];
      x = csub(x, cadd(cmul(vv[r], cconj(pp[c])), cmul(pp[r], cconj(vv[c]))));
      A[(j + 1 + r) + (j + 1 + c) * n] = x;
    }
    __syncthreads();
  }
  if (tid == 0) {
    dd[n - 1] = A[(n - 1) + (n - 1) * n].x;
    double lo = 0.0, hi = 0.0;
    for (int i = 0; i < n; ++i) {
      const double r = (i > 0 ? fabs(ee[i - 1]) : 0.0) + (i < n - 1 ? fabs(ee[i]) : 0.0);
      lo = (i == 0) ? dd[i] - r : fmin(lo, dd[i] - r);
      hi = (i == 0) ? dd[i] + r : fmax(hi, dd[i] + r);
    }
    s_tn = fmax(fabs(lo), fabs(hi));
    const double pad = 4.0 * DBL_EPSILON * s_tn + 1e-300;
    s_lo = lo - pad;
    s_hi = hi + pad;
  }
  __syncthreads();
  // ---- 2. multisection bisection down to ~2^-44 of the Gershgorin width
  const int G = max(1, bs / nb);
  int rounds = 1;
  {
    double shrink = 1.0;
    while (shrink > 0x1p-44 && rounds < 64) {
      shrink /= (double)(G + 1);
      ++rounds;
    }
  }
  const double ig = 1.0 / (double)(G + 1);
  for (int e = tid; e < nb; e += bs) {
    blo[e] = s_lo;
    bhi[e] = s_hi;
  }
  __syncthreads();
  for (int rd = 0; rd < rounds; ++rd) {
    const int e = tid / G, g = tid % G;
    if (e < nb) {
      const double lo = blo[e], hi = bhi[e];
      const double x = lo + (hi - lo) * ((double)(g + 1) * ig);
      cnt[tid] = sturm_count(dd, ee, n, x);
    }
    __syncthreads();
    if (e < nb && g == 0) {
      const int mi = descending ? (n - 1 - e) : e;
      const double lo = blo[e], hi = bhi[e];
      double nlo = lo, nhi = hi;
      for (int gg = 0; gg < G; ++gg) {
        const double x = lo + (hi - lo) * ((double)(gg + 1) * ig);
        if (cnt[e * G + gg] <= mi) {
          nlo = x;
        } else {
          nhi = x;
          break;
        }
      }
      blo[e] = nlo;
      bhi[e] = nhi;
    }
    __syncthreads();
  }
  for (int e = tid; e < nb; e += bs) lam[e] = 0.5 * (blo[e] + bhi[e]);
  __syncthreads();
  // ---- 3. inverse iteration: T - lambda I = P L U factored once (partial pivoting), three
  //         solves; eigenvalues closer than 1e-7 |T| are done in order by their first thread
  if (tid < nb) {
    const double ctol = 1e-7 * fmax(1e-3, s_tn);
    const bool leader = (tid == 0) || fabs(lam[tid] - lam[tid - 1]) > ctol;
    if (leader) {
      int cs = 1;
      while (tid + cs < nb && fabs(lam[tid + cs] - lam[tid + cs - 1]) <= ctol) ++cs;
      const double pert = DBL_EPSILON * fmax(s_tn, 1e-300);
      double r1[kMaxRR], u2[kMaxRR], u3[kMaxRR], ml[kMaxRR];
      unsigned char sw[kMaxRR];
      for (int sidx = 0; sidx < cs; ++sidx) {
        const int col = tid + sidx;
        double* x = Z + col * n;
        const double lm = lam[col];
        double diag = dd[0] - lm, sup = (n > 1) ? ee[0] : 0.0;
        for (int k = 0; k < n - 1; ++k) {
          const double sub = ee[k], nd = dd[k + 1] - lm, nsup = (k + 1 < n - 1) ? ee[k + 1] : 0.0;
          if (fabs(diag) >= fabs(sub)) {
            if (fabs(diag) < pert) diag = copysign(pert, diag);
            const double rp = 1.0 / diag;
            const double mult = sub * rp;
            r1[k] = rp;
            u2[k] = sup;
            u3[k] = 0.0;
            ml[k] = mult;
            sw[k] = 0;
            diag = nd - mult * sup;
            sup = nsup;
          } else {
            const double rp = 1.0 / sub;
            const double mult = diag * rp;
            r1[k] = rp;
            u2[k] = nd;
            u3[k] = nsup;
            ml[k] = mult;
            sw[k] = 1;
            diag = sup - mult * nd;
            sup = -mult * nsup;
          }
        }
        if (fabs(diag) < pert) diag = copysign(pert, diag);
        const double rlast = 1.0 / diag;
        for (int k = 0; k < n; ++k) x[k] = 1.0 + 0.1 * (double)((k * 7 + col * 13) % 17) / 17.0;
        for (int itr = 0; itr < 3; ++itr) {
          double cur = x[0];
          for (int k = 0; k < n - 1; ++k) {
            const double nxt = x[k + 1];
            if (sw[k]) {
              x[k] = nxt;
              cur = cur - ml[k] * nxt;
            } else {
              x[k] = cur;
              cur = nxt - ml[k] * cur;
            }
          }
          double x2 = 0.0, x1 = cur * rlast, nrm = x1 * x1;
          x[n - 1] = x1;
          for (int k = n - 2; k >= 0; --k) {
            const double xk = (x[k] - u2[k] * x1 - u3[k] * x2) * r1[k];
            x[k] = xk;
            nrm += xk * xk;
            x2 = x1;
            x1 = xk;
          }
          double sc = 1.0 / sqrt(nrm);
          for (int k = 0; k < n; ++k) x[k] *= sc;
          if (sidx > 0) {
            for (int t2 = 0; t2 < sidx; ++t2) {
              const double* y = Z + (tid + t2) * n;
              double dot = 0.0;
              for (int k = 0; k < n; ++k) dot += x[k] * y[k];
              for (int k = 0; k < n; ++k) x[k] -= dot * y[k];
            }
            double n2 = 0.0;
            for (int k = 0; k < n; ++k) n2 += x[k] * x[k];
            sc = 1.0 / sqrt(n2);
            for (int k = 0; k < n; ++k) x[k] *= sc;
          }
        }
      }
    }
  }
  __syncthreads();
  // ---- 4. back-transform y = H_0 H_1 ... H_{n-2} z: each warp carries its vectors together
  {
    constexpr int VPW = (kMaxRR / 2 + NW - 1) / NW;   // vectors per warp (nb <= kMaxRR / 2)
    int cols[VPW];
    int nv = 0;
    for (int c = wp; c < nb && nv < VPW; c += NW) cols[nv++] = c;
    for (int q = 0; q < nv; ++q)
      for (int k = lane; k < n; k += 32) Ys[cols[q] * n + k] = make_double2(Z[cols[q] * n + k], 0.0);
    __syncwarp();
    for (int j = n - 2; j >= 0; --j) {
      const double2 tau = taus[j];
      if (tau.x == 0.0 && tau.y == 0.0) continue;
      double2 dot[VPW];
#pragma unroll
      for (int q = 0; q < VPW; ++q) dot[q] = make_double2(0, 0);
      for (int k = j + 1 + lane; k < n; k += 32) {
        const double2 v = A[k + j * n];
#pragma unroll
        for (int q = 0; q < VPW; ++q)
          if (q < nv) dot[q] = cadd(dot[q], cmulc(v, Ys[cols[q] * n + k]));
      }
#pragma unroll
      for (int q = 0; q < VPW; ++q) dot[q] = warp_sum2(dot[q]);
      for (int k = j + 1 + lane; k < n; k += 32) {
        const double2 v = A[k + j * n];
#pragma unroll
        for (int q = 0; q < VPW; ++q)
          if (q < nv) Ys[cols[q] * n + k] = csub(Ys[cols[q] * n + k], cmul(v, cmul(tau, dot[q])));
      }
      __syncwarp();
    }
    for (int q = 0; q < nv; ++q)
      for (int k = lane; k < n; k += 32) Yout[(long long)cols[q] * n + k] = Ys[cols[q] * n + k];
  }
  if (tid < nb) theta[tid] = lam[tid];
  if (tid == 0) *status = 0;
}

// out(:, j) = in(:, idx[j])
__global__ void k_gather_cols(const double2* in, long long N, const int* idx, double2* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int j = blockIdx.y;
  out[i + (long long)j * N] = in[i + (long long)idx[j] * N];
}

__global__ void k_diag(const double2* A, long long N, double* D) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < N) D[i] = A[i + i * N].x;
}

__global__ void k_unit_block(const int* idx, int nb, long long N, double2* X, int ldx) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N * nb) return;
  const long long row = i % N;
  const int v = (int)(i / N);
  X[row + (long long)v * ldx] = make_double2(row == idx[v] ? 1.0 : 0.0, 0.0);
}

// R = HX - X diag(theta); T = R / (D - theta) (guarded); per-column |R|^2 partials
__global__ void __launch_bounds__(256) k_resid_precond(const double2* X, const double2* HX, int ldx, int nb,
                                                       const double* theta, const double* D, long long N, double2* T,
                                                       int ldt, double* rpart) {
  __shared__ double red[8][64];
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const long long rr = blockIdx.x * (long long)blockDim.x + tid;
  for (int v = 0; v < nb; ++v) {
    double n2 = 0.0;
    if (rr < N) {
      const double th = theta[v];
      const double2 r = csub(HX[rr + (long long)v * ldx], cscale(X[rr + (long long)v * ldx], th));
      n2 = r.x * r.x + r.y * r.y;
      double den = D[rr] - th;
      if (fabs(den) < 0.05) den = copysign(0.05, den);   // clamp of the Davidson preconditioner (eV)
      T[rr + (long long)v * ldt] = cscale(r, 1.0 / den);
    }
    for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    if (lane == 0) red[wp][v] = n2;
  }
  __syncthreads();
  if (tid < nb) {
    double s = 0;
    for (int k = 0; k < 8; ++k) s += red[k][tid];
    rpart[(long long)blockIdx.x * 64 + tid] = s;
  }
}

// oscillators of the nev converged vectors: s_al = sum_j X_jn h_al(j) (no conjugate)
__global__ void __launch_bounds__(256) k_osc_part(const double2* X, int ldx, int nev, const double2* h, long long N,
                                                  double2* part) {
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const long long rows_per = (N + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * rows_per, r1 = min(N, r0 + rows_per);
  for (int pq = wp; pq < nev * NG; pq += 8) {
    const int n = pq % nev, al = pq / nev;
    double2 s = make_double2(0, 0);
    for (long long rr = r0 + lane; rr < r1; rr += 32) s = cadd(s, cmul(X[rr + (long long)n * ldx], h[al * N + rr]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
      s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
    }
    if (lane == 0) part[(long long)blockIdx.x * nev * NG + pq] = s;
  }
}

__global__ void k_osc_final(const double2* part, int nparts, int nev, int dtfull, int cpol, double* act) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nev) return;
  double2 s[NG];
  for (int al = 0; al < NG; ++al) {
    double2 t = make_double2(0, 0);
    for (int k = 0; k < nparts; ++k) t = cadd(t, part[(long long)k * nev * NG + al * nev + n]);
    s[al] = t;
  }
  act[0 * nev + n] = s[0].x * s[0].x + s[0].y * s[0].y;
  act[1 * nev + n] = s[1].x * s[1].x + s[1].y * s[1].y;
  act[2 * nev + n] = s[2].x * s[2].x + s[2].y * s[2].y;
  act[3 * nev + n] = dtfull ? s[0].x * s[1].x + s[0].y * s[1].y : 0.0;
  act[4 * nev + n] = dtfull ? s[0].x * s[2].x + s[0].y * s[2].y : 0.0;
  act[5 * nev + n] = dtfull ? s[1].x * s[2].x + s[1].y * s[2].y : 0.0;
  act[6 * nev + n] = cpol ? s[3].x * s[3].x + s[3].y * s[3].y : 0.0;
  act[7 * nev + n] = cpol ? s[4].x * s[4].x + s[4].y * s[4].y : 0.0;
}

}  // namespace

// ---------------------------------------------------------------------------------------
struct DavWork {
  double2 *V, *HV, *Xn, *HXn, *Yp, *small, *part;
  double *D, *theta, *rpart;
  int* istat;
};

static int hemm(wtbg_ctx* ctx, const double2* X, int ldx, int m, double2* Y, int ldy, double2* Yp) {
  if (ctx->fast_mode) return run_fastprod(ctx, X, ldx, m, Y, ldy);
  const long long N = ctx->N;
  const int nblk = (int)((N + TB - 1) / TB);
  dim3 grid(nblk, JCH);
  const size_t sm = sizeof(double2) * TB * HT + sizeof(double2) * TB * (m + 2);
  switch (m / 8) {
#define WTBG_HEMM_CASE(MV)                                                                       \
  case MV:                                                                                       \
    CK(cudaFuncSetAttribute(k_hemm<MV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
    k_hemm<MV><<<grid, 256, sm, ctx->stream>>>(ctx->H.as<double2>(), N, X, ldx, Yp);            \
    break;
    WTBG_HEMM_CASE(1) WTBG_HEMM_CASE(2) WTBG_HEMM_CASE(3) WTBG_HEMM_CASE(4) WTBG_HEMM_CASE(5)
#undef WTBG_HEMM_CASE
    default: return set_err(ctx, WTBG_ERR_UNSUPPORTED, "davidson: block size must be 8, 16, 24, 32 or 40");
  }
  if (m % 8) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "davidson: block size must be a multiple of 8");
  WTBG_COUNT(ctx, 1);
  const long long tot = N * m;
  k_sum_parts<<<(int)((tot + 255) / 256), 256, 0, ctx->stream>>>(Yp, N, m, Y, ldy); WTBG_COUNT(ctx, 1);
  CKL("hemm");
  return 0;
}

static int gram(wtbg_ctx* ctx, const double2* A, int lda, int p, const double2* B, int ldb, int q, double2* C,
                double2* part) {
  const long long N = ctx->N;
  if (p > 16 * GT || q > 16 * GT) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "davidson: gram too large");
  const int nparts = (int)std::min<long long>(296, (N + 63) / 64);
  const int t = (std::max(p, q) + 15) / 16;
  if (t <= 1)
    k_gram<1><<<nparts, 256, 0, ctx->stream>>>(A, lda, p, B, ldb, q, N, part);
  else if (t == 2)
    k_gram<2><<<nparts, 256, 0, ctx->stream>>>(A, lda, p, B, ldb, q, N, part);
  else if (t == 3)
    k_gram<3><<<nparts, 256, 0, ctx->stream>>>(A, lda, p, B, ldb, q, N, part);
  else if (t == 4)
    k_gram<4><<<nparts, 256, 0, ctx->stream>>>(A, lda, p, B, ldb, q, N, part);
  else
    k_gram<5><<<nparts, 256, 0, ctx->stream>>>(A, lda, p, B, ldb, q, N, part);
  WTBG_COUNT(ctx, 1);
  k_gram_sum<<<(p * q + 31) / 32, 256, 0, ctx->stream>>>(part, nparts, p * q, C); WTBG_COUNT(ctx, 1);
  CKL("gram");
  return 0;
}

static int tall(wtbg_ctx* ctx, const double2* A, int lda, int p, const double2* B, int q, double2* Cm, int ldc,
                bool sub) {
  const long long N = ctx->N;
  if (p > kMaxRR) return set_err(ctx, WTBG_ERR_UNSUPPORTED, "davidson: small matrix too large");
  const dim3 grid((unsigned)((N + 255) / 256), (unsigned)((q + 7) / 8));
  if (sub)
    k_tall_gemm<true><<<grid, 256, 0, ctx->stream>>>(A, lda, p, B, q, N, Cm, ldc);
  else
    k_tall_gemm<false><<<grid, 256, 0, ctx->stream>>>(A, lda, p, B, q, N, Cm, ldc);
  WTBG_COUNT(ctx, 1);
  CKL("tall");
  return 0;
}

// orthonormalise the q columns of T (ld N) in place: T <- T R^-1, twice (CholQR2)
static int cholqr2(wtbg_ctx* ctx, double2* T, int q, double2* tmp, DavWork& w) {
  const long long N = ctx->N;
  for (int pass = 0; pass < 2; ++pass) {
    if (int r = gram(ctx, T, (int)N, q, T, (int)N, q, w.small, w.part)) return r;
    const size_t csm = (size_t)2 * q * (q + 1) * 16;
    CK(cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm));
    k_chol_inv<<<1, 512, csm, ctx->stream>>>(w.small, q, w.small + 64 * 64, w.istat); WTBG_COUNT(ctx, 1);
    CKL("chol");
    if (int r = tall(ctx, T, (int)N, q, w.small + 64 * 64, q, tmp, (int)N, false)) return r;
    CK(cudaMemcpyAsync(T, tmp, (size_t)N * q * 16, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  return 0;
}

int run_davidson(wtbg_ctx* ctx, int nev, int nb, int largest, int max_iter, double tol, const double2* dX0, int dtfull,
                 int cpol, std::vector<double>& W, std::vector<double>& act, double2* dXout, int* iters, double* maxres) {
  const long long N = ctx->N;
  if (nb < nev || nb % 8 != 0 || nb > 40 || 2 * nb > kMaxRR)
    return set_err(ctx, WTBG_ERR_ARG, "davidson: block size must be a multiple of 8, >= nev and <= 40");
  const int n2 = 2 * nb;
  // workspace
  const size_t vbytes = (size_t)N * n2 * 16;
  ENSURE(ctx->ws, 2 * vbytes + 2 * (size_t)N * nb * 16 + (size_t)JCH * N * nb * 16 + 4096);
  char* base = ctx->ws.as<char>();
  DavWork w;
  w.V = reinterpret_cast<double2*>(base);
  w.HV = w.V + (size_t)N * n2;
  w.Xn = w.HV + (size_t)N * n2;
  w.HXn = w.Xn + (size_t)N * nb;
  w.Yp = w.HXn + (size_t)N * nb;
  ENSURE(ctx->tmp, (size_t)N * 8 + (size_t)kMaxRR * kMaxRR * 16 * 3 + 4096 * 16 + 300 * kMaxRR * kMaxRR * 16 + (size_t)N * 4 * 2 + 65536);
  char* tb = ctx->tmp.as<char>();
  w.D = reinterpret_cast<double*>(tb);
  w.small = reinterpret_cast<double2*>(tb + (size_t)N * 8);                     // M, Y, ...
  w.theta = reinterpret_cast<double*>(w.small + 3 * kMaxRR * kMaxRR);
  w.rpart = w.theta + kMaxRR;
  w.part = reinterpret_cast<double2*>(w.rpart + 4096);
  w.istat = reinterpret_cast<int*>(w.part + 300 * kMaxRR * kMaxRR);
  int* d_idx = w.istat + 16;
  cudaStream_t s = ctx->stream;
  const int th = 256;
  k_diag<<<(int)((N + th - 1) / th), th, 0, s>>>(ctx->H.as<double2>(), N, w.D); WTBG_COUNT(ctx, 1);
  CKL("k_diag");
  double2* X = w.V;          // first nb columns of V
  double2* T = w.V + (size_t)N * nb;
  double2* HX = w.HV;
  double2* HT = w.HV + (size_t)N * nb;
  // initial block
  if (dX0) {
    CK(cudaMemcpyAsync(X, dX0, (size_t)N * nb * 16, cudaMemcpyDeviceToDevice, s));
  } else {
    // unit vectors at the nb smallest (largest) diagonal entries
    std::vector<double> Dh(N);
    CK(cudaMemcpyAsync(Dh.data(), w.D, N * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::vector<int> idx(N);
    for (long long i = 0; i < N; ++i) idx[i] = (int)i;
    if (largest)
      std::partial_sort(idx.begin(), idx.begin() + nb, idx.end(), [&](int a, int b) { return Dh[a] > Dh[b] || (Dh[a] == Dh[b] && a < b); });
    else
      std::partial_sort(idx.begin(), idx.begin() + nb, idx.end(), [&](int a, int b) { return Dh[a] < Dh[b] || (Dh[a] == Dh[b] && a < b); });
    CK(cudaMemcpyAsync(d_idx, idx.data(), nb * 4, cudaMemcpyHostToDevice, s));
    k_unit_block<<<(int)((N * nb + th - 1) / th), th, 0, s>>>(d_idx, nb, N, X, (int)N); WTBG_COUNT(ctx, 1);
    CKL("k_unit_block");
  }
  if (int r = cholqr2(ctx, X, nb, w.Xn, w)) return r;
  if (int r = hemm(ctx, X, (int)N, nb, HX, (int)N, w.Yp)) return r;
  // first Rayleigh-Ritz on X alone
  const size_t rrsm = rr_smem_bytes(kMaxRR, kMaxRR / 2);
  CK(cudaFuncSetAttribute(k_rr_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rrsm));
  double2* Mm = w.small;
  double2* Y = w.small + kMaxRR * kMaxRR;
  auto rr = [&](const double2* Vb, const double2* HVb, int n) -> int {
    if (int r = gram(ctx, Vb, (int)N, n, HVb, (int)N, n, Mm, w.part)) return r;
    const size_t sm = rr_smem_bytes(n, nb);
    k_rr_tridiag<<<1, RR_THREADS, sm, s>>>(Mm, n, nb, largest, w.theta, Y, w.istat + 1); WTBG_COUNT(ctx, 1);
    CKL("k_rr_tridiag");
    // X = V Y(:, :nb), HX = HV Y(:, :nb)
    if (int r = tall(ctx, Vb, (int)N, n, Y, nb, w.Xn, (int)N, false)) return r;
    if (int r = tall(ctx, HVb, (int)N, n, Y, nb, w.HXn, (int)N, false)) return r;
    CK(cudaMemcpyAsync(X, w.Xn, (size_t)N * nb * 16, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(HX, w.HXn, (size_t)N * nb * 16, cudaMemcpyDeviceToDevice, s));
    return 0;
  };
  if (int r = rr(X, HX, nb)) return r;
  std::vector<double> res(nb), thh(nb);
  const int nrb = (int)((N + th - 1) / th);
  ENSURE(ctx->tmp2, (size_t)nrb * 64 * 8 + 64);
  double* rp = ctx->tmp2.as<double>();
  int it = 0;
  double worst = 0.0;
  // With the tensor-core product the residual stalls at its rounding level (FP32 accumulation,
  // ~1e-5 of |H x|): iterate with it down to kFastSwitch (or until it stops improving), then
  // refresh H X with the FP64 product and finish in FP64.
  struct FastGuard {
    wtbg_ctx* c;
    int saved;
    ~FastGuard() { c->fast_mode = saved; }
  } guard{ctx, ctx->fast_mode};
  constexpr double kFastSwitch = 4e-6, kFastStall = 5e-4;
  double lock_best = 1e300;
  int lock_stall = 0;
  bool lock_off = false;
  double best = 1e300;
  int since_best = 0;
  ctx->stats.dav_fast_iters = 0;
  ctx->stats.dav_fp64_iters = 0;
  for (; it < max_iter; ++it) {
    ++(ctx->fast_mode ? ctx->stats.dav_fast_iters : ctx->stats.dav_fp64_iters);
    k_resid_precond<<<nrb, th, 0, s>>>(X, HX, (int)N, nb, w.theta, w.D, N, T, (int)N, rp); WTBG_COUNT(ctx, 1);
    CKL("k_resid_precond");
    std::vector<double> rph((size_t)nrb * 64);
    CK(cudaMemcpyAsync(rph.data(), rp, rph.size() * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(thh.data(), w.theta, nb * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    worst = 0.0;
    for (int v = 0; v < nb; ++v) {
      double ss = 0;
      for (int b = 0; b < nrb; ++b) ss += rph[(size_t)b * 64 + v];
      res[v] = sqrt(ss);
      if (v < nev) worst = std::max(worst, res[v]);
    }
    if (worst < tol) break;
    if (ctx->fast_mode) {
      // the worst residual of a block is not monotone: stagnation counts only near the
      // product's rounding level (no halving of the best residual for 6 iterations)
      if (worst < 0.5 * best) {
        best = worst;
        since_best = 0;
      } else if (best < kFastStall) {
        ++since_best;
      }
      if (worst < std::max(kFastSwitch, tol) || since_best >= 6) {
        ctx->fast_mode = 0;
        if (int r = hemm(ctx, X, (int)N, nb, HX, (int)N, w.Yp)) return r;
        if (int r = rr(X, HX, nb)) return r;
        continue;
      }
    }
    // With the FP64 product (compute-bound, cost ~ block width) only the directions of the
    // largest residuals are expanded: a multiple of 8 covering every unconverged wanted state.
    // Only near convergence (worst < 1e-4 eV), and while the best residual keeps falling.
    int m_act = nb;
    const bool lock_zone = !ctx->fast_mode && worst < 1e-4;
    if (lock_zone) {
      if (worst < 0.5 * lock_best) {
        lock_best = worst;
        lock_stall = 0;
      } else if (++lock_stall >= 8) {
        lock_off = true;
      }
    }
    if (lock_zone && !lock_off) {
      int nun = 0;
      for (int v = 0; v < nev; ++v) nun += (res[v] >= tol);
      m_act = std::min(nb, std::max(16, (nun + 7) / 8 * 8));
      if (m_act < nb) {
        std::vector<int> ord(nb);
        for (int v = 0; v < nb; ++v) ord[v] = v;
        // unconverged wanted states first, then the rest, each by decreasing residual
        auto want = [&](int v) { return v < nev && res[v] >= tol; };
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
          if (want(a) != want(b)) return want(a);
          return res[a] > res[b];
        });
        CK(cudaMemcpyAsync(d_idx, ord.data(), m_act * 4, cudaMemcpyHostToDevice, s));
        k_gather_cols<<<dim3((unsigned)((N + 255) / 256), m_act), 256, 0, s>>>(T, N, d_idx, w.Xn);
        WTBG_COUNT(ctx, 1);
        CKL("k_gather_cols");
        CK(cudaMemcpyAsync(T, w.Xn, (size_t)N * m_act * 16, cudaMemcpyDeviceToDevice, s));
      }
    }
    // T <- T - X (X^H T), twice; orthonormalise
    for (int pass = 0; pass < 2; ++pass) {
      if (int r = gram(ctx, X, (int)N, nb, T, (int)N, m_act, w.small + 2 * kMaxRR * kMaxRR, w.part)) return r;
      if (int r = tall(ctx, X, (int)N, nb, w.small + 2 * kMaxRR * kMaxRR, m_act, T, (int)N, true)) return r;
    }
    if (int r = cholqr2(ctx, T, m_act, w.Xn, w)) return r;
    if (int r = hemm(ctx, T, (int)N, m_act, HT, (int)N, w.Yp)) return r;
    if (int r = rr(w.V, w.HV, nb + m_act)) return r;
  }
  if (iters) *iters = it;
  if (maxres) *maxres = worst;
  W.assign(thh.begin(), thh.begin() + nev);
  // oscillators
  act.assign((size_t)nev * 8, 0.0);
  if (ctx->have_velocity) {
    const int nparts = (int)std::min<long long>(296, (N + 255) / 256);
    k_osc_part<<<nparts, 256, 0, s>>>(X, (int)N, nev, ctx->h.as<double2>(), N, w.part); WTBG_COUNT(ctx, 1);
    double* dact = w.rpart;
    k_osc_final<<<(nev + 63) / 64, 64, 0, s>>>(w.part, nparts, nev, dtfull, cpol, dact); WTBG_COUNT(ctx, 1);
    CKL("oscillators");
    CK(cudaMemcpyAsync(act.data(), dact, (size_t)nev * 8 * 8, cudaMemcpyDeviceToHost, s));
  }
  if (dXout) CK(cudaMemcpyAsync(dXout, X, (size_t)N * nev * 16, cudaMemcpyDeviceToDevice, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int run_hemm_public(wtbg_ctx* ctx, const double2* X, int ldx, int m, double2* Y, int ldy, double2* Yp) {
  return hemm(ctx, X, ldx, m, Y, ldy, Yp);
}

// Y = H X for a narrow block (m = 8 or 16), reading the lower triangle once
int run_hemm_narrow(wtbg_ctx* ctx, const double2* X, int ldx, int m, double2* Y, int ldy) {
  if (ctx->fast_mode) return run_fastprod(ctx, X, ldx, m, Y, ldy);
  const long long N = ctx->N;
  const int nblk = (int)((N + TB - 1) / TB);
  ENSURE(ctx->slots, (size_t)nblk * nblk * TB * m * 16);
  double2* slots = ctx->slots.as<double2>();
  const size_t sm = sizeof(double2) * TB * (TB + 1) + 2 * sizeof(double2) * TB * (m + 1);
  dim3 grid(nblk, (nblk + LHS - 1) / LHS);
  if (m == 8) {
    CK(cudaFuncSetAttribute(k_hemm_lower<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_hemm_lower<1><<<grid, 256, sm, ctx->stream>>>(ctx->H.as<double2>(), N, X, ldx, nblk, slots);
  } else if (m == 16) {
    CK(cudaFuncSetAttribute(k_hemm_lower<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_hemm_lower<2><<<grid, 256, sm, ctx->stream>>>(ctx->H.as<double2>(), N, X, ldx, nblk, slots);
  } else {
    return set_err(ctx, WTBG_ERR_UNSUPPORTED, "hemm_narrow: m must be 8 or 16");
  }
  WTBG_COUNT(ctx, 1);
  const long long tot = (long long)nblk * TB * m;
  k_sum_slots<<<(int)((tot + 255) / 256), 256, 0, ctx->stream>>>(slots, N, nblk, m, Y, ldy); WTBG_COUNT(ctx, 1);
  CKL("hemm_narrow");
  return 0;
}
