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
//   (mma.sync m16n8k16 f64; Blackwell has no tcgen05 kind for f64).
// The oscillator sums need only A^T h = Z^T (Q^T h) (Z = eigenvectors of T), so the
// reflectors are also applied to the five h vectors as they are generated,
// g <- g - tau conj(v) (v^T g) -- the full O(N^3) eigenvector back-transform is never formed.
// All reductions are deterministic two-pass (no atomics).
#include <cfloat>

#include <cudaTypedefs.h>

#include "common.cuh"
#include "tc_sm100.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <string>

namespace {

constexpr int TB = WTBG_HEMV_TILE;   // 64
constexpr int NB = WTBG_PANEL;       // 32
constexpr int RB = 256;              // rows per block of k_wfix_last
constexpr int RA = 64;               // rows per block of k_colA / k_colC
constexpr int NG = 10;               // h vectors carried through (x, y, z, sp, sm [, each times f])

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

__device__ __forceinline__ double2 vload(const double2* p) {
  const volatile double* q = reinterpret_cast<const volatile double*>(p);
  return make_double2(q[0], q[1]);
}

// Per-column state shared by the column kernels (device memory).  Reductions across
// blocks use the "last block finishes" pattern: every block writes its partial, fences,
// and takes a ticket; the block that takes the last ticket reduces and resets the counter.
struct ColState {
  double2 tau;
  double2 scal;
  double2 alpha2;   // w(prev) += alpha2 * v(prev): applied by the next column kernel
  double beta;
  int trivial;
  unsigned int cntA, cntC, cntE;
  double2 z[2 * NB + NG];   // z1 = W^H v (p values), z2 = V^H v (p values), s = v^T g (ng)
};

__device__ __forceinline__ bool last_block(unsigned int* cnt) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int t = atomicAdd(cnt, 1u);
    s_last = (t == gridDim.x * gridDim.y - 1);
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// Programmatic dependent launch: every kernel of the column chain starts by waiting for its
// predecessor grid (all of its memory operations visible), then lets its own dependent grid
// be scheduled, so that launch latency and the CTA ramp of the next kernel overlap the tail of
// this one. Outside a programmatic launch both instructions are no-ops.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// (A) apply the previous column's w correction, update column i with the panel's pending
//     rank-2 terms, |x|^2 partials; the last block computes the reflector (ZLARFG).
//     RA rows per block; the four 64-thread groups split the panel columns q (mod 4), so that
//     each thread keeps few loads in flight and the grid covers the SMs at moderate N.
__global__ void __launch_bounds__(256) k_colA(double2* A, long long N, double2* Wp, int j0, int p, int i, double* part,
                                              ColState* st, double* d, double* e, double2* tau_out) {
  pdl_enter();
  __shared__ double2 wrow[NB], vrow[NB];
  __shared__ double2 sacc[4][RA];
  __shared__ double red[8];
  const int tid = threadIdx.x, el = tid & (RA - 1), grp = tid >> 6;
  const double2 alpha2 = (p > 0) ? st->alpha2 : make_double2(0, 0);
  if (tid < p) {
    double2 wv = Wp[i + (long long)tid * N];
    if (tid == p - 1) wv = cadd(wv, alpha2);   // v(prev)(i) = 1
    wrow[tid] = wv;
    vrow[tid] = A[i + (long long)(j0 + tid) * N];
  }
  __syncthreads();
  const long long r = (long long)i + (long long)blockIdx.x * RA + el;
  const bool rv = r < N;
  double2 wlast = make_double2(0, 0);
  double2 s = make_double2(0, 0);
  if (rv && p > 0) {
    // finish w of the previous column for this row
    const double2 vprev = A[r + (long long)(i - 1) * N];
    wlast = cadd(Wp[r + (long long)(p - 1) * N], cmul(alpha2, vprev));
#pragma unroll 4
    for (int q = grp; q < p; q += 4) {
      const double2 vq = A[r + (long long)(j0 + q) * N];
      const double2 wq = (q == p - 1) ? wlast : Wp[r + (long long)q * N];
      s = cadd(s, cadd(cmul(vq, cconj(wrow[q])), cmul(wq, cconj(vrow[q]))));
    }
  }
  sacc[grp][el] = s;
  __syncthreads();
  double nrm = 0.0;
  if (grp == 0 && rv) {
    if (p > 0) Wp[r + (long long)(p - 1) * N] = wlast;
    double2 a = A[r + (long long)i * N];
    a = csub(a, cadd(cadd(sacc[0][el], sacc[1][el]), cadd(sacc[2][el], sacc[3][el])));
    if (r == i) a.y = 0.0;
    A[r + (long long)i * N] = a;
    if (r >= (long long)i + 2) nrm = a.x * a.x + a.y * a.y;
  }
  nrm = warp_sum(nrm);
  if ((tid & 31) == 0) red[tid >> 5] = nrm;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += red[k];
    part[blockIdx.x] = t;
  }
  if (!last_block(&st->cntA)) return;
  // reflector scalars
  double t = 0.0;
  for (int k = tid; k < (int)gridDim.x; k += 256) t += ((volatile double*)part)[k];
  t = warp_sum(t);
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = t;
  __syncthreads();
  if (tid == 0) {
    double xn2 = 0.0;
    for (int k = 0; k < 8; ++k) xn2 += red[k];
    const double2 alpha = vload(A + (i + 1) + (long long)i * N);
    if (xn2 == 0.0 && alpha.y == 0.0) {
      st->tau = make_double2(0, 0);
      st->scal = make_double2(0, 0);
      st->beta = alpha.x;
      st->trivial = 1;
    } else {
      const double beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x);
      st->tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
      const double2 den = make_double2(alpha.x - beta, alpha.y);
      const double dd = den.x * den.x + den.y * den.y;
      st->scal = make_double2(den.x / dd, -den.y / dd);
      st->beta = beta;
      st->trivial = 0;
    }
    e[i] = st->beta;
    d[i] = vload(A + i + (long long)i * N).x;
    tau_out[i] = st->tau;
    st->cntA = 0;
  }
}

// (C) scale v in place (v(i+1) = 1); partial dots z1 = W^H v, z2 = V^H v, s = v^T g over the
//     block's RA rows, one warp per dot (two rows per lane); the last block reduces the
//     partials into st->z, again one warp per dot with the lanes striding over the blocks.
__global__ void __launch_bounds__(256) k_colC(double2* A, long long N, const double2* Wp, int j0, int p, int i,
                                              ColState* st, const double2* g, int ng, double2* part) {
  pdl_enter();
  __shared__ double2 vs[RA];
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const long long rbase = (long long)i + 1 + (long long)blockIdx.x * RA;
  if (tid < RA) {
    const long long r = rbase + tid;
    double2 v = make_double2(0, 0);
    if (r < N) {
      if (r == i + 1) v = make_double2(1.0, 0.0);
      else v = st->trivial ? make_double2(0, 0) : cmul(A[r + (long long)i * N], st->scal);
      A[r + (long long)i * N] = v;
    }
    vs[tid] = v;
  }
  __syncthreads();
  const int nval = 2 * p + ng;
  const long long r0 = rbase + lane, r1 = r0 + 32;
  const bool ok0 = r0 < N, ok1 = r1 < N;
  const double2 x0 = vs[lane], x1 = vs[lane + 32];
  for (int q = wp; q < nval; q += 8) {
    double2 t;
    if (q < 2 * p) {
      const double2* col = (q < p) ? Wp + (long long)q * N : A + (long long)(j0 + q - p) * N;
      const double2 a0 = ok0 ? col[r0] : make_double2(0, 0);
      const double2 a1 = ok1 ? col[r1] : make_double2(0, 0);
      t = cadd(cmulc(a0, x0), cmulc(a1, x1));
    } else {
      const double2* col = g + (long long)(q - 2 * p) * N;
      const double2 a0 = ok0 ? col[r0] : make_double2(0, 0);
      const double2 a1 = ok1 ? col[r1] : make_double2(0, 0);
      t = cadd(cmul(x0, a0), cmul(x1, a1));
    }
    t = warp_sum2(t);
    if (lane == 0) part[(long long)blockIdx.x * (2 * NB + NG) + q] = t;
  }
  if (!last_block(&st->cntC)) return;
  for (int q = wp; q < nval; q += 8) {
    double2 s = make_double2(0, 0);
    for (int k = lane; k < (int)gridDim.x; k += 32) s = cadd(s, vload(part + (long long)k * (2 * NB + NG) + q));
    s = warp_sum2(s);
    if (lane == 0) st->z[q] = s;
  }
  __syncthreads();
  if (tid == 0) st->cntC = 0;
}

// (D) y = A22 v, A22 = rows/cols [i+1, N) of the lower-stored Hermitian matrix.
// Work item = a chunk of up to hs 64x64 tiles down one block-column J. The row sums A_IJ x_J
// go to slot[I][J] per tile; the column sums A_IJ^H x_I stay in registers across the chunk and
// go to slot[J][I0] (I0 = first tile of the chunk, I0 = J + y*hs), so that
// y_a = sum of slot[a][b] over b0 <= b <= a and over b = a + hs, a + 2 hs, ... < nblk.
// Persistent: one CTA per SM walks its items round-robin; thread 0 keeps HV_STAGES tiles in
// flight through TMA (one 64 KB box of 64 columns x 64 rows per tile, column-major as stored,
// zero fill past N) into a shared-memory ring, across item boundaries, so that the HBM stream
// does not drain between chunks. Every wait is bounded; a timed-out wait sets *err after the
// CTA's own copies in flight have landed.
constexpr int HV_STAGES = 3;
constexpr uint32_t HV_TILE_BYTES = TB * TB * 16;
constexpr size_t HV_SMEM = (size_t)HV_STAGES * HV_TILE_BYTES + 1024;

__global__ void __launch_bounds__(256, 1) k_hemv(const __grid_constant__ CUtensorMap tm, const double2* __restrict__ A,
                                                 long long N, int i, int nblk, int hs, double2* __restrict__ slots,
                                                 int* err) {
  pdl_enter();
  extern __shared__ unsigned char hv_raw[];
  __shared__ double2 xJs[TB];
  __shared__ double2 rowp[2][8][TB];
  __shared__ double2 diagrow[TB];
  __shared__ double2 colp[TB];
  __shared__ __align__(8) uint64_t full[HV_STAGES];
  __shared__ int s_flag;
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const uint32_t raw = tc::smem_u32(hv_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  const double2* tiles = reinterpret_cast<const double2*>(hv_raw + (base - raw));
  const int b0 = (i + 1) / TB, nt = nblk - b0;
  const int nyc = (nt + hs - 1) / hs;
  const long long nitems = (long long)nt * nyc, stride = gridDim.x;
  const long long lo = (long long)i + 1;
  const double2* xcol = A + (long long)i * N;
  if (tid == 0) {
    for (int s = 0; s < HV_STAGES; ++s) tc::mbar_init(tc::smem_u32(&full[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_flag = 0;
  }
  __syncthreads();

  // producer state (thread 0): the same item/tile sequence as the consumers
  long long p_it = (long long)blockIdx.x - stride;
  int p_I = 0, p_I1 = 0, p_J = 0, issued = 0;
  auto p_next = [&]() -> bool {
    while (p_I >= p_I1) {
      p_it += stride;
      if (p_it >= nitems) return false;
      const int jj = (int)(p_it % nt), y = (int)(p_it / nt);
      p_J = b0 + jj;
      p_I = p_J + y * hs;
      p_I1 = min(p_I + hs, nblk);
    }
    return true;
  };
  auto issue = [&]() {
    const int s = issued % HV_STAGES;
    const uint32_t bar = tc::smem_u32(&full[s]);
    tc::mbar_expect_tx(bar, HV_TILE_BYTES);
    tc::tma_load_2d(base + (uint32_t)s * HV_TILE_BYTES, &tm, p_I * TB * 2, p_J * TB, bar);
    ++p_I;
    ++issued;
  };
  if (tid == 0)
    for (int s = 0; s < HV_STAGES && p_next(); ++s) issue();

  int t = 0;
  bool aborted = false;
  for (long long it = blockIdx.x; it < nitems && !aborted; it += stride) {
    const int jj = (int)(it % nt), y = (int)(it / nt);
    const int J = b0 + jj, I0 = J + y * hs;
    if (I0 >= nblk) continue;
    const int I1 = min(I0 + hs, nblk);
    const long long C0 = (long long)J * TB;
    __syncthreads();   // the previous item's readers of xJs and colp are done
    if (tid < TB) {
      const long long c = C0 + tid;
      xJs[tid] = (c >= lo && c < N) ? xcol[c] : make_double2(0, 0);
    }
    __syncthreads();
    double2 cacc[8];
    bool cvalid[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      cacc[m] = make_double2(0, 0);
      const long long c = C0 + wp + 8 * m;
      cvalid[m] = (c >= lo && c < N);
    }
    const bool interior_cols = (C0 >= lo && C0 + TB <= N);
    // x rows of the next tile are loaded one tile ahead
    double2 xa_n, xb_n;
    {
      const long long ra = (long long)I0 * TB + lane, rb = ra + 32;
      xa_n = (ra >= lo && ra < N) ? xcol[ra] : make_double2(0, 0);
      xb_n = (rb >= lo && rb < N) ? xcol[rb] : make_double2(0, 0);
    }
    for (int I = I0; I < I1; ++I, ++t) {
      const double2 xa = xa_n, xb = xb_n;
      if (I + 1 < I1) {
        const long long ra = (long long)(I + 1) * TB + lane, rb = ra + 32;
        xa_n = (ra >= lo && ra < N) ? xcol[ra] : make_double2(0, 0);
        xb_n = (rb >= lo && rb < N) ? xcol[rb] : make_double2(0, 0);
      }
      const int s = t % HV_STAGES;
      const bool ok = tc::mbar_wait(tc::smem_u32(&full[s]), (uint32_t)((t / HV_STAGES) & 1), &s_flag, false);
      const double2* T = tiles + (size_t)s * TB * TB;   // T[c * 64 + r]
      const int buf = (I - I0) & 1;
      const long long R0 = (long long)I * TB;
      const long long ra = R0 + lane, rb = ra + 32;
      const bool diag = (I == J);
      const bool va = (ra >= lo && ra < N), vb = (rb >= lo && rb < N);
      double2 rp0 = make_double2(0, 0), rp1 = make_double2(0, 0);
      if (interior_cols && !diag && R0 >= lo && R0 + TB <= N) {
        // interior tile: every element is in the trailing matrix, no masks
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          const int cl = wp + 8 * m;
          const double2 e0 = T[cl * TB + lane], e1 = T[cl * TB + lane + 32];
          const double2 xj = xJs[cl];
          rp0 = cadd(rp0, cmul(e0, xj));
          rp1 = cadd(rp1, cmul(e1, xj));
          cacc[m] = cadd(cacc[m], cadd(cmulc(e0, xa), cmulc(e1, xb)));
        }
      } else
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const int cl = wp + 8 * m;
        const bool ok0 = cvalid[m] && va && (!diag || lane >= cl);
        const bool ok1 = cvalid[m] && vb && (!diag || lane + 32 >= cl);
        double2 e0 = ok0 ? T[cl * TB + lane] : make_double2(0, 0);
        double2 e1 = ok1 ? T[cl * TB + lane + 32] : make_double2(0, 0);
        const double2 xj = xJs[cl];
        const bool d0 = diag && (lane == cl), d1 = diag && (lane + 32 == cl);
        if (d0) e0.y = 0.0;
        if (d1) e1.y = 0.0;
        rp0 = cadd(rp0, cmul(e0, xj));
        rp1 = cadd(rp1, cmul(e1, xj));
        if (!d0) cacc[m] = cadd(cacc[m], cmulc(e0, xa));
        if (!d1) cacc[m] = cadd(cacc[m], cmulc(e1, xb));
      }
      rowp[buf][wp][lane] = rp0;
      rowp[buf][wp][lane + 32] = rp1;
      if (__syncthreads_or(!ok)) {   // every thread has left stage s (and agrees on failure)
        aborted = true;
        break;
      }
      if (tid == 0 && p_next()) issue();
      if (tid < TB) {
        double2 sm = make_double2(0, 0);
#pragma unroll
        for (int k = 0; k < 8; ++k) sm = cadd(sm, rowp[buf][k][tid]);
        if (diag) diagrow[tid] = sm;
        else slots[((long long)I * nblk + J) * TB + tid] = sm;
      }
    }
    if (aborted) break;
    // column sums of the chunk
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const double2 sm = warp_sum2(cacc[m]);
      if (lane == m) colp[wp + 8 * m] = sm;
    }
    __syncthreads();
    if (tid < TB) {
      double2 v = colp[tid];
      if (I0 == J) v = cadd(v, diagrow[tid]);
      slots[((long long)J * nblk + I0) * TB + tid] = v;
    }
  }
  if (aborted && tid == 0) {
    // let this CTA's copies in flight land before the shared memory is released
    for (int u = t; u < issued; ++u)
      tc::mbar_wait(tc::smem_u32(&full[u % HV_STAGES]), (uint32_t)((u / HV_STAGES) & 1), &s_flag, false);
    atomicExch(err, 1);
  }
}

// (E) y rows from the slots; w = tau (y - V z1 - W z2); g <- g - tau conj(v) s; partial
//     w^H v.  The last block computes alpha2 = -tau/2 w^H v for the next column kernel.
__global__ void __launch_bounds__(256) k_colE(const double2* A, long long N, double2* Wp, int j0, int p, int i, int nblk,
                                              int hs, const double2* slots, ColState* st, double2* g, int ng,
                                              double2* part) {
  pdl_enter();
  __shared__ double2 acc4[4][TB];
  __shared__ double2 tq4[4][TB];
  __shared__ double2 zz[2 * NB + NG];
  __shared__ double2 red[8];
  const int tid = threadIdx.x;
  const int nval = 2 * p + ng;
  for (int q = tid; q < nval; q += blockDim.x) zz[q] = st->z[q];
  const double2 tau = st->tau;
  const int b0 = (i + 1) / TB;
  const int a = b0 + blockIdx.x;
  const int el = tid & (TB - 1), grp = tid >> 6;
  // slots of row block a: the tile row sums b0 <= b <= a, then the chunk column sums at
  // b = a + hs, a + 2 hs, ... (the only slots the mat-vec writes above the diagonal)
  const int n1 = a - b0 + 1, n2 = (nblk - 1 - a) / hs;
  double2 s = make_double2(0, 0);
#pragma unroll 4
  for (int u = grp; u < n1 + n2; u += 4) {
    const int b = (u < n1) ? b0 + u : a + hs * (u - n1 + 1);
    s = cadd(s, slots[((long long)a * nblk + b) * TB + el]);
  }
  acc4[grp][el] = s;
  __syncthreads();
  const long long r = (long long)a * TB + el;
  const bool rv = (r >= (long long)i + 1 && r < N);
  // V z1 + W z2 for this row, the q range split over the 4 thread groups
  double2 t = make_double2(0, 0);
  if (rv) {
    for (int q = grp; q < p; q += 4) {
      t = cadd(t, cmul(A[r + (long long)(j0 + q) * N], zz[q]));
      t = cadd(t, cmul(Wp[r + (long long)q * N], zz[p + q]));
    }
  }
  tq4[grp][el] = t;
  __syncthreads();
  double2 dot = make_double2(0, 0);
  if (tid < TB && rv) {
    const double2 y = cadd(cadd(acc4[0][tid], acc4[1][tid]), cadd(acc4[2][tid], acc4[3][tid]));
    const double2 vz = cadd(cadd(tq4[0][tid], tq4[1][tid]), cadd(tq4[2][tid], tq4[3][tid]));
    const double2 w = cmul(tau, csub(y, vz));
    Wp[r + (long long)p * N] = w;
    const double2 v = A[r + (long long)i * N];
    dot = cmulc(w, v);
    const double2 tv = cmul(tau, cconj(v));
    for (int al = 0; al < ng; ++al) {
      const double2 sa = zz[2 * p + al];
      g[(long long)al * N + r] = csub(g[(long long)al * N + r], cmul(tv, sa));
    }
  }
  if (tid < 64) {
    dot = warp_sum2(dot);
    if ((tid & 31) == 0) red[tid >> 5] = dot;
  }
  __syncthreads();
  if (tid == 0) part[blockIdx.x] = cadd(red[0], red[1]);
  if (!last_block(&st->cntE)) return;
  double2 sum = make_double2(0, 0);
  for (int k = tid; k < (int)gridDim.x; k += 256) sum = cadd(sum, vload(part + k));
  sum = warp_sum2(sum);
  if ((tid & 31) == 0) red[tid >> 5] = sum;
  __syncthreads();
  if (tid == 0) {
    double2 tot = make_double2(0, 0);
    for (int k = 0; k < 8; ++k) tot = cadd(tot, red[k]);
    st->alpha2 = cscale(cmul(tau, tot), -0.5);
    st->cntE = 0;
  }
}

// w(last column of the panel) += alpha2 v, rows [k0, N), before the trailing update
__global__ void __launch_bounds__(RB) k_wfix_last(const double2* A, long long N, double2* Wp, int p, int i, long long k0,
                                                  const ColState* st) {
  pdl_enter();
  const long long r = k0 + (long long)blockIdx.x * RB + threadIdx.x;
  if (r >= N) return;
  const double2 alpha2 = st->alpha2;
  Wp[r + (long long)p * N] = cadd(Wp[r + (long long)p * N], cmul(alpha2, A[r + (long long)i * N]));
}

// Trailing update A22 -= V W^H + W V^H on the lower triangle with FP64 mma.sync.
// Real form: C_re -= Vr Wr^T + Vi Wi^T + Wr Vr^T + Wi Vi^T
//            C_im -= Vi Wr^T - Vr Wi^T + Wi Vr^T - Wr Vi^T
// One CTA per 64x64 tile of the lower triangle. The panel columns arrive in chunks of HK
// through a two-stage cp.async ring (the next chunk loads while the current one multiplies),
// and the tile of A itself is prefetched into L2 at the start so that the read-modify-write
// epilogue does not wait on HBM.  Each staged operand is k-major, [q][row] with row stride
// HLD = 66: the copying lanes step along the rows (consecutive 16-byte slots) and a fragment
// load's 8-lane phase (rows r, r+1 at k .. k+3) falls on 8 distinct bank groups.
constexpr int HK = 8;         // q-chunk staged per step
constexpr int HLD = TB + 2;   // row stride of a staged [q][row] operand
constexpr int HSTAGE = 4 * HK * HLD;   // double2 per stage (Vr, Wr, Vc, Wc)
constexpr size_t HER2K_SMEM = 2 * (size_t)HSTAGE * sizeof(double2);

// D += A B with A 16x16 (k = tq + 4*(i/2) for a_i, row gq + 8*(i%2)) and B 16x8 (k = tq + 4*j for
// b_j, column gq): the four real products of one complex accumulator concatenated along k.
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]), "d"(b[1]),
        "d"(b[2]), "d"(b[3]));
}

// 16-byte asynchronous copy global -> shared; zero fill (no global read) when !valid
__device__ __forceinline__ void cp_async16(double2* dst, const double2* src, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N_>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N_) : "memory"); }

// V (row, q) = Vs[row + (vc0 + q) * N]: the panel columns of A in the one-stage reduction, the
// dense V of the two-stage panel otherwise.
__global__ void __launch_bounds__(256, 2) k_her2k(double2* A, long long N, const double2* Wp, const double2* Vs,
                                                  int vc0, int jb, int k0) {
  pdl_enter();
  extern __shared__ __align__(16) double2 hsm[];
  const long long t = blockIdx.x;
  int bi = (int)floor((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((long long)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((long long)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (long long)bi * (bi + 1) / 2);
  const long long r0 = (long long)k0 + (long long)bi * TB, c0 = (long long)k0 + (long long)bj * TB;
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const int wr = wp & 3, wc = wp >> 2;
  const int gq = lane >> 2, tq = lane & 3;

  // L2 prefetch of this thread's epilogue elements
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int k = 0; k < 4; k += 2) {
      const long long row = r0 + wr * 16 + gq + ((k >> 1) ? 8 : 0);
      const long long col = c0 + wc * 32 + n * 8 + 2 * tq;
      if (row < N && col < N && row >= col) asm volatile("prefetch.global.L2 [%0];" ::"l"(A + row + col * N));
    }

  auto stage = [&](int c, int buf) {
    double2* sVr = hsm + (size_t)buf * HSTAGE;
    double2* sWr = sVr + HK * HLD;
    double2* sVc = sWr + HK * HLD;
    double2* sWc = sVc + HK * HLD;
    const int qc = c * HK;
    for (int it = tid; it < TB * HK; it += 256) {
      const int rr = it % TB, q = it / TB;
      const long long rg = r0 + rr, cg = c0 + rr;
      const bool qv = (qc + q) < jb;
      const long long qcol = (long long)(vc0 + qc + q);
      const bool vr = qv && rg < N, vc = qv && cg < N;
      cp_async16(sVr + q * HLD + rr, vr ? Vs + rg + qcol * N : Vs, vr);
      cp_async16(sWr + q * HLD + rr, vr ? Wp + rg + (long long)(qc + q) * N : Wp, vr);
      cp_async16(sVc + q * HLD + rr, vc ? Vs + cg + qcol * N : Vs, vc);
      cp_async16(sWc + q * HLD + rr, vc ? Wp + cg + (long long)(qc + q) * N : Wp, vc);
    }
    cp_async_commit();
  };

  double accr[4][4], acci[4][4];
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int k = 0; k < 4; ++k) accr[n][k] = acci[n][k] = 0.0;

  const int nch = (jb + HK - 1) / HK;
  stage(0, 0);
  if (nch > 1) stage(1, 1);
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) cp_async_wait<1>();
    else cp_async_wait<0>();
    __syncthreads();
    const double2* sVr = hsm + (size_t)(c & 1) * HSTAGE;
    const double2* sWr = sVr + HK * HLD;
    const double2* sVc = sWr + HK * HLD;
    const double2* sWc = sVc + HK * HLD;
#pragma unroll
    for (int kk = 0; kk < HK; kk += 4) {
      const int row = wr * 16 + gq;
      const double2 v0 = sVr[(kk + tq) * HLD + row], v1 = sVr[(kk + tq) * HLD + row + 8];
      const double2 w0 = sWr[(kk + tq) * HLD + row], w1 = sWr[(kk + tq) * HLD + row + 8];
      // k segments: [Vr | Vi | Wr | Wi] (re) and [Vi | -Vr | Wi | -Wr] (im) against [Wr; Wi; Vr; Vi]
      const double are[8] = {v0.x, v1.x, v0.y, v1.y, w0.x, w1.x, w0.y, w1.y};
      const double aim[8] = {v0.y, v1.y, -v0.x, -v1.x, w0.y, w1.y, -w0.x, -w1.x};
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const int col = wc * 32 + n * 8 + gq;
        const double2 bw = sWc[(kk + tq) * HLD + col], bv = sVc[(kk + tq) * HLD + col];
        const double b[4] = {bw.x, bw.y, bv.x, bv.y};
        dmma16(accr[n], are, b);
        dmma16(acci[n], aim, b);
      }
    }
    __syncthreads();
    if (c + 2 < nch) stage(c + 2, c & 1);
  }
  // epilogue per column block n: its four loads are issued before its stores, so a thread
  // waits for one round trip per block instead of one per element
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    double2 a[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const long long row = r0 + wr * 16 + gq + ((k >> 1) ? 8 : 0);
      const long long col = c0 + wc * 32 + n * 8 + 2 * tq + (k & 1);
      a[k] = (row < N && col < N && row >= col) ? __ldcg(A + row + col * N) : make_double2(0, 0);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const long long row = r0 + wr * 16 + gq + ((k >> 1) ? 8 : 0);
      const long long col = c0 + wc * 32 + n * 8 + 2 * tq + (k & 1);
      if (row < N && col < N && row >= col) {
        double2 v = a[k];
        v.x -= accr[n][k];
        v.y = (row == col) ? 0.0 : v.y - acci[n][k];
        A[row + col * N] = v;
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

namespace {

// launch with programmatic stream serialisation (see pdl_enter)
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

cudaError_t launch_hemv(wtbg_ctx* ctx, int hs, int nt, cudaStream_t s, const double2* A, long long N, int i, int nblk,
                        double2* slots) {
  const long long nitems = (long long)nt * ((nt + hs - 1) / hs);
  const int grid = (int)std::min<long long>(nitems, ctx->nsm);
  return launch_pdl(k_hemv, dim3(grid), dim3(256), HV_SMEM, s, *reinterpret_cast<const CUtensorMap*>(ctx->tmH), A, N,
                    i, nblk, hs, slots, ctx->triErr.as<int>());
}

PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
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

}  // namespace

// TMA map of the BSE matrix for the mat-vec: FP64 view of the column-major complex array,
// dims (2N doubles, N columns), box (128 doubles = 64 rows, 64 columns); kept while H and N
// stay the same. Also sizes the error flag and reads the SM count.
int prepare_hemv(wtbg_ctx* ctx) {
  const long long N = ctx->N;
  ENSURE(ctx->triErr, 16);
  if (ctx->nsm <= 0) CK(cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, ctx->device));
  CK(cudaFuncSetAttribute(k_hemv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HV_SMEM));
  if (ctx->tmH_ptr == ctx->H.p && ctx->tmH_n == N) return 0;
  auto fn = tma_encoder();
  if (!fn) return set_err(ctx, WTBG_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t dims[2] = {(cuuint64_t)(2 * N), (cuuint64_t)N};
  cuuint64_t strides[1] = {(cuuint64_t)N * 16};
  cuuint32_t box[2] = {(cuuint32_t)(2 * TB), (cuuint32_t)TB};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(reinterpret_cast<CUtensorMap*>(ctx->tmH), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, ctx->H.p, dims, strides,
                  box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_err(ctx, WTBG_ERR_CUDA, "cuTensorMapEncodeTiled(H) failed: " + std::to_string((int)r));
  ctx->tmH_ptr = ctx->H.p;
  ctx->tmH_n = N;
  return 0;
}

// Autotuner for the mat-vec chunk (tiles per CTA, 4 / 8 / 16): times each variant on the
// column N/4 (three launches each, CUDA events; the launches only write the slot partials,
// which the reduction overwrites) and keeps the fastest per (device, N).
int autotune_hemv(wtbg_ctx* ctx, int* hs_out) {
  static std::mutex mu;
  static std::map<std::pair<int, long long>, int> cache;
  const long long N = ctx->N;
  const std::pair<int, long long> key(ctx->device, N);
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      *hs_out = it->second;
      return 0;
    }
  }
  const int nblk = (int)((N + TB - 1) / TB);
  *hs_out = 8;
  if (N < 4 * TB) return 0;
  ENSURE(ctx->slots, (size_t)nblk * nblk * TB * 16);
  if (int r = prepare_hemv(ctx)) return r;
  if (int r = ensure_events(ctx, 2)) return r;
  const int i = (int)(N / 4);
  const int nt = nblk - (i + 1) / TB;
  const int cand[3] = {4, 8, 16};
  float best = 1e30f;
  for (int c : cand) {
    float tot = 0.f;
    for (int rep = 0; rep < 4; ++rep) {
      CK(cudaEventRecord(ctx->evpool[0], ctx->stream));
      CK(launch_hemv(ctx, c, nt, ctx->stream, ctx->H.as<double2>(), N, i, nblk, ctx->slots.as<double2>()));
      CK(cudaEventRecord(ctx->evpool[1], ctx->stream));
      CK(cudaEventSynchronize(ctx->evpool[1]));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ctx->evpool[0], ctx->evpool[1]));
      if (rep > 0) tot += ms;   // the first launch warms up
    }
    WTBG_COUNT(ctx, 4);
    if (tot < best) {
      best = tot;
      *hs_out = c;
    }
  }
  CKL("autotune_hemv");
  std::lock_guard<std::mutex> g(mu);
  cache[key] = *hs_out;
  return 0;
}

// Trailing update of the two-stage panel: A22 -= V W^H + W V^H with V (row, q) = V[row + (vc0 + q) vld]
int launch_her2k_v(wtbg_ctx* ctx, double2* A, long long N, const double2* Wp, const double2* V, long long vld, int vc0,
                   int jb, long long k0) {
  if (vld != N) return set_err(ctx, WTBG_ERR_ARG, "her2k: V must have leading dimension N");
  CK(cudaFuncSetAttribute(k_her2k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HER2K_SMEM));
  const long long T = (N - k0 + TB - 1) / TB;
  const long long ntile = T * (T + 1) / 2;
  CK(launch_pdl(k_her2k, dim3((unsigned)ntile), dim3(256), HER2K_SMEM, ctx->stream, A, N, Wp, V, vc0, jb, (int)k0));
  WTBG_COUNT(ctx, 1);
  return 0;
}

bool use_two_stage(wtbg_ctx* ctx);
int run_tridiagonalise2(wtbg_ctx* ctx);
static int run_tridiagonalise1(wtbg_ctx* ctx);

// Reduction of the current matrix to tridiagonal form: two-stage (tridiag2.cu) where it is
// selected and fits, else the one-stage column loop below.
int run_tridiagonalise(wtbg_ctx* ctx) {
  if (ctx->N < 2) return set_err(ctx, WTBG_ERR_ARG, "tridiagonalise: N < 2");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(ctx->stream, &cap));
  if (cap == cudaStreamCaptureStatusNone && use_two_stage(ctx)) return run_tridiagonalise2(ctx);
  return run_tridiagonalise1(ctx);
}

static int run_tridiagonalise1(wtbg_ctx* ctx) {
  const long long N = ctx->N;
  ctx->tri_two = false;
  const int nblk = (int)((N + TB - 1) / TB);
  const int maxRB = (int)((N + RA - 1) / RA) + 1;   // blocks of k_colA / k_colC
  ENSURE(ctx->d, (size_t)N * 8);
  ENSURE(ctx->e, (size_t)N * 8);
  ENSURE(ctx->tau, (size_t)N * 16);
  ENSURE(ctx->g, (size_t)N * 16 * NG);
  ENSURE(ctx->Wp, (size_t)N * 16 * NB);
  ENSURE(ctx->slots, (size_t)nblk * nblk * TB * 16);
  ENSURE(ctx->part, (size_t)maxRB * (2 * NB + NG) * 16 + (size_t)maxRB * 16 + (size_t)(nblk + 1) * 16 + 4096);
  ENSURE(ctx->scal, sizeof(ColState) + 64);
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
  ColState* st = ctx->scal.as<ColState>();
  cudaStream_t s = ctx->stream;
  int hs = 8;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(s, &cap));
  if (cap == cudaStreamCaptureStatusNone) {
    CK(cudaFuncSetAttribute(k_her2k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HER2K_SMEM));
    if (int r = prepare_hemv(ctx)) return r;
    if (int r = autotune_hemv(ctx, &hs)) return r;
  } else {
    hs = ctx->hemv_hs > 0 ? ctx->hemv_hs : 8;   // chosen before the capture
  }
  ctx->hemv_hs = hs;
  CK(cudaMemsetAsync(st, 0, sizeof(ColState), s));
  CK(cudaMemsetAsync(ctx->triErr.p, 0, 4, s));

  const int ng = (ctx->have_velocity && ctx->temp_on) ? 10 : 5;
  ctx->ng = ng;
  if (ctx->have_velocity && ctx->temp_on) {
    if (int r = fill_g_vectors(ctx, g)) return r;
  } else if (ctx->have_velocity) {
    k_copy_g<<<(int)((N * 5 + 255) / 256), 256, 0, s>>>(ctx->h.as<double2>(), g, N * 5); WTBG_COUNT(ctx, 1);
  } else {
    CK(cudaMemsetAsync(g, 0, (size_t)N * 16 * 5, s));
  }
  CKL("k_copy_g");
  const bool prof = ctx->profiling != 0;
  const size_t npanel = (size_t)((N - 1 + NB - 1) / NB);
  const size_t evh = 2 * (size_t)N;            // her2k event pairs follow the mat-vec ones
  const size_t evt = evh + 2 * npanel;         // then the pair around the whole reduction
  if (prof) {
    if (int r = ensure_events(ctx, evt + 2)) return r;
    cudaEventRecord(ctx->evpool[evt], s);
  }

  for (long long j0 = 0; j0 < N - 1; j0 += NB) {
    const int jb = (int)((N - 1 - j0) < NB ? (N - 1 - j0) : NB);
    for (int p = 0; p < jb; ++p) {
      const int i = (int)(j0 + p);
      const int nA = (int)((N - i + RA - 1) / RA);
      CK(launch_pdl(k_colA, dim3(nA), dim3(256), 0, s, A, N, Wp, (int)j0, p, i, partA, st, d, e, tau)); WTBG_COUNT(ctx, 1);
      const int nC = (int)((N - i - 1 + RA - 1) / RA);
      CK(launch_pdl(k_colC, dim3(nC), dim3(256), 0, s, A, N, (const double2*)Wp, (int)j0, p, i, st, (const double2*)g, ng,
                    partC)); WTBG_COUNT(ctx, 1);
      const int b0 = (i + 1) / TB;
      const int nt = nblk - b0;
      if (prof) cudaEventRecord(ctx->evpool[2 * i], s);
      CK(launch_hemv(ctx, hs, nt, s, A, N, i, nblk, slots)); WTBG_COUNT(ctx, 1);
      if (prof) cudaEventRecord(ctx->evpool[2 * i + 1], s);
      CK(launch_pdl(k_colE, dim3(nt), dim3(256), 0, s, (const double2*)A, N, Wp, (int)j0, p, i, nblk, hs,
                    (const double2*)slots, st, g, ng, partE)); WTBG_COUNT(ctx, 1);
    }
    CKL("tridiagonal panel");
    const long long k0 = j0 + jb;
    if (k0 < N) {
      const int il = (int)(j0 + jb - 1);
      CK(launch_pdl(k_wfix_last, dim3((int)((N - k0 + RB - 1) / RB)), dim3(RB), 0, s, (const double2*)A, N, Wp, jb - 1, il,
                    k0, (const ColState*)st)); WTBG_COUNT(ctx, 1);
      const long long T = (N - k0 + TB - 1) / TB;
      const long long ntile = T * (T + 1) / 2;
      if (prof) cudaEventRecord(ctx->evpool[evh + 2 * (j0 / NB)], s);
      CK(launch_pdl(k_her2k, dim3((unsigned)ntile), dim3(256), HER2K_SMEM, s, A, N, (const double2*)Wp,
                    (const double2*)A, (int)j0, jb, (int)k0)); WTBG_COUNT(ctx, 1);
      if (prof) cudaEventRecord(ctx->evpool[evh + 2 * (j0 / NB) + 1], s);
      CKL("k_her2k");
    }
  }
  k_last_diag<<<1, 1, 0, s>>>(A, N, d); WTBG_COUNT(ctx, 1);
  CKL("k_last_diag");
  if (prof) {
    cudaEventRecord(ctx->evpool[evt + 1], s);
    CK(cudaEventSynchronize(ctx->evpool[evt + 1]));
    float tt = 0.f;
    CK(cudaEventElapsedTime(&tt, ctx->evpool[evt], ctx->evpool[evt + 1]));
    ctx->stats.tri_ms += tt;
    for (long long j0 = 0; j0 < N - 1; j0 += NB) {
      const int jb = (int)((N - 1 - j0) < NB ? (N - 1 - j0) : NB);
      const long long k0 = j0 + jb;
      if (k0 >= N) continue;
      CK(cudaEventElapsedTime(&tt, ctx->evpool[evh + 2 * (j0 / NB)], ctx->evpool[evh + 2 * (j0 / NB) + 1]));
      const double nt = (double)(N - k0);
      ctx->stats.her2k_ms += tt;
      ctx->stats.her2k_flops += nt * (nt + 1.0) * 0.5 * 16.0 * (double)jb;   // 2 rank-jb products, 8 flop per cmac
      ctx->stats.her2k_launches += 1;
    }
    double ms = 0.0, bytes = 0.0;
    for (long long i = 0; i < N - 1; ++i) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ctx->evpool[2 * i], ctx->evpool[2 * i + 1]));
      ms += t;
      const double np = (double)(N - i - 1);
      bytes += np * (np + 1.0) * 0.5 * 16.0;   // lower triangle of the trailing matrix
    }
    ctx->stats.hemv_ms += ms;
    ctx->stats.hemv_bytes += bytes;
    ctx->stats.hemv_launches += N - 1;
  }
  return 0;
}
